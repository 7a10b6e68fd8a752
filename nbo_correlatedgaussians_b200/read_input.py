"""Drop-in ``read_input`` (python/read_input.py:16-157): parse an oldquit.dat
format file and populate ``shared`` in the reference's layouts."""
from __future__ import annotations

import numpy as np

from . import shared as sh
from .problem import read_oldquit
from .utils import biout


def read_input(filename: str = "oldquit.dat") -> None:
    try:
        p = read_oldquit(filename)
    except OSError:
        biout(f"Could not open input file: {filename}")
        raise
    sh.M, sh.ne, sh.nst, sh.efs = p.K, p.n, p.nst, p.efs
    sh.skp = 3 * p.n
    sh.svh = p.n * (p.n + 1) // 2
    sh.siv = sh.M * (sh.svh + sh.skp)
    sh.mass = p.mass.copy()
    sh.ncv = p.ncv.copy()
    sh.iv = p.iv.copy()
    sh.C = p.C.copy()
    sh.scvv = p.scvv.copy()
    sh.sml = np.ascontiguousarray(np.transpose(p.sml, (1, 2, 0)))
    sh.sms = np.ascontiguousarray(np.transpose(p.sms, (1, 2, 0)))
    for name in ("H", "S", "Kinetic", "Potential"):
        setattr(sh, name, np.zeros((sh.M, sh.M)))
    sh.grad = np.zeros(sh.siv + sh.M)
