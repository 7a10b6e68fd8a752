"""Drop-in ``make_grad(eng, norm)`` (python/make_grad.py:18-90): gradient of the
Rayleigh quotient for the parameters and matrices in ``shared``, stored in
``shared.grad`` as [GRADA, GRADC].  The per-pair derivatives are contracted with
C inside the kernels, so the dense DH/DS matrices of the reference are not built."""
from __future__ import annotations

from . import _state
from . import shared as sh


def make_grad(eng: float, norm: float) -> None:
    g = _state.engine().make_grad(sh.iv, sh.C, sh.H, sh.S, eng, norm)
    sh.grad = g.cpu().numpy()
    sh.GRADA = sh.grad[:sh.siv]
    sh.GRADC = sh.grad[sh.siv:]
