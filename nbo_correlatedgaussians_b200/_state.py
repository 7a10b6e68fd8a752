"""Bridge from the module state in ``shared`` to a cached ``Engine``."""
from __future__ import annotations

import hashlib

import numpy as np

from . import shared as sh
from .engine import Engine
from .problem import Problem

_cache: dict = {}


def problem_from_shared() -> Problem:
    if sh.ne <= 0 or sh.M <= 0 or sh.iv is None:
        raise RuntimeError("shared state is empty: call read_input first")
    return Problem(
        n=int(sh.ne), K=int(sh.M), efs=float(sh.efs),
        mass=np.asarray(sh.mass, dtype=np.float64), ncv=np.asarray(sh.ncv, dtype=np.float64),
        scvv=np.asarray(sh.scvv, dtype=np.float64),
        sml=np.ascontiguousarray(np.transpose(sh.sml, (2, 0, 1))),
        sms=np.ascontiguousarray(np.transpose(sh.sms, (2, 0, 1))),
        iv=np.asarray(sh.iv, dtype=np.float64), C=np.asarray(sh.C, dtype=np.float64))


def engine() -> Engine:
    """Engine for the current constants in ``shared`` (rebuilt when they change)."""
    p = problem_from_shared()
    hsh = hashlib.sha1()
    for a in (p.mass, p.ncv, p.scvv, p.sml, p.sms):
        hsh.update(np.ascontiguousarray(a).tobytes())
    key = (p.n, p.nst, p.K, p.efs, hsh.hexdigest())
    eng = _cache.get("engine")
    if eng is None or _cache.get("key") != key:
        if eng is not None:
            eng.close()
        eng = Engine(p, K_max=p.K)
        # the autotuner's setting for this (GPU, n, nst, K bucket): timed once, then cached
        from .autotune import tuned
        tuned(eng, p.x, p.K)
        _cache["engine"] = eng
        _cache["key"] = key
    return eng
