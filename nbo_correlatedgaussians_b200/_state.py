"""Bridge from the module state in ``shared`` to a cached ``Engine`` and to the
pinned host buffers the drop-in ``outprod`` copies through."""
from __future__ import annotations

import hashlib

import numpy as np
import torch

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


def _scalars() -> tuple:
    return int(sh.ne), int(sh.nst), int(sh.M), float(sh.efs)


def _constants() -> tuple:
    return sh.mass, sh.ncv, sh.scvv, sh.sml, sh.sms


def _unchanged() -> bool:
    """The constants in ``shared`` are those the cached engine was built from
    (a value comparison of the small constant arrays: a few microseconds)."""
    seen = _cache.get("seen")
    if seen is None or seen[0] != _scalars():
        return False
    return all(a is not None and np.shape(a) == b.shape and np.array_equal(a, b) for a, b in zip(_constants(), seen[1]))


def engine() -> Engine:
    """Engine for the current constants in ``shared`` (rebuilt when they change)."""
    eng = _cache.get("engine")
    if eng is not None and _unchanged():
        return eng
    p = problem_from_shared()
    hsh = hashlib.sha1()
    for a in (p.mass, p.ncv, p.scvv, p.sml, p.sms):
        hsh.update(np.ascontiguousarray(a).tobytes())
    key = (p.n, p.nst, p.K, p.efs, hsh.hexdigest())
    if eng is None or _cache.get("key") != key:
        if eng is not None:
            eng.close()
        _cache.pop("buffers", None)
        eng = Engine(p, K_max=p.K)
        # the autotuner's setting for this (GPU, n, nst, K bucket): timed once, then cached
        from .autotune import tuned
        tuned(eng, p.x, p.K)
        _cache["engine"] = eng
        _cache["key"] = key
    _cache["seen"] = (_scalars(), tuple(np.array(a, dtype=np.float64, copy=True) for a in _constants()))
    return eng


class Buffers:
    """Per-K buffers of the drop-in outprod: x, g, f, H, S on the device and
    pinned host copies of them, so that the copies run asynchronously on the
    engine's stream and the host waits once."""

    def __init__(self, eng: Engine, K: int):
        n = K * eng.blk + K
        dev = eng.device
        self.K = K
        self.x = torch.empty(n, dtype=torch.float64, device=dev)
        self.g = torch.empty(n, dtype=torch.float64, device=dev)
        self.f = torch.empty(1, dtype=torch.float64, device=dev)
        self.H = torch.empty((K, K), dtype=torch.float64, device=dev)
        self.S = torch.empty((K, K), dtype=torch.float64, device=dev)
        self.x_h = torch.empty(n, dtype=torch.float64).pin_memory()
        self.g_h = torch.empty(n, dtype=torch.float64).pin_memory()
        self.f_h = torch.empty(1, dtype=torch.float64).pin_memory()
        self.H_h = torch.zeros((K, K), dtype=torch.float64).pin_memory()
        self.S_h = torch.zeros((K, K), dtype=torch.float64).pin_memory()
        self.x_np, self.g_np = self.x_h.numpy(), self.g_h.numpy()
        self.H_np, self.S_np = self.H_h.numpy(), self.S_h.numpy()
        self.bound = False  # shared.H / shared.S are these pinned arrays


def buffers(eng: Engine, K: int) -> Buffers:
    b = _cache.get("buffers")
    if b is None or b.K != K:
        b = Buffers(eng, K)
        _cache["buffers"] = b
    return b
