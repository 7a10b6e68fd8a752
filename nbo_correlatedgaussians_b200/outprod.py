"""Drop-in ``outprod(x) -> (f, g)`` (python/outprod.py:20-76): the objective the
optimiser calls.  x = [iv, C] is copied to the GPU, H, S, the Rayleigh quotient
and the gradient are computed there, and f and a copy of g come back.  Like the
reference it updates shared.iv, shared.C, shared.grad and (when
shared.sync_matrices) shared.H and shared.S, which it fills in place as the
reference does (python/outprod.py:46-60).

All copies go through pinned host buffers on the engine's stream: x in, the
evaluation, then g, f (and H, S) out, and the host waits once.  The first call
binds shared.H and shared.S to pinned arrays so that later calls copy straight
into them."""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, _state
from . import shared as sh
from .engine import _stream_ptr


def outprod(x: np.ndarray) -> tuple[float, np.ndarray]:
    x = np.ascontiguousarray(x, dtype=np.float64)
    sh.iv[:] = x[:sh.siv]
    sh.C[:] = x[sh.siv:]
    eng = _state.engine()
    K = sh.M
    b = _state.buffers(eng, K)
    if x.size != b.x.numel():
        raise ValueError(f"x has {x.size} entries, expected {b.x.numel()}")
    stream = torch.cuda.current_stream(eng.device)
    b.x_np[:] = x
    b.x.copy_(b.x_h, non_blocking=True)
    sync = bool(sh.sync_matrices)
    rc = eng.L.necg_outprod(eng.h, K, b.x.data_ptr(), b.f.data_ptr(), b.g.data_ptr(),
                            b.H.data_ptr() if sync else None, b.S.data_ptr() if sync else None,
                            _stream_ptr(stream))
    _lib.check(rc, "necg_outprod")
    b.g_h.copy_(b.g, non_blocking=True)
    b.f_h.copy_(b.f, non_blocking=True)
    if sync:
        b.H_h.copy_(b.H, non_blocking=True)
        b.S_h.copy_(b.S, non_blocking=True)
    stream.synchronize()
    eng.raise_status("outprod")
    f = float(b.f_h[0])
    g = b.g_np.copy()
    if sync:
        if not b.bound:  # from now on the copies land in shared.H and shared.S directly
            sh.H, sh.S = b.H_np, b.S_np
            b.bound = True
        for name, host in (("H", b.H_np), ("S", b.S_np)):
            cur = getattr(sh, name)
            if cur is host:
                continue
            if isinstance(cur, np.ndarray) and cur.shape == host.shape and cur.dtype == host.dtype:
                cur[:] = host  # an array the caller put there since: filled in place
            else:
                setattr(sh, name, host)
    if isinstance(sh.grad, np.ndarray) and sh.grad.shape == g.shape:
        sh.grad[:] = g
    else:
        sh.grad = g.copy()
    return f, g
