"""Drop-in ``outprod(x) -> (f, g)`` (python/outprod.py:20-76): the objective the
optimiser calls.  x = [iv, C] is copied to the GPU, H, S, the Rayleigh quotient
and the gradient are computed there, and f and a copy of g come back.  Like the
reference it updates shared.iv, shared.C, shared.grad and (when
shared.sync_matrices) shared.H and shared.S."""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, _state
from . import shared as sh


def outprod(x: np.ndarray) -> tuple[float, np.ndarray]:
    x = np.ascontiguousarray(x, dtype=np.float64)
    sh.iv[:] = x[:sh.siv]
    sh.C[:] = x[sh.siv:]
    eng = _state.engine()
    if not sh.sync_matrices:
        f, g = eng.outprod(x)
    else:
        K = sh.M
        H = torch.empty((K, K), dtype=torch.float64, device=eng.device)
        S = torch.empty_like(H)
        ft, gt = eng.outprod_device(torch.from_numpy(x).to(eng.device), K, H=H, S=S)
        eng.raise_status("outprod")
        f = float(ft.item())
        g = gt.cpu().numpy()
        sh.H = H.cpu().numpy()
        sh.S = S.cpu().numpy()
    sh.grad = g.copy()
    return f, g
