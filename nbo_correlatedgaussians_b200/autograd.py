"""The Rayleigh quotient E(iv, C) as a torch.autograd.Function.

forward  -- the energy tiles build H and S and E = C^T H C / C^T S C on the
            device (python/outprod.py:46-68); H, S and [E, norm] are kept
            (K^2 + 2 doubles, no per-pair K^2 n^2 intermediates).
backward -- the hand-written gradient kernel (necg_make_grad_dev): it
            recomputes the pair intermediates tile by tile and contracts them
            with C on the fly (python/make_grad.py:18-90); autodiff is not used.
The result is grad_output * dE/d(iv, C), split into the two inputs.
"""
from __future__ import annotations

import torch

from .engine import Engine


class EnergyFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, iv: torch.Tensor, C: torch.Tensor, engine: Engine):
        iv = iv.detach().contiguous()
        C = C.detach().contiguous()
        H, S, _, _, en = engine.build_matrices(iv, C, K=C.numel(), parts=False, check=False)
        ctx.engine = engine
        ctx.save_for_backward(iv, C, H, S, en)
        return en[0].clone()

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        iv, C, H, S, en = ctx.saved_tensors
        eng = ctx.engine
        g = eng.make_grad_dev(iv, C, H, S, en)
        siv = iv.numel()
        gi = grad_out * g[:siv]
        gc = grad_out * g[siv:]
        return gi.view_as(iv), gc.view_as(C), None


def energy(iv: torch.Tensor, C: torch.Tensor, engine: Engine) -> torch.Tensor:
    """E(iv, C) with the hand-written gradient as its backward."""
    return EnergyFn.apply(iv, C, engine)
