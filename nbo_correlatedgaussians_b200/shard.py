"""One evaluation split across ranks (one process per GPU, torch.distributed).

The replacement of the reference's MPI split (source/outprod.f90:34-45 and
source/make_grad.f90:16-90: rows dealt round-robin to ranks, then two
MPI_REDUCE calls): each rank takes a contiguous range of the fused pass's
tiles, which balances the triangle of pairs by work instead of by rows.  Two
small all-reduces carry everything the ranks need from each other:

  1. rows (H C, S C) of each rank's share of H and S   (2 K doubles)
     -> every rank forms E, norm and GRADC from the sums;
  2. each rank's per-basis gradient sums g_H - E g_S   (part_stride(n) K doubles)
     -> every rank forms GRADA;
  3. the worst status code (one int), so that every rank raises together when
     some rank met a pair whose A_k + A_l' is not positive definite.

H and S themselves never cross the link.  The orchestration is independent of
where the shard work runs: ``DeviceShardOps`` calls the CUDA library, and the
test suite drives the same class on CPU ranks with an emulation of the kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
import torch.distributed as dist

from . import _lib
from .engine import Engine, _stream_ptr
from .problem import Problem


def tile_range(ntiles: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [t0, t1) of ``ntiles`` tiles for ``rank`` (sizes differ by
    at most one)."""
    q, r = divmod(ntiles, world)
    t0 = rank * q + min(rank, r)
    return t0, t0 + q + (1 if rank < r else 0)


class DeviceShardOps:
    """Shard steps on this rank's GPU through the C ABI (include/necg.h:
    necg_shard_tiles / _pairs / _grad / _finish)."""

    def __init__(self, prob: Problem, K_max: int | None = None, device=None, lc: int = 2, minw: int = 108):
        self.eng = Engine(prob, K_max=K_max, device=device)
        # every rank must number the tiles the same way: fixed chunk, not tuned
        _lib.check(self.eng.L.necg_set_symmetric(self.eng.h, 2, int(lc), int(minw)), "necg_set_symmetric")
        self.n, self.blk = prob.n, prob.blk
        self.ps = self.n * (self.n + 1) // 2 + 1 + 3 * self.n
        self.device = self.eng.device

    def tiles(self, K: int) -> int:
        n = ctypes.c_int(0)
        _lib.check(self.eng.L.necg_shard_tiles(self.eng.h, K, ctypes.byref(n)), "necg_shard_tiles")
        return n.value

    def pairs(self, x: torch.Tensor, K: int, t0: int, t1: int) -> torch.Tensor:
        rows = torch.empty(2 * K, dtype=torch.float64, device=self.device)
        _lib.check(self.eng.L.necg_shard_pairs(self.eng.h, K, x.data_ptr(), t0, t1, rows.data_ptr(),
                                               _stream_ptr(None)), "necg_shard_pairs")
        return rows

    def grad(self, x: torch.Tensor, K: int, rows: torch.Tensor, t0: int, t1: int):
        f = torch.empty(1, dtype=torch.float64, device=self.device)
        g = torch.empty(K * self.blk + K, dtype=torch.float64, device=self.device)
        sums = torch.empty(self.ps * K, dtype=torch.float64, device=self.device)
        _lib.check(self.eng.L.necg_shard_grad(self.eng.h, K, x.data_ptr(), rows.data_ptr(), t0, t1, f.data_ptr(),
                                              g.data_ptr(), sums.data_ptr(), _stream_ptr(None)), "necg_shard_grad")
        return f, g, sums

    def finish(self, x: torch.Tensor, K: int, sums: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
        _lib.check(self.eng.L.necg_shard_finish(self.eng.h, K, x.data_ptr(), sums.data_ptr(), g.data_ptr(),
                                                _stream_ptr(None)), "necg_shard_finish")
        return g

    def status(self) -> int:
        return self.eng.status()[0]


class ShardedEngine:
    """outprod(x) -> (f, g) with the pair work split over the process group;
    every rank returns the same f and g."""

    def __init__(self, ops, group=None):
        self.ops = ops
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def outprod_device(self, x: torch.Tensor, K: int):
        t0, t1 = tile_range(self.ops.tiles(K), self.rank, self.world)
        rows = self.ops.pairs(x, K, t0, t1)
        dist.all_reduce(rows, group=self.group)
        f, g, sums = self.ops.grad(x, K, rows, t0, t1)
        dist.all_reduce(sums, group=self.group)
        g = self.ops.finish(x, K, sums, g)
        return f, g

    def status(self) -> int:
        """Worst status code over the ranks (collective: every rank calls it)."""
        code = torch.tensor([int(self.ops.status())], dtype=torch.int64, device=self.ops.device)
        dist.all_reduce(code, op=dist.ReduceOp.MAX, group=self.group)
        return int(code.item())

    def outprod(self, x: np.ndarray) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, dtype=np.float64)
        K = x.size // (self.ops.blk + 1)
        xt = torch.from_numpy(x).to(self.ops.device)
        f, g = self.outprod_device(xt, K)
        code = self.status()
        if code == _lib.NECG_ERR_NOT_PD:
            raise np.linalg.LinAlgError("sharded outprod: A_k + A_l' is not positive definite for some basis pair")
        if code != _lib.NECG_OK:
            raise _lib.NecgError(code, "sharded outprod")
        return float(f.cpu()[0]), g.cpu().numpy()
