"""The sharded evaluation (nbo_correlatedgaussians_b200.shard) on CPU ranks:
world_size 2 and 3 with the gloo backend, each rank running its contiguous
share of the fused tiles through the host emulation of the kernels, with the
same two all-reduces the GPU path uses.  Every rank must end with the same
(E, g), equal to the oracle's."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, system, K, lc, out):
    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.dirname(HERE))
    import torch.distributed as dist
    from emu.emu import EmuShardOps
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.shard import ShardedEngine
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        p = synth.make_problem(system, K, 5 * K)
        p.C = np.random.default_rng(K).normal(size=K)
        se = ShardedEngine(EmuShardOps(p, lc))
        f, g = se.outprod(p.x)
        out[rank] = (f, g)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("system,K,lc,world", [("He", 70, 2, 2), ("H2", 45, 3, 3), ("LiH", 36, 4, 2)])
def test_sharded_matches_oracle(system, K, lc, world):
    from oracle.oracle import Oracle
    from nbo_correlatedgaussians_b200 import synth
    from _util import TOL_E, TOL_G, normwise
    from emu.emu import build
    build()  # once, before the ranks start
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, system, K, lc, out)) for r in range(world)]
    for q in ps:
        q.start()
    for q in ps:
        q.join(timeout=300)
        assert q.exitcode == 0
    p = synth.make_problem(system, K, 5 * K)
    p.C = np.random.default_rng(K).normal(size=K)
    fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=4)
    f0, g0 = out[0]
    for r in range(world):
        f, g = out[r]
        assert f == f0 and np.array_equal(g, g0)  # identical on every rank
    assert abs(f0 - fo) < TOL_E and normwise(g0, go) < TOL_G


def test_tile_ranges_cover_once():
    from nbo_correlatedgaussians_b200.shard import tile_range
    for nt in (0, 1, 7, 100, 8448):
        for world in (1, 2, 3, 8):
            rs = [tile_range(nt, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == nt
            assert all(rs[i][1] == rs[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in rs]
            assert max(sizes) - min(sizes) <= 1


def _rank_not_pd(rank, world, port, out):
    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.dirname(HERE))
    import torch.distributed as dist
    from emu.emu import EmuShardOps
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.shard import ShardedEngine, tile_range
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        p = synth.make_problem("LiH", 36, 77)
        ops = EmuShardOps(p, 2)
        se = ShardedEngine(ops)
        bad = p.copy()
        j = p.K - 1  # L_j = 0: only the pair (j, j) is singular
        bad.iv[j * p.blk:j * p.blk + p.svh] = 0.0
        t0, t1 = tile_range(ops.tiles(p.K), rank, world)
        raised = False
        try:
            se.outprod(bad.x)
        except np.linalg.LinAlgError:
            raised = True
        own = ops.status()  # this rank's own status, before the next call resets it
        f, g = se.outprod(p.x)
        out[rank] = (raised, own, (t0, t1), f, g)
    finally:
        dist.destroy_process_group()


def test_sharded_not_positive_definite_on_one_rank_raises_on_all():
    """Only rank 1's tiles hold the singular pair (j, j): its own status says so,
    rank 0's does not, and the status all-reduce makes both ranks raise
    LinAlgError (python/matel.py:93 raises it from np.linalg.inv); the next
    evaluation on a good input then succeeds on both ranks."""
    from oracle.oracle import Oracle
    from nbo_correlatedgaussians_b200 import _lib, synth
    from _util import TOL_E, TOL_G, normwise
    from emu.emu import build
    build()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    ps = [ctx.Process(target=_rank_not_pd, args=(r, 2, port, out)) for r in range(2)]
    for q in ps:
        q.start()
    for q in ps:
        q.join(timeout=300)
        assert q.exitcode == 0
    p = synth.make_problem("LiH", 36, 77)
    fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=4)
    assert out[0][1] == _lib.NECG_OK and out[1][1] == _lib.NECG_ERR_NOT_PD
    for r in range(2):
        raised, _, _, f, g = out[r]
        assert raised
        assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
