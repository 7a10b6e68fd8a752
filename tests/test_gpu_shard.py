"""The sharded evaluation's device steps (necg_shard_pairs / _grad / _finish)
on one GPU: virtual ranks in one process, each with its own handle and tile
range, the all-reduces done by summing their outputs; and ShardedEngine over
a one-rank NCCL group.  Against the single-call path and the oracle."""
import socket

import numpy as np
import pytest

from oracle.oracle import Oracle
from _util import TOL_E, TOL_G, normwise

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("system,K,world", [("He", 90, 2), ("H2", 70, 3), ("LiH", 64, 2), ("LiH", 40, 5)])
def test_virtual_ranks_match_single_call(torch_cuda, system, K, world):
    torch = torch_cuda
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.engine import Engine
    from nbo_correlatedgaussians_b200.shard import DeviceShardOps, tile_range
    p = synth.make_problem(system, K, 13 * K)
    p.C = np.random.default_rng(K).normal(size=K)
    x = torch.from_numpy(p.x).cuda()
    ops = [DeviceShardOps(p) for _ in range(world)]
    nt = ops[0].tiles(K)
    assert all(o.tiles(K) == nt for o in ops)
    rngs = [tile_range(nt, r, world) for r in range(world)]
    rows = sum(o.pairs(x, K, *rg) for o, rg in zip(ops, rngs))  # all-reduce 1
    outs = [o.grad(x, K, rows.clone(), *rg) for o, rg in zip(ops, rngs)]
    sums = sum(s for _, _, s in outs)  # all-reduce 2
    res = []
    for o, (f, g, _) in zip(ops, outs):
        g = o.finish(x, K, sums.clone(), g)
        torch.cuda.synchronize()
        assert o.status() == 0
        res.append((float(f.item()), g.cpu().numpy()))
    for f, g in res[1:]:
        assert f == res[0][0] and np.array_equal(g, res[0][1])
    f, g = res[0]
    fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
    assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
    fs, gs = Engine(p).outprod(p.x)
    assert abs(f - fs) < 1e-12 * abs(fs) and normwise(g, gs) < 1e-12


def test_sharded_engine_one_rank_nccl(torch_cuda):
    import torch.distributed as dist
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.shard import DeviceShardOps, ShardedEngine
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        p = synth.make_problem("LiH", 48, 9)
        p.C = np.random.default_rng(3).normal(size=p.K)
        se = ShardedEngine(DeviceShardOps(p))
        f, g = se.outprod(p.x)
        fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
        assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
        bad = p.copy()
        bad.iv[2 * p.blk:2 * p.blk + p.svh] = 0.0
        with pytest.raises(np.linalg.LinAlgError):
            se.outprod(bad.x)
        f2, g2 = se.outprod(p.x)  # usable after the error
        assert f2 == f and np.array_equal(g2, g)
    finally:
        dist.destroy_process_group()
