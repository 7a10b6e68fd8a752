"""Autograd Function, batched persistent launch (with CUDA graph replay) and
the continuous-batching server, on the GPU."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from oracle.oracle import Oracle  # noqa: E402
from _util import TOL_E, TOL_G, normwise  # noqa: E402


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def _mixed(seed=0):
    from nbo_correlatedgaussians_b200 import synth
    return [synth.make_problem("He", 40, seed + 1), synth.make_problem("H2", 70, seed + 2),
            synth.make_problem("LiH", 33, seed + 3), synth.make_problem("He", 17, seed + 4),
            synth.make_problem("H2", 9, seed + 5)]


def test_autograd_backward_is_the_gradient_kernel(torch_cuda):
    torch = torch_cuda
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.autograd import energy
    from nbo_correlatedgaussians_b200.engine import Engine
    p = synth.make_problem("H2", 96, 2)
    p.C = np.random.default_rng(5).normal(size=p.K)
    eng = Engine(p)
    iv = torch.tensor(p.iv, device="cuda", requires_grad=True)
    C = torch.tensor(p.C, device="cuda", requires_grad=True)
    E = energy(iv, C, eng)
    (3.0 * E).backward()
    fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
    assert abs(float(E.detach()) - fo) < TOL_E
    g = torch.cat([iv.grad, C.grad]).cpu().numpy()
    assert normwise(g, 3.0 * go) < TOL_G


def test_autograd_central_differences(torch_cuda):
    """H2 K=2048 (n=3, nst=4, seed 2): E through the autograd Function, its
    gradient (the hand-written backward) against the oracle's gradel-based
    gradient (1e-9 norm-wise) and against finite differences on 64 random
    parameters (indices from seed 2): central h = 1e-6 (the requested check;
    round-off in E limits it to ~1e-6 relative, so it is bounded at 1e-5) and a
    5-point stencil with h = 1e-4 (bounded at 1e-7).  C is random (seed 7): with
    C = 1/K the gradient components are small and the FD quotients noisier."""
    torch = torch_cuda
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.autograd import energy
    from nbo_correlatedgaussians_b200.engine import Engine
    p = synth.workload("h2_k2048")
    p.C = np.random.default_rng(7).normal(size=p.K)
    eng = Engine(p)
    x = torch.tensor(p.x, device="cuda")
    siv = p.siv
    xg = x.clone().requires_grad_(True)
    E = energy(xg[:siv], xg[siv:], eng)
    E.backward()
    g = xg.grad.cpu().numpy()
    import os
    _, go = Oracle.from_problem(p).outprod(p.x, nthreads=len(os.sched_getaffinity(0)))
    assert normwise(g, go) < TOL_G
    idx = np.random.default_rng(2).choice(p.x.size, 64, replace=False)

    def e_at(i, dx):
        xp = x.clone()
        xp[i] += dx
        return float(energy(xp[:siv], xp[siv:], eng))

    h = 1e-6
    fd2 = np.array([(e_at(i, h) - e_at(i, -h)) / (2 * h) for i in idx])
    h5 = 1e-4
    fd5 = np.array([(e_at(i, -2 * h5) - 8 * e_at(i, -h5) + 8 * e_at(i, h5) - e_at(i, 2 * h5)) / (12 * h5)
                    for i in idx])
    scale = np.max(np.abs(g[idx]))
    assert np.max(np.abs(fd2 - g[idx])) / scale < 1e-5
    assert np.max(np.abs(fd5 - g[idx])) / scale < 1e-7


def test_batch_matches_single_and_is_order_independent(torch_cuda):
    from nbo_correlatedgaussians_b200.batch import BatchEngine
    from nbo_correlatedgaussians_b200.engine import Engine
    probs = _mixed()
    be = BatchEngine(probs, tune=False)
    be.plan()
    be.step(graph=False)
    be.check()
    res = [be.results(i) for i in range(len(probs))]
    for p, (f, g) in zip(probs, res):
        fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
        assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
        fs, gs = Engine(p).outprod(p.x)
        assert abs(f - fs) < 1e-12 * abs(fs) and normwise(g, gs) < 1e-12
    # one instance alone, then a different subset in another order: bitwise equal
    be.plan([2])
    be.step(graph=True)
    be.check()
    f2, g2 = be.results(2)
    assert f2 == res[2][0] and np.array_equal(g2, res[2][1])
    be.plan([4, 2, 0])
    be.step(graph=True)
    be.check()
    for i in (4, 2, 0):
        fi, gi = be.results(i)
        assert fi == res[i][0] and np.array_equal(gi, res[i][1])


def test_batch_modes_fused_and_ordered(torch_cuda):
    """A plan whose instances all have symmetry sets closed under inverse runs
    the fused step; adding one instance without that property switches the
    whole plan to the ordered step (and its own CUDA graph).  Both against the
    oracle, and the fused results are bitwise the same before and after."""
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.batch import BatchEngine
    probs = _mixed(30)
    r = synth.make_problem("H2", 24, 31)  # a lone non-involutory map: no inverse in the set
    M = np.array([[1.0, 0, 0], [0, 0, 1.0], [0, 1.0, 0]]) @ np.array([[1.0, 0, 0], [1.0, 1.0, 0], [0, 0, 1.0]])
    r.sml = np.stack([np.eye(3), M])
    r.sms = np.stack([np.eye(9), np.kron(np.linalg.inv(M), np.eye(3))])
    r.scvv = np.array([0.5, 0.5])
    be = BatchEngine(probs + [r], tune=False)
    res = {}
    for active in (list(range(len(probs))), list(range(len(probs) + 1)), list(range(len(probs)))):
        be.plan(active)
        be.step(graph=True)
        be.check()
        for i in active:
            p = (probs + [r])[i]
            f, g = be.results(i)
            fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
            assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
            if len(active) == len(probs):
                if i in res:
                    assert f == res[i][0] and np.array_equal(g, res[i][1])
                res[i] = (f, g)


def test_batch_split_terms(torch_cuda):
    """Instances whose handles split the fused pass's symmetry terms
    (necg_set_splits) in the batched one-warp step, mixed with unsplit ones:
    against the oracle and the per-call path, and bitwise the same alone and
    in the mix."""
    from nbo_correlatedgaussians_b200 import _lib
    from nbo_correlatedgaussians_b200.batch import BatchEngine
    probs = _mixed(50)
    be = BatchEngine(probs, tune=False)
    splits = [2, 1, 3, 2, 4]
    for eng, p, npc in zip(be.engines, probs, splits):
        assert eng.L.necg_set_symmetric(eng.h, 2, 2, 118) == _lib.NECG_OK
        assert eng.L.necg_set_splits(eng.h, min(npc, p.nst)) == _lib.NECG_OK
    be.plan()
    be.step(graph=True)
    be.check()
    res = [be.results(i) for i in range(len(probs))]
    for i, (p, (f, g)) in enumerate(zip(probs, res)):
        fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
        assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
        fs, gs = be.engines[i].outprod(p.x)
        assert abs(f - fs) < 1e-12 * abs(fs) and normwise(g, gs) < 1e-12
    be.plan([3, 0])
    be.step(graph=True)
    be.check()
    for i in (3, 0):
        fi, gi = be.results(i)
        assert fi == res[i][0] and np.array_equal(gi, res[i][1])


@pytest.mark.parametrize("big", [False, True])
def test_batch_failing_instance_is_isolated(torch_cuda, big):
    """One instance with a singular A_k + A_l' in a batched step: its status is
    NOT_PD and the other instances' results are unaffected (one-warp step for a
    small plan; lockstep step when large instances fill the SMs)."""
    from nbo_correlatedgaussians_b200 import _lib, synth
    from nbo_correlatedgaussians_b200.batch import BatchEngine
    probs = _mixed(40)
    if big:
        probs += [synth.make_problem("LiH", 700, 41), synth.make_problem("H2", 900, 42)]
    bad = probs[2].copy()
    bad.iv[3 * bad.blk:3 * bad.blk + bad.svh] = 0.0
    allp = probs + [bad]
    be = BatchEngine(allp, tune=False)
    be.plan()
    be.step(graph=True)
    codes = be.status()
    assert codes[-1] == _lib.NECG_ERR_NOT_PD
    assert all(c == _lib.NECG_OK for c in codes[:-1])
    for i, p in enumerate(probs):
        f, g = be.results(i)
        fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=16)
        assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G


def test_batch_graph_replay_tracks_new_inputs(torch_cuda):
    from nbo_correlatedgaussians_b200.batch import BatchEngine
    probs = _mixed(10)
    be = BatchEngine(probs, tune=False)
    be.plan()
    be.step(graph=True)
    be.check()
    rng = np.random.default_rng(1)
    for i, p in enumerate(probs):
        x = p.x.copy()
        x[p.siv:] = rng.normal(size=p.K)
        be.set_x(i, x)
        p.C = x[p.siv:]
    be.step(graph=True)
    be.check()
    for i, p in enumerate(probs):
        f, g = be.results(i)
        fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
        assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G


def test_server_results_alone_and_in_mix(torch_cuda):
    from nbo_correlatedgaussians_b200.serve import Server
    probs = _mixed(20)
    rng = np.random.default_rng(3)
    xs = [[p.x + 1e-3 * rng.normal(size=p.x.size) for _ in range(3)] for p in probs]
    # alone
    alone = []
    with Server(budget_bytes=8e9, max_slots=8, tune=False) as srv:
        for p, xl in zip(probs, xs):
            run = srv.open_run(p)
            alone.append([srv.evaluate(run, x) for x in xl])
            srv.close_run(run)
    # all runs concurrently
    mix = [None] * len(probs)
    with Server(budget_bytes=8e9, max_slots=8, tune=False) as srv:
        def client(i):
            run = srv.open_run(probs[i])
            mix[i] = [srv.evaluate(run, x) for x in xs[i]]
            srv.close_run(run)
        th = [threading.Thread(target=client, args=(i,)) for i in range(len(probs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        st = srv.stats()
    assert st["requests"] == 15 and st["p99_ms"] >= st["p50_ms"] > 0
    for a, m in zip(alone, mix):
        for (fa, ga), (fm, gm) in zip(a, m):
            assert fa == fm and np.array_equal(ga, gm)


def test_server_admission_under_budget(torch_cuda):
    """A budget that fits one run at a time: runs are admitted one after another
    as earlier runs close, and every run completes."""
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.serve import Server, workspace_estimate
    probs = [synth.make_problem("He", 64, 30 + i) for i in range(3)]
    budget = 1.5 * max(workspace_estimate(p) for p in probs)
    order = []
    with Server(budget_bytes=budget, max_slots=4, tune=False) as srv:
        def client(i):
            run = srv.open_run(probs[i])
            order.append(("in", i, srv.used))
            srv.evaluate(run, probs[i].x)
            order.append(("out", i))
            srv.close_run(run)
        th = [threading.Thread(target=client, args=(i,)) for i in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    assert all(u <= budget for tag, *rest in order if tag == "in" for u in [rest[1]])
    assert len([o for o in order if o[0] == "out"]) == 3
    with pytest.raises(MemoryError):
        with Server(budget_bytes=1e3, max_slots=1, tune=False) as srv:
            srv.open_run(probs[0])


def test_server_admission_failure_releases_the_reservation(torch_cuda):
    """A run whose device state cannot be built (here a problem the library
    rejects at creation: no symmetry terms) fails in open_run, and its budget
    and slot go back, so the next run is admitted and served."""
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.serve import Server, workspace_estimate
    good = synth.make_problem("He", 40, 51)
    bad = synth.make_problem("He", 40, 52)
    bad.sml, bad.sms, bad.scvv = bad.sml[:0], bad.sms[:0], bad.scvv[:0]
    budget = 1.2 * max(workspace_estimate(good), 1)
    with Server(budget_bytes=budget, max_slots=1, tune=False) as srv:
        with pytest.raises(Exception):
            srv.open_run(bad, timeout=60)
        assert srv.used == 0 and srv.pending_slots == 0
        run = srv.open_run(good, timeout=60)
        f, g = srv.evaluate(run, good.x, timeout=60)
        fo, go = Oracle.from_problem(good).outprod(good.x, nthreads=8)
        assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
        srv.close_run(run)


def test_server_endpoint_remote_run(torch_cuda):
    """A run driven through the cross-process front end (serve.Endpoint,
    clients.RemoteRun) gets the same f and g as an in-process run of the same
    server, and a failing evaluation comes back as LinAlgError."""
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.clients import RemoteRun
    from nbo_correlatedgaussians_b200.serve import Endpoint, Server
    p = synth.make_problem("LiH", 24, 61)
    with Server(max_slots=4, tune=False) as srv:
        ep = Endpoint(srv)
        try:
            rr = RemoteRun(ep.address, ep.authkey, p, timeout=60)
            f, g = rr.evaluate(p.x)
            local = srv.open_run(p, timeout=60)
            fl, gl = srv.evaluate(local, p.x, timeout=60)
            assert f == fl and np.array_equal(g, gl)
            fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
            assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
            bad = p.x.copy()
            bad[2 * p.blk:2 * p.blk + p.svh] = 0.0
            with pytest.raises(np.linalg.LinAlgError):
                rr.evaluate(bad)
            f2, _ = rr.evaluate(p.x)
            assert f2 == f
            rr.close()
            srv.close_run(local)
        finally:
            ep.close()


def test_server_faults_injected_on_the_host(torch_cuda):
    """Malformed and failing requests do not disturb the server: a wrong-sized
    x is refused at submission, a NaN parameter comes back as a status error
    (the run stays usable), a non-positive-definite pair as LinAlgError, and a
    request still queued when its run is closed fails instead of hanging."""
    from nbo_correlatedgaussians_b200 import _lib, synth
    from nbo_correlatedgaussians_b200.serve import Request, Server
    p = synth.make_problem("H2", 40, 71)
    with Server(max_slots=4, tune=False) as srv:
        run = srv.open_run(p, timeout=60)
        f0, g0 = srv.evaluate(run, p.x, timeout=60)
        with pytest.raises(ValueError):
            srv.evaluate(run, p.x[:-1])
        bad = p.x.copy()
        bad[5] = np.nan
        with pytest.raises((_lib.NecgError, np.linalg.LinAlgError)):
            srv.evaluate(run, bad, timeout=60)
        npd = p.x.copy()
        npd[3 * p.blk:3 * p.blk + p.svh] = 0.0
        with pytest.raises(np.linalg.LinAlgError):
            srv.evaluate(run, npd, timeout=60)
        f1, g1 = srv.evaluate(run, p.x, timeout=60)
        assert f1 == f0 and np.array_equal(g1, g0)
        # a request that no step has taken yet when the run closes
        with srv.lock:
            held = list(srv.free_batches)
            srv.free_batches.clear()  # hold the step loop: no plan is free
            req = Request(run, p.x.copy())
            srv.pending.append(req)
        closer = threading.Thread(target=srv.close_run, args=(run,))
        closer.start()
        assert req.done.wait(60) and isinstance(req.error, RuntimeError)
        closer.join(60)
        with srv.lock:
            srv.free_batches.extend(held)
            srv.lock.notify_all()
        with pytest.raises(RuntimeError):
            srv.evaluate(run, p.x)
