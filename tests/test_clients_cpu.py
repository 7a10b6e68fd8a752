"""The cross-process front end of the serving loop (serve.Endpoint and
clients.RemoteRun / client_worker) on CPU, against a stand-in for Server that
evaluates a quadratic: the request plumbing, error propagation, the closing of
dropped runs and the client processes of the load generator."""
import multiprocessing as mp
import threading

import numpy as np
import pytest

from nbo_correlatedgaussians_b200 import synth
from nbo_correlatedgaussians_b200.clients import RemoteRun, client_worker
from nbo_correlatedgaussians_b200.serve import Endpoint


class _Run:
    def __init__(self, rid, problem):
        self.id = rid
        self.problem = problem


class FakeServer:
    """open_run / evaluate / close_run with Server's signatures: f = |x - 1|^2 / 2,
    g = x - 1; a NaN in x raises LinAlgError; K = 0 is refused at admission."""

    def __init__(self):
        self.lock = threading.Lock()
        self.open, self.closed, self.evals = {}, [], 0
        self.next_id = 0

    def open_run(self, problem, timeout=None):
        if problem.K == 0:
            raise MemoryError("refused")
        with self.lock:
            run = _Run(self.next_id, problem)
            self.next_id += 1
            self.open[run.id] = run
        return run

    def evaluate(self, run, x, timeout=None):
        assert run.id in self.open
        if np.isnan(x).any():
            raise np.linalg.LinAlgError("A_k + A_l' is not positive definite for some basis pair")
        with self.lock:
            self.evals += 1
        d = np.asarray(x, dtype=np.float64) - 1.0
        return 0.5 * float(d @ d), d.copy()

    def close_run(self, run):
        with self.lock:
            if self.open.pop(run.id, None) is not None:
                self.closed.append(run.id)


@pytest.fixture
def endpoint():
    srv = FakeServer()
    ep = Endpoint(srv)
    yield srv, ep
    ep.close()


def test_round_trip_and_errors(endpoint):
    srv, ep = endpoint
    p = synth.make_problem("He", 8, 3)
    run = RemoteRun(ep.address, ep.authkey, p)
    x = np.random.default_rng(0).normal(size=p.x.size)
    f, g = run.evaluate(x)
    assert f == 0.5 * float((x - 1) @ (x - 1)) and np.array_equal(g, x - 1)
    bad = x.copy()
    bad[3] = np.nan
    with pytest.raises(np.linalg.LinAlgError):
        run.evaluate(bad)
    f2, _ = run.evaluate(x)  # the run stays usable after an error
    assert f2 == f
    run.close()
    assert srv.closed == [run.id] and not srv.open


def test_admission_error_and_wrong_key(endpoint):
    srv, ep = endpoint
    p = synth.make_problem("He", 8, 3)
    p.K = 0
    with pytest.raises(MemoryError):
        RemoteRun(ep.address, ep.authkey, p)
    from multiprocessing import AuthenticationError
    with pytest.raises(AuthenticationError):
        RemoteRun(ep.address, b"not the key", synth.make_problem("He", 8, 3))
    assert not srv.open


def test_malformed_requests(endpoint):
    srv, ep = endpoint
    run = RemoteRun(ep.address, ep.authkey, synth.make_problem("He", 8, 3))
    with pytest.raises(ValueError):
        run._call(b"Z")  # unknown request
    with pytest.raises(RuntimeError):
        run._call(b"O" + __import__("pickle").dumps((synth.make_problem("He", 8, 3), None)))  # second open
    f, _ = run.evaluate(np.ones(run_size := synth.make_problem("He", 8, 3).x.size))
    assert f == 0.0 and run_size > 0
    run.close()
    assert srv.closed == [run.id]


def test_dropped_connection_closes_the_run(endpoint):
    srv, ep = endpoint
    run = RemoteRun(ep.address, ep.authkey, synth.make_problem("H2", 6, 1))
    run.conn.close()  # the client goes away without closing
    for _ in range(200):
        if srv.closed:
            break
        threading.Event().wait(0.01)
    assert srv.closed == [run.id]


@pytest.mark.parametrize("saturate", [True, False])
def test_client_processes(endpoint, saturate):
    srv, ep = endpoint
    probs = [synth.make_problem(("He", "H2")[j % 2], 6 + j, 40 + j) for j in range(6)]
    ctx = mp.get_context("spawn")
    nproc = 2
    ready = ctx.Barrier(nproc + 1)
    gate = ctx.Barrier(len(probs) + 1) if saturate else None
    go, t0, q = ctx.Event(), ctx.Value("d", 0.0), ctx.Queue()
    jobs = [[(j, p, 0.01 * j) for j, p in enumerate(probs) if j % nproc == w] for w in range(nproc)]
    ws = [ctx.Process(target=client_worker, args=(ep.address, ep.authkey, jobs[w], 5, ready, gate, go, t0, q),
                      daemon=True) for w in range(nproc)]
    for w in ws:
        w.start()
    ready.wait(timeout=120)
    if gate is not None:
        gate.wait(timeout=120)
    else:
        import time
        t0.value = time.time()
        go.set()
    res = [q.get(timeout=120) for _ in ws]
    for w in ws:
        w.join(timeout=60)
    assert all(not r["errors"] for r in res)
    counts = {j: n for r in res for j, n in r["evals"].items()}
    assert sorted(counts) == list(range(len(probs)))
    assert all(n >= 1 for n in counts.values())  # TNC may pass maxfun within an iteration
    assert sum(counts.values()) == srv.evals
    assert sorted(srv.closed) == list(range(len(probs))) and not srv.open
