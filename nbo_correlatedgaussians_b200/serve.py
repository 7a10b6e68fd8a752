"""Serving loop for many concurrent optimiser runs (continuous batching).

Each run is one basis being optimised by its own client (e.g. a truncated-Newton
minimiser calling ``evaluate(x)`` as its objective, the role outprod plays for
the reference's optimiser, python/necg.py:159-171 and source/tn.f).  The server:

* keeps each admitted run's state on the device: its ``Engine`` (bra/ket
  records, H, S, gradient partials for its K), its parameters x = [iv, C] and
  its outputs g, E;
* admits runs under an HBM budget and a slot count: a run that does not fit
  waits until earlier runs close and free their workspace;
* batches continuously: a worker thread takes every request that is ready,
  plans one batched step over those runs (all their tiles in one flattened
  queue) and launches it as a CUDA-graph replay.  Requests that arrive while a
  step is on the GPU go into the next step, which is launched at once behind
  it: two batch plans are used alternately, so up to two steps are in flight
  and the GPU does not wait for the host to deliver results.
* reports per-request latency (submit to result) and throughput.

Clients may be threads of this process (``open_run`` / ``evaluate``) or other
processes connected through an ``Endpoint`` (``clients.RemoteRun``); the
requests of both kinds go into the same steps.

Because every run's tiles and reductions are the same in any batch, a run's
results do not depend on which other runs share its steps.
"""
from __future__ import annotations

import collections
import pickle
import secrets
import struct
import threading
import time

import numpy as np
import torch

from . import _lib
from .clients import OP_CLOSE, OP_EVAL, OP_OPEN, REPLY_OK, encode_error
from .autotune import tuned
from .batch import Batch
from .engine import Engine
from .problem import Problem


def workspace_estimate(p: Problem, K_max: int | None = None) -> int:
    """Device bytes a run's Engine allocates (mirror of necg_create's sizes)."""
    K, n, nst = int(K_max or p.K), p.n, p.nst
    tri = n * (n + 1) // 2
    ket = (2 * tri + 6 * n + n * n + 5 + 2) & ~1
    bra = tri + 6 * n + tri + 3 + tri
    ps = tri + 1 + 3 * n
    blk = tri + 3 * n
    # symmetric-pass partials at the tuner's narrowest ket chunk (2), doubled
    # for the fused pass (H and S partials kept apart)
    ntiles = sum(min(kb * 32 + 31, K - 1) // 2 + 1 for kb in range((K + 31) // 32))
    sym = 2 * ntiles * ps * (32 + 2) if n <= 5 else 0
    doubles = (bra * K + ket * K * nst + ps * K * ((K + 3) // 4) + 2 * K * K + 2 * K + 4
               + 2 * (K * blk + K) + 2 + nst * (n * n + 9 * n * n + 1) + sym)
    return 8 * doubles + 3 * 8 * (K * blk + K) + 4096


class Run:
    def __init__(self, rid: int, problem: Problem):
        self.id = rid
        self.problem = problem
        self.engine: Engine | None = None
        self.bytes = workspace_estimate(problem)
        self.x = self.g = self.f = None
        self.xh = self.gh = self.fh = None
        self.admitted = threading.Event()
        self.admit_error: BaseException | None = None  # set when building its device state failed
        self.evals = 0
        self.closed = False
        self.inflight = 0  # requests of this run in launched, undelivered steps


class Request:
    __slots__ = ("run", "x", "done", "f", "g", "t_submit", "t_done", "error")

    def __init__(self, run: Run, x: np.ndarray):
        self.run = run
        self.x = x
        self.done = threading.Event()
        self.f = None
        self.g = None
        self.error = None
        self.t_submit = time.perf_counter()
        self.t_done = None


class Server:
    def __init__(self, budget_bytes: float = 120e9, max_slots: int = 256, graph: bool = True, tune: bool = True,
                 device=None, max_tiles: int = 1 << 22):
        self.budget = float(budget_bytes)
        self.max_slots = int(max_slots)
        self.max_tiles = int(max_tiles)  # tiles of one step (all runs); 16 bytes each per queue
        self.graph = graph
        self.tune = tune
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.lock = threading.Condition()
        self.pending: collections.deque[Request] = collections.deque()
        self.waiting_runs: collections.deque[Run] = collections.deque()
        self.runs: dict[int, Run] = {}
        self.used = 0
        self.pending_slots = 0  # admitted runs whose device state is being built
        self.next_id = 0
        self.latencies: list[float] = []
        self.steps = 0
        self.step_sizes: list[int] = []
        self.step_log: list[tuple] = []  # per step: host time delivered, requests, device ms, idle ms before it
        self._stop = False
        self._thread = None
        self.batches = None
        self.stream = None
        self.t_start = None
        self.evals_done = 0
        self.gpu_ms = 0.0   # device time of the batched steps (CUDA events on the server stream)
        self.gpu_idle_ms = 0.0  # device time between consecutive steps
        self._last_end = None
        self.plan_s = 0.0   # host time spent planning steps

    # ----------------------------------------------------------- lifecycle
    def start(self) -> "Server":
        self.stream = torch.cuda.Stream(device=self.device)
        self.batches = [Batch(self.max_slots, self.max_tiles), Batch(self.max_slots, self.max_tiles)]
        self.flags = [torch.zeros(2 * self.max_slots, dtype=torch.int32).pin_memory() for _ in range(2)]
        self.free_batches = collections.deque([0, 1])  # plans not in flight
        self.t_start = time.perf_counter()
        self._thread = threading.Thread(target=self._loop, name="necg-server", daemon=True)
        self._thread.start()
        return self

    def stop(self) -> None:
        with self.lock:
            self._stop = True
            self.lock.notify_all()
        if self._thread:
            self._thread.join()
        for b in self.batches or []:
            b.close()

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    # ------------------------------------------------------------- clients
    def open_run(self, problem: Problem, timeout: float | None = None) -> Run:
        """Register a run; blocks until it is admitted (memory budget and slots).
        If building its device state fails (the library refuses the problem,
        or memory runs out), its reservation is released and the error is
        raised here."""
        if problem.n > 5:
            raise ValueError("the batched path supports n <= 5")
        with self.lock:
            run = Run(self.next_id, problem)
            self.next_id += 1
            if run.bytes > self.budget:
                raise MemoryError(f"run needs {run.bytes} bytes, more than the whole budget {self.budget:.0f}")
            self.waiting_runs.append(run)
            ready = self._admit_locked()
        self._materialise(ready)
        if not run.admitted.wait(timeout):
            raise TimeoutError("run was not admitted in time")
        if run.admit_error is not None:
            raise run.admit_error
        return run

    def close_run(self, run: Run) -> None:
        """Close a run: its requests not yet in a step fail, and its device
        state is freed once the steps holding its requests are delivered.  The
        server keeps planning and launching steps meanwhile (the wait and the
        free run outside the server lock)."""
        with self.lock:
            if run.closed:
                return
            run.closed = True
            self.runs.pop(run.id, None)
            keep: collections.deque[Request] = collections.deque()
            for r in self.pending:
                if r.run is run:
                    r.error = RuntimeError("run was closed before this request was served")
                    r.done.set()
                else:
                    keep.append(r)
            self.pending = keep
            while run.inflight > 0:
                self.lock.wait()
            eng, run.engine = run.engine, None
        if eng is None:
            return
        eng.close(sync=False)  # its steps are delivered, so none of its work is running
        with self.lock:
            self.used -= run.bytes
            ready = self._admit_locked()
        self._materialise(ready)

    def evaluate(self, run: Run, x: np.ndarray, timeout: float | None = None):
        """E and gradient at x = [iv, C] for this run (blocking)."""
        if run.engine is None:
            raise RuntimeError("run is not admitted or already closed")
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.ndim != 1 or x.size != run.x.numel():
            raise ValueError(f"x has shape {x.shape}, expected ({run.x.numel()},)")
        req = Request(run, x)
        with self.lock:
            if run.closed:
                raise RuntimeError("run is closed")
            if self._stop:
                raise RuntimeError("server is stopped")
            self.pending.append(req)
            self.lock.notify_all()
        if not req.done.wait(timeout):
            raise TimeoutError("request timed out")
        if req.error is not None:
            raise req.error
        return req.f, req.g

    def _admit_locked(self) -> list[Run]:
        """Reserve budget and a slot for every waiting run that fits (in arrival
        order); the caller builds their device state outside the lock."""
        ready = []
        while self.waiting_runs:
            run = self.waiting_runs[0]
            if len(self.runs) + self.pending_slots >= self.max_slots or self.used + run.bytes > self.budget:
                break
            self.waiting_runs.popleft()
            self.used += run.bytes
            self.pending_slots += 1
            ready.append(run)
        return ready

    def _materialise(self, runs: list[Run]) -> None:
        """Device state of newly admitted runs: engine (handle + workspace,
        tuned tiles, the fused pass's partial buffers) and resident x, g, f.
        Runs outside the server lock, so steps keep being planned meanwhile."""
        for run in runs:
            p = run.problem
            eng = None
            try:
                with torch.cuda.device(self.device):
                    eng = Engine(p, device=self.device)
                    run.x = torch.from_numpy(np.ascontiguousarray(p.x)).to(self.device)
                    run.g = torch.empty_like(run.x)
                    run.f = torch.zeros(1, dtype=torch.float64, device=self.device)
                    run.xh = torch.empty(run.x.numel(), dtype=torch.float64).pin_memory()
                    run.gh = torch.empty(run.x.numel(), dtype=torch.float64).pin_memory()
                    run.fh = torch.empty(1, dtype=torch.float64).pin_memory()
                    if self.tune:
                        tuned(eng, run.x, p.K)
                    eng.prepare_fused(p.K)
            except Exception as exc:  # noqa: BLE001 -- handed to the client in open_run
                # give back the reservation, so other runs can be admitted
                if eng is not None:
                    eng.close()
                run.x = run.g = run.f = run.xh = run.gh = run.fh = None
                run.admit_error = exc
                with self.lock:
                    self.pending_slots -= 1
                    self.used -= run.bytes
                    run.closed = True
                    more = self._admit_locked()
                run.admitted.set()
                self._materialise(more)
                continue
            with self.lock:
                run.engine = eng
                self.pending_slots -= 1
                self.runs[run.id] = run
            run.admitted.set()

    # -------------------------------------------------------------- worker
    def _loop(self) -> None:
        """Launch a step as soon as requests are ready and a batch plan is free
        (two plans: up to two steps in flight).  A watcher thread waits for each
        step's completion with the GIL released and delivers its results, so
        clients' responses overlap the GPU's work on the other step and nothing
        polls."""
        import queue
        done_q: queue.Queue = queue.Queue()
        watcher = threading.Thread(target=self._watch, args=(done_q,), name="necg-deliver", daemon=True)
        watcher.start()
        with torch.cuda.device(self.device):
            while True:
                reqs = []
                with self.lock:
                    while not (self.pending and self.free_batches) and not (self._stop and not self.pending):
                        self.lock.wait()
                    if self._stop and not self.pending:
                        break
                    # at most one request per run per step (runs issue back to back)
                    seen, rest = set(), collections.deque()
                    while self.pending:
                        r = self.pending.popleft()
                        if r.run.id in seen:
                            rest.append(r)
                        else:
                            seen.add(r.run.id)
                            r.run.inflight += 1
                            reqs.append(r)
                    self.pending = rest
                    bi = self.free_batches.popleft()
                done_q.put(self._launch(reqs, bi))
        done_q.put(None)
        watcher.join()

    def _watch(self, done_q) -> None:
        with torch.cuda.device(self.device):
            while True:
                flight = done_q.get()
                if flight is None:
                    return
                self._deliver(*flight)

    def _launch(self, reqs: list[Request], bi: int):
        batch = self.batches[bi]
        s = self.stream
        with torch.cuda.stream(s):
            for r in reqs:
                r.run.xh.numpy()[:] = r.x
                r.run.x.copy_(r.run.xh, non_blocking=True)
            runs = [r.run for r in reqs]
            t0 = time.perf_counter()
            batch.plan([u.engine for u in runs], [u.problem.K for u in runs], [u.x for u in runs],
                       [u.g for u in runs], [u.f for u in runs], stream=s)
            self.plan_s += time.perf_counter() - t0
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            batch.step(self.graph, stream=s)
            e1.record(s)
            flags = self.flags[bi]
            batch.status_async(flags, stream=s)
            for u in runs:
                u.gh.copy_(u.g, non_blocking=True)
                u.fh.copy_(u.f, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        self.steps += 1
        self.step_sizes.append(len(reqs))
        return reqs, ev, bi, (e0, e1)

    def _deliver(self, reqs: list[Request], ev, bi: int, timing) -> None:
        ev.synchronize()
        dev_ms = timing[0].elapsed_time(timing[1])
        self.gpu_ms += dev_ms
        gap = 0.0
        if self._last_end is not None:  # device time with no step running since the previous one
            gap = max(0.0, self._last_end.elapsed_time(timing[0]))
            self.gpu_idle_ms += gap
        self._last_end = timing[1]
        if len(self.step_log) < 100000:
            self.step_log.append((time.perf_counter(), len(reqs), dev_ms, gap))
        codes = Batch.decode(self.flags[bi][0:2 * len(reqs):2].tolist())
        now = time.perf_counter()
        for r, code in zip(reqs, codes):
            if code == _lib.NECG_ERR_NOT_PD:
                r.error = np.linalg.LinAlgError("A_k + A_l' is not positive definite for some basis pair")
            elif code != _lib.NECG_OK:
                r.error = _lib.NecgError(code, f"run {r.run.id}")
            else:
                r.f = float(r.run.fh[0])
                r.g = r.run.gh.numpy().copy()
            r.t_done = now
            r.run.evals += 1
            self.latencies.append(now - r.t_submit)
            self.evals_done += 1
            r.done.set()
        with self.lock:
            for r in reqs:
                r.run.inflight -= 1
            self.free_batches.append(bi)
            self.lock.notify_all()

    # ------------------------------------------------------------ metrics
    def stats(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        wall = time.perf_counter() - (self.t_start or time.perf_counter())
        return {"requests": len(self.latencies), "steps": self.steps,
                "mean_batch": float(np.mean(self.step_sizes)) if self.step_sizes else 0.0,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "evals_per_s": self.evals_done / wall if wall > 0 else 0.0, "wall_s": wall,
                "gpu_step_s": self.gpu_ms * 1e-3, "gpu_idle_between_steps_s": self.gpu_idle_ms * 1e-3,
                "plan_s": self.plan_s, "hbm_used_bytes": self.used}


class Endpoint:
    """Front end of a ``Server`` for clients in other processes
    (``clients.RemoteRun``): a listener on 127.0.0.1 (a free port, an
    authentication key) and one handler thread per connection, each connection
    carrying one run.  A handler turns the connection's requests into
    ``open_run`` / ``evaluate`` / ``close_run`` calls, so remote requests join
    the same batched steps as in-process ones; a dropped connection closes its
    run."""

    def __init__(self, srv: Server, authkey: bytes | None = None):
        from multiprocessing.connection import Listener
        self.srv = srv
        self.authkey = authkey if authkey is not None else secrets.token_bytes(16)
        self.listener = Listener(("127.0.0.1", 0), backlog=1024, authkey=self.authkey)  # runs connect together
        self.address = self.listener.address
        self._closed = False
        self._thread = threading.Thread(target=self._accept, name="necg-endpoint", daemon=True)
        self._thread.start()

    def _accept(self) -> None:
        while not self._closed:
            try:
                conn = self.listener.accept()
            except Exception:  # noqa: BLE001 -- listener closed, or a client failed the handshake
                continue
            threading.Thread(target=self._serve, args=(conn,), name="necg-endpoint-run", daemon=True).start()

    def _serve(self, conn) -> None:
        run = None
        try:
            while True:
                try:
                    msg = conn.recv_bytes()
                except (EOFError, OSError):
                    return
                op = msg[:1]
                try:
                    if op == OP_EVAL:
                        if run is None:
                            raise RuntimeError("no run is open on this connection")
                        f, g = self.srv.evaluate(run, np.frombuffer(msg, dtype=np.float64, offset=1))
                        conn.send_bytes(REPLY_OK + struct.pack("<d", f) + g.tobytes())
                    elif op == OP_OPEN:
                        if run is not None:
                            raise RuntimeError("a run is already open on this connection")
                        problem, timeout = pickle.loads(msg[1:])
                        run = self.srv.open_run(problem, timeout=timeout)
                        conn.send_bytes(REPLY_OK + struct.pack("<q", run.id))
                    elif op == OP_CLOSE:
                        if run is not None:
                            self.srv.close_run(run)
                            run = None
                        conn.send_bytes(REPLY_OK)
                    else:
                        raise ValueError(f"unknown request {op!r}")
                except Exception as exc:  # noqa: BLE001 -- returned to the client
                    conn.send_bytes(encode_error(exc))
        finally:
            if run is not None:
                self.srv.close_run(run)
            conn.close()

    def close(self) -> None:
        self._closed = True
        self.listener.close()
