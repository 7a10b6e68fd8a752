"""Load generator for the serving loop: streams of concurrent truncated-Newton
runs, each minimising E over x = [iv, C] with SciPy's TNC (the Python analogue
of the reference's LMQN/TN optimiser, source/tn.f) and calling the engine for
every energy+gradient evaluation, as python/necg.py:159-171 calls outprod.

Two ways to serve the same runs:
  plain_stream   the runs one after another through the per-call host entry
                 point (Engine.outprod: copy x in, one evaluation, copy f, g out)
  served_stream  the runs as concurrent clients of a continuous-batching
                 ``Server``; runs arrive as a Poisson process (or all at t=0,
                 which measures the server's capacity).  The clients are
                 threads of this process, or (procs > 0) threads of that many
                 client processes connected through a ``serve.Endpoint``, so
                 that their optimiser work runs on several host cores
Results of a run do not depend on which other runs share a step (the batched
tiles and reductions are the same alone and in any mix), so both ways make the
same evaluations and the evaluation counts match.
"""
from __future__ import annotations

import multiprocessing as mp
import queue
import threading
import time

import numpy as np

from .autotune import tuned
from .clients import client_worker, tn_run
from .engine import Engine
from .problem import Problem
from .serve import Endpoint, Server

__all__ = ["tn_run", "arrival_times", "plain_stream", "served_stream"]


def arrival_times(n: int, rate: float, seed: int) -> np.ndarray:
    """Poisson arrivals: cumulative exponential gaps of mean 1/rate (rate <= 0:
    every run at t = 0)."""
    if rate <= 0:
        return np.zeros(n)
    return np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, n))


def plain_stream(problems: list[Problem], maxfun: int, tune: bool = True) -> dict:
    """The runs one after another through the per-call path; engine creation
    and tuning are not timed."""
    evals, busy = 0, 0.0
    lat = []
    for p in problems:
        eng = Engine(p)
        if tune:
            tuned(eng, p.x, p.K)
        eng.outprod(p.x)  # warm-up (first-launch costs), not counted

        def evaluate(x, eng=eng):
            t = time.perf_counter()
            r = eng.outprod(x)
            lat.append(time.perf_counter() - t)
            return r

        t0 = time.perf_counter()
        evals += tn_run(evaluate, p.x.copy(), maxfun)
        busy += time.perf_counter() - t0
        eng.close()
    la = np.array(lat) if lat else np.zeros(1)
    return {"runs": len(problems), "evals": evals, "wall_s": busy, "evals_per_s": evals / busy,
            "p50_ms": float(np.percentile(la, 50) * 1e3), "p99_ms": float(np.percentile(la, 99) * 1e3)}


def served_stream(problems: list[Problem], maxfun: int, rate: float = 20.0, seed: int = 4,
                  budget_bytes: float = 120e9, max_slots: int = 256, tune: bool = True,
                  procs: int = 0) -> dict:
    """The runs as concurrent clients of one Server: run j opens at its
    arrival time (admission waits for HBM budget and a slot), makes its TN
    evaluations back to back, and closes.  procs > 0: the clients are spread
    over that many client processes."""
    if procs > 0:
        return _served_stream_procs(problems, maxfun, rate, seed, budget_bytes, max_slots, tune, procs)
    t_arr = arrival_times(len(problems), rate, seed)
    evals = [0] * len(problems)
    errors = []
    # all runs at t = 0 and all admissible at once: time from the moment every
    # run is admitted (setup excluded, as in plain_stream) -- the capacity
    from .serve import workspace_estimate
    saturate = rate <= 0 and len(problems) <= max_slots and \
        sum(workspace_estimate(p) for p in problems) <= budget_bytes
    gate = threading.Barrier(len(problems) + 1) if saturate else None
    with Server(budget_bytes=budget_bytes, max_slots=max_slots, tune=tune) as srv:
        t0 = time.perf_counter()

        def client(j):
            try:
                dt = t_arr[j] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                run = srv.open_run(problems[j])
                if gate is not None:
                    gate.wait()
                evals[j] = tn_run(lambda x: srv.evaluate(run, x), problems[j].x.copy(), maxfun)
                srv.close_run(run)
            except Exception as exc:  # noqa: BLE001 -- reported by the caller
                errors.append((j, repr(exc)))
                if gate is not None:
                    gate.abort()

        th = [threading.Thread(target=client, args=(j,), daemon=True) for j in range(len(problems))]
        for t in th:
            t.start()
        if gate is not None:
            try:
                gate.wait()
            except threading.BrokenBarrierError:
                pass
            t0 = time.perf_counter()
        srv.t_start = t0
        for t in th:
            t.join()
        wall = time.perf_counter() - t0
        st = srv.stats()
    if errors:
        raise RuntimeError(f"{len(errors)} runs failed, first: {errors[0]}")
    total = int(sum(evals))
    return {"runs": len(problems), "evals": total, "wall_s": wall, "evals_per_s": total / wall,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "steps": st["steps"],
            "mean_batch": st["mean_batch"], "gpu_step_s": st["gpu_step_s"],
            "gpu_idle_between_steps_s": st["gpu_idle_between_steps_s"], "plan_s": st["plan_s"],
            "arrival_rate_per_s": rate,
            "last_arrival_s": float(t_arr[-1]) if len(t_arr) else 0.0}


def _served_stream_procs(problems, maxfun, rate, seed, budget_bytes, max_slots, tune, procs) -> dict:
    from .serve import workspace_estimate
    t_arr = arrival_times(len(problems), rate, seed)
    saturate = rate <= 0 and len(problems) <= max_slots and \
        sum(workspace_estimate(p) for p in problems) <= budget_bytes
    ctx = mp.get_context("spawn")  # client processes never touch CUDA
    gate = ctx.Barrier(len(problems) + 1) if saturate else None
    go = ctx.Event()
    t0_epoch = ctx.Value("d", 0.0)
    out_q = ctx.Queue()
    procs = max(1, min(int(procs), len(problems)))
    ready = ctx.Barrier(procs + 1)
    with Server(budget_bytes=budget_bytes, max_slots=max_slots, tune=tune) as srv:
        ep = Endpoint(srv)
        try:
            jobs = [[] for _ in range(procs)]
            for j, p in enumerate(problems):
                jobs[j % procs].append((j, p, float(t_arr[j])))
            workers = [ctx.Process(target=client_worker, args=(ep.address, ep.authkey, jobs[w], maxfun, ready, gate,
                                                               go, t0_epoch, out_q), daemon=True)
                       for w in range(procs)]
            for w in workers:
                w.start()
            ready.wait(timeout=300)  # every client process has started
            if gate is not None:
                try:
                    gate.wait(timeout=1800)  # every run admitted: time the capacity from here
                except threading.BrokenBarrierError:
                    pass  # a run failed to open; its client reports it
                t0 = time.time()
            else:
                t0 = time.time()
                t0_epoch.value = t0
                go.set()
            srv.t_start = time.perf_counter() + (t0 - time.time())
            results = []
            while len(results) < len(workers):
                try:
                    results.append(out_q.get(timeout=1.0))
                except queue.Empty:
                    dead = [w.exitcode for w in workers if w.exitcode not in (None, 0)]
                    if dead:
                        raise RuntimeError(f"a client process exited with code {dead[0]}") from None
            for w in workers:
                w.join()
            st = srv.stats()
        finally:
            ep.close()
    errors = [e for r in results for e in r["errors"]]
    if errors:
        raise RuntimeError(f"{len(errors)} runs failed, first: {errors[0]}")
    evals = sum(n for r in results for n in r["evals"].values())
    wall = max(t for r in results for t in r["t_done"].values()) - t0
    return {"runs": len(problems), "evals": int(evals), "wall_s": wall, "evals_per_s": evals / wall,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "steps": st["steps"],
            "mean_batch": st["mean_batch"], "gpu_step_s": st["gpu_step_s"],
            "gpu_idle_between_steps_s": st["gpu_idle_between_steps_s"], "plan_s": st["plan_s"],
            "arrival_rate_per_s": rate, "client_procs": procs,
            "last_arrival_s": float(t_arr[-1]) if len(t_arr) else 0.0}
