"""Load generator for the serving loop: streams of concurrent truncated-Newton
runs, each minimising E over x = [iv, C] with SciPy's TNC (the Python analogue
of the reference's LMQN/TN optimiser, source/tn.f) and calling the engine for
every energy+gradient evaluation, as python/necg.py:159-171 calls outprod.

Two ways to serve the same runs:
  plain_stream   the runs one after another through the per-call host entry
                 point (Engine.outprod: copy x in, one evaluation, copy f, g out)
  served_stream  the runs as concurrent clients of a continuous-batching
                 ``Server``; runs arrive as a Poisson process (or all at t=0,
                 which measures the server's capacity)
Results of a run do not depend on which other runs share a step (the batched
tiles and reductions are the same alone and in any mix), so both ways make the
same evaluations and the evaluation counts match.
"""
from __future__ import annotations

import threading
import time

import numpy as np
from scipy.optimize import minimize

from .autotune import tuned
from .engine import Engine
from .problem import Problem
from .serve import Server


def tn_run(evaluate, x0: np.ndarray, maxfun: int) -> int:
    """One truncated-Newton run of at most ``maxfun`` evaluations; returns the
    number of evaluations made."""
    count = [0]

    def fun(x):
        count[0] += 1
        return evaluate(x)

    minimize(fun, x0, method="TNC", jac=True, options={"maxfun": int(maxfun)})
    return count[0]


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
                  budget_bytes: float = 120e9, max_slots: int = 256, tune: bool = True) -> dict:
    """The runs as concurrent clients of one Server: run j opens at its
    arrival time (admission waits for HBM budget and a slot), makes its TN
    evaluations back to back, and closes."""
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
