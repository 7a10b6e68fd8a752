"""Time the reference Python's own outprod (python/outprod.py:20-76) on this
host's cores: the CPU baseline of the unmodified reference.

TEST INFRASTRUCTURE ONLY (a measurement of the reference, never part of the
product path).  It needs a checkout of the reference; the reference ships no
packaging (no setup.py or pyproject.toml), so it cannot be installed to travel
to another machine, and its timing is taken where a checkout exists:

    NECG_REF=/path/to/NBO_CorrelatedGaussians python oracle/time_reference.py

Measured, with OMP_NUM_THREADS=OPENBLAS_NUM_THREADS=1 in every process:
  * LiH K=12 (seed 0, the 12-term workload): one full outprod in one process,
    and P processes each running full outprods at the same time (aggregate
    evals/s over P cores; P independent evaluations bound from above what any
    split of one evaluation over P cores can reach, since a split only adds
    reduction work);
  * LiH K=1024 (seed 1): per-call times of matel and gradel on a random sample
    of (stf, ii, jj), extrapolated with the exact call counts of one outprod,
    K(K+1)/2 nst matel calls + K^2 nst gradel calls (python/outprod.py:46-52,
    python/make_grad.py:38-50), over P cores.
Writes oracle/reference_python_timing.json.
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import platform
import sys
import time

for _v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ[_v] = "1"

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "reference_python_timing.json")


def _reference_path() -> str:
    ref = os.environ.get("NECG_REF")
    if not ref:
        sys.exit("set NECG_REF to a checkout of MauricioCafiero/NBO_CorrelatedGaussians")
    return os.path.join(ref, "python")


def _load(workload: str):
    """Import the reference modules and set their shared state to a seeded
    workload (the layout python/read_input.py:78-157 produces)."""
    sys.path.insert(0, REPO)
    sys.path.insert(0, _reference_path())
    import shared as sh  # reference module
    from nbo_correlatedgaussians_b200 import synth
    p = synth.workload(workload)
    sh.M, sh.ne, sh.nst, sh.efs = p.K, p.n, p.nst, p.efs
    sh.skp, sh.svh = 3 * p.n, p.n * (p.n + 1) // 2
    sh.siv = sh.M * (sh.svh + sh.skp)
    sh.mass, sh.ncv, sh.scvv = p.mass.copy(), p.ncv.copy(), p.scvv.copy()
    sh.iv, sh.C = p.iv.copy(), p.C.copy()
    sh.sml = np.ascontiguousarray(np.transpose(p.sml, (1, 2, 0)))
    sh.sms = np.ascontiguousarray(np.transpose(p.sms, (1, 2, 0)))
    for name in ("H", "S", "Kinetic", "Potential", "ki", "po", "hh", "ss"):
        setattr(sh, name, np.zeros((sh.M, sh.M)))
    sh.grad = np.zeros(sh.siv + sh.M)
    return p


def _outprod_worker(args):
    workload, reps, start = args
    p = _load(workload)
    from outprod import outprod  # reference module
    while time.time() < start:
        time.sleep(0.001)
    t0 = time.perf_counter()
    f = None
    for _ in range(reps):
        f, _g = outprod(p.x)
    return time.perf_counter() - t0, f


def _sample_worker(args):
    workload, n, seed = args
    p = _load(workload)
    from gradel import gradel  # reference module
    from matel import matel  # reference module
    rng = np.random.default_rng(seed)
    terms = np.stack([rng.integers(1, p.nst + 1, n), rng.integers(1, p.K + 1, n), rng.integers(1, p.K + 1, n)], 1)
    t0 = time.perf_counter()
    for stf, i, j in terms:
        matel(int(stf), int(i), int(j))
    tm = time.perf_counter() - t0
    t0 = time.perf_counter()
    for stf, i, j in terms:
        gradel(int(stf), int(i), int(j))
    return tm / n, (time.perf_counter() - t0) / n


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or platform.machine()


def main():
    procs = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    ctx = mp.get_context("spawn")
    out = {"host": _cpu_model(), "cores": procs, "python": platform.python_version(), "numpy": np.__version__}
    with ctx.Pool(1) as pool:
        t, f = pool.map(_outprod_worker, [("lih_k12", 3, 0.0)])[0]
    out["lih_k12_one_process"] = {"s_per_eval": t / 3, "evals_per_s": 3 / t, "E": f, "processes": 1}
    reps = 2
    with ctx.Pool(procs) as pool:
        start = time.time() + 5.0  # every worker has imported and loaded before the clock starts
        res = pool.map(_outprod_worker, [("lih_k12", reps, start)] * procs)
    wall = max(r[0] for r in res)
    out["lih_k12_all_cores"] = {"processes": procs, "evals": procs * reps, "wall_s": wall,
                                "evals_per_s": procs * reps / wall}
    n = 150
    with ctx.Pool(procs) as pool:
        res = pool.map(_sample_worker, [("lih_k1024", n, s) for s in range(procs)])
    tm = float(np.mean([r[0] for r in res]))
    tg = float(np.mean([r[1] for r in res]))
    K, nst = 1024, 24
    calls_m, calls_g = K * (K + 1) // 2 * nst, K * K * nst
    core_s = calls_m * tm + calls_g * tg
    out["lih_k1024_extrapolated"] = {
        "matel_s_per_call": tm, "gradel_s_per_call": tg, "sampled_calls_per_process": n, "processes": procs,
        "matel_calls": calls_m, "gradel_calls": calls_g, "core_seconds_per_eval": core_s,
        "evals_per_s_on_all_cores": procs / core_s,
        "note": "per-call times sampled while all processes ran; one outprod makes these call counts"}
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
