#!/usr/bin/env python
"""Benchmark: FP64 energy+gradient evaluations/s of the NECG objective
(outprod, python/outprod.py:20-76) on LiH, n=5, K=1024, nst=24.

One step = one full evaluation (H, S, E, gradient of E with respect to all
K*30 + K parameters) of the seeded synthetic LiH K=1024 basis.

  python bench.py [--gpus N --steps K --warmup W] [--impl engine|reference]

* value: whole-job evals/s with x resident on the device, device-timed with
  CUDA events on the launch stream (sum of per-step times; a 256 MiB buffer is
  written between steps to flush L2 and is not timed), max over ranks.
* e2e: the same metric through the C-ABI host-pointer entry point
  necg_outprod_host: pinned host x in, host f and g out, copies timed.
* roofline: the gradient-tile kernel (the dominant one): algorithmic FP64
  FLOPs per launch (counted from the kernel's own templates) / its live
  CUDA-event duration, against the FP64 FMA throughput measured on this GPU.
* cpu_baseline: the oracle (a C restatement of the reference's matel/gradel
  loops) on all host cores over a random sample of the workload's terms,
  extrapolated to evals/s; beside it, the reference Python's own outprod as
  timed by oracle/time_reference.py where a checkout of the reference exists
  (it has no packaging and cannot travel to this machine).
* parity: E and g of the timed evaluation against the oracle's full-size
  fixture (tests/golden/fullsize_<workload>.npz), checked after the timed
  region.
* dropin: evals/s through the drop-in module API (outprod.outprod with the
  shared module state, python/outprod.py:20), with and without copying H and
  S back, host wall clock.
* --impl reference: the same CPU port timed as the reference arm.
Multi-GPU (torchrun): every rank evaluates its own replica of the workload
(no collective on the data path); value = all ranks' evals / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "FP64 energy+grad evals/s, LiH K=1024 (dE<1e-10 Eh); served p50/p99 latency"
WORKLOADS = {"lih_k1024": "LiH n=5 K=1024 nst=24 efs=-2e-4, seed 1, C=1/K",
             "h2_k2048": "H2 n=3 K=2048 nst=4, seed 2, C=1/K",
             "lih_k12": "LiH n=5 K=12 nst=24, seed 0"}
PHASES = ["prep", "energy", "finalize", "grad_tiles", "grad_reduce"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="lih_k1024", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--pair-pass", default="auto", choices=["auto", "ordered", "symmetric", "fused"],
                    help="force the pair pass (auto: the autotuner's choice)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner and use the default tiles (for short profiling runs)")
    ap.add_argument("--serve-runs", type=int, default=256,
                    help="truncated-Newton runs (the first of the 256-run serving stream) for the served "
                         "latency / throughput figures; 0 skips them")
    ap.add_argument("--serve-maxfun", type=int, default=50, help="evaluations per run of that stream")
    ap.add_argument("--no-dropin", action="store_true", help="skip the drop-in module figure")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-instance batched figure")
    ap.add_argument("--serve-procs", type=int, default=-1,
                    help="client processes for the served figures (0: clients as threads of the bench process; "
                         "default: min(12, host cores - 2))")
    return ap.parse_args()


DEFAULT_TILES = {"lc_e": 2, "minb_e": 16, "lc_g": 4, "minb_g": 8, "sym": 2, "lc_s": 2, "minw_s": 268}
# the fused-pass variant measured fastest for other n (n = 3: one-warp blocks, 12 per SM)
DEFAULT_FUSED = {3: {"lc_s": 2, "minw_s": 122}}
PASS_MODE = {"ordered": 0, "symmetric": 1, "fused": 2}
# FP64 FLOPs per (k, l, P) term (FMA = 2; each div/sqrt/rsqrt/exp = 1), frozen at
# the counts the kernels' own templates gave when the fused pass was first
# measured; the roofline fraction is reported at these and at the current count
FROZEN_FLOPS = {5: {"energy": 1339, "grad": 3337, "sym": 4362, "fused": 4639},
                3: {"energy": 511, "grad": 1236, "sym": 1586, "fused": 1710},
                2: {"energy": 253, "grad": 598, "sym": 762, "fused": 832}}
FIXTURES = {"lih_k1024": "fullsize_lih_k1024.npz", "h2_k2048": "fullsize_h2_k2048.npz"}


def bench_config(args, world: int) -> dict:
    """The workload, as both arms print it."""
    from nbo_correlatedgaussians_b200 import synth
    prob = synth.workload(args.workload)
    K, nst = prob.K, prob.nst
    return {"workload": args.workload, "desc": WORKLOADS[args.workload],
            "pair_elements_per_eval": prob.pairs, "terms_per_eval": (prob.pairs + K * K) * nst,
            "l2": "flushed between steps by a 256 MiB write, not timed",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def parity_against_fixture(workload: str, E: float, g) -> dict | None:
    """|dE| and the norm-wise gradient error against the oracle's full-size
    fixture (made by tests/golden/make_fullsize.py)."""
    name = FIXTURES.get(workload)
    path = os.path.join(HERE, "tests", "golden", name) if name else None
    if not path or not os.path.exists(path):
        return None
    d = np.load(path)
    dE = abs(E - float(d["f"]))
    dg = float(np.max(np.abs(g - d["g"])) / np.max(np.abs(d["g"])))
    return {"fixture": f"tests/golden/{name}", "dE_Eh": dE, "g_normwise": dg, "tol": {"E_Eh": 1e-10, "g": 1e-9},
            "ok": bool(dE < 1e-10 and dg < 1e-9)}


def python_reference_timing() -> dict | None:
    """The reference Python's own outprod, timed by oracle/time_reference.py
    where a checkout of the reference exists (not on this machine)."""
    path = os.path.join(HERE, "oracle", "reference_python_timing.json")
    if not os.path.exists(path):
        return None
    d = json.load(open(path))
    k12, k1024 = d["lih_k12_all_cores"], d["lih_k1024_extrapolated"]
    return {"kind": "python", "measured_on": f"{d['host']}, {d['cores']} cores (the build machine, not this one)",
            "lih_k12_evals_per_s": k12["evals_per_s"],
            "lih_k12_s_per_eval_one_process": d["lih_k12_one_process"]["s_per_eval"],
            "lih_k1024_evals_per_s_extrapolated": k1024["evals_per_s_on_all_cores"],
            "lih_k1024_core_seconds_per_eval": k1024["core_seconds_per_eval"],
            "why_not_here": "the reference ships no setup.py/pyproject, so it cannot be installed to travel "
                            "to the GPU machine, and its sources may not be copied into this repository",
            "source": "oracle/reference_python_timing.json (oracle/time_reference.py)"}


# ----------------------------------------------------------------------------- CPU port
def cpu_port_rate(prob, seconds: float, seed: int = 0):
    """evals/s of the oracle port over a random sample of the workload's terms,
    using every host core (one ctypes call per chunk; ctypes releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle.oracle import Oracle
    o = Oracle.from_problem(prob)
    K, nst = prob.K, prob.nst
    n_mat, n_grad = K * (K + 1) // 2 * nst, K * K * nst  # calls per evaluation
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    rng = np.random.default_rng(seed)

    def terms(count, lower):
        stf = rng.integers(1, nst + 1, count)
        i = rng.integers(1, K + 1, count)
        j = rng.integers(1, K + 1, count)
        if lower:
            i, j = np.maximum(i, j), np.minimum(i, j)
        return np.stack([stf, i, j], 1).astype(np.int32)

    # calibrate on one core
    cal_m, cal_g = terms(200, True), terms(400, False)
    t0 = time.perf_counter()
    o.sample_terms(prob.iv, cal_m, cal_g)
    per = (time.perf_counter() - t0) / 600.0
    frac = min(1.0, seconds * cores / (per * (n_mat + n_grad)))
    nm, ng = max(cores, int(frac * n_mat)), max(cores, int(frac * n_grad))
    mt, gt = terms(nm, True), terms(ng, False)
    chunks = [(mt[c::cores], gt[c::cores]) for c in range(cores)]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(cores) as ex:
        list(ex.map(lambda c: o.sample_terms(prob.iv, c[0], c[1]), chunks))
    wall = time.perf_counter() - t0
    evals = 0.5 * (nm / n_mat + ng / n_grad)
    return {"value": evals / wall, "unit": "evals/s", "cores": cores, "kind": "port",
            "sample": f"{nm} matel + {ng} gradel terms ({100 * evals:.3f}% of one evaluation's "
                      f"{n_mat} + {n_grad}), {wall:.1f} s wall on {cores} threads, extrapolated"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from nbo_correlatedgaussians_b200 import synth
    prob = synth.workload(args.workload)
    per_step = max(1.0, 150.0 / max(1, args.steps + args.warmup))
    per_step = min(per_step, 6.0)
    for w in range(args.warmup):
        cpu_port_rate(prob, per_step / 3, seed=100 + w)
    rates, walls, last = [], [], None
    for s in range(args.steps):
        t0 = time.perf_counter()
        last = cpu_port_rate(prob, per_step, seed=s)
        walls.append(time.perf_counter() - t0)
        rates.append(last["value"])
    value = statistics.mean(rates)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    out = {"metric": METRIC, "value": value, "unit": "evals/s", "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls),
           "ms_per_eval_extrapolated": 1e3 / value, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, oldquit.dat layout)",
           "config": bench_config(args, world),
           "cpu_baseline": dict(last, value=value, python_reference=python_reference_timing()),
           "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "reference arm = oracle/ C port of the reference's matel/gradel loops (the reference "
                   "itself is Python and cannot travel to the GPU box); each step times a bounded random "
                   "sample of the evaluation's terms on all host threads"}
    print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "power_w_max": max(power),
                "samples": len(sm), "reasons": sorted(reasons)}


# ----------------------------------------------------------------------------- engine arm
def run_engine(args):
    import ctypes

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    from nbo_correlatedgaussians_b200 import _lib, synth
    from nbo_correlatedgaussians_b200.engine import Engine, term_flops
    L = _lib.lib()
    prob = synth.workload(args.workload)
    eng = Engine(prob)
    stream = torch.cuda.current_stream()
    x = torch.from_numpy(prob.x).cuda()
    from nbo_correlatedgaussians_b200.autotune import apply, tuned
    if args.no_tune:
        tiles = dict(DEFAULT_TILES, **DEFAULT_FUSED.get(prob.n, {}))
    else:
        tiles = dict(tuned(eng, x, prob.K))  # untimed; cached per (GPU, n, nst, K bucket)
    if args.pair_pass != "auto":
        tiles["sym"] = PASS_MODE[args.pair_pass]
        if tiles["sym"] != 2:  # variants above 100 and the splits exist for the fused pass only
            tiles["npc"] = 1
            if int(tiles.get("minw_s", 8)) not in (8, 12, 16):
                tiles["minw_s"] = 8
    apply(eng, tiles)
    _lib.check(L.necg_profile(eng.h, 1), "necg_profile")
    g = torch.empty_like(x)
    f = torch.empty(1, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        rc = L.necg_outprod(eng.h, prob.K, x.data_ptr(), f.data_ptr(), g.data_ptr(), None, None,
                            stream.cuda_stream)
        _lib.check(rc, "necg_outprod")

    phase_buf = (ctypes.c_double * 5)()
    for _ in range(args.warmup):
        flush.fill_(1.0)
        step()
    eng.raise_status("warm-up")
    peak = ctypes.c_double(0.0)
    _lib.check(L.necg_fp64_peak(200000, ctypes.byref(peak), stream.cuda_stream), "necg_fp64_peak")

    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
    barrier()
    step_ms, phases = [], []
    for _ in range(args.steps):
        flush.fill_(float(len(step_ms)))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        _lib.check(L.necg_phase_ms(eng.h, phase_buf), "necg_phase_ms")
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        phases.append(list(phase_buf))
    barrier()
    clk = clocks.stop() if clocks else None
    eng.raise_status("timed steps")
    E = float(f.item())
    parity = parity_against_fixture(args.workload, E, g.cpu().numpy())
    total = torch.tensor([sum(step_ms)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(total, op=dist.ReduceOp.MAX)
    total_ms = float(total.item())
    value = world * args.steps / (total_ms * 1e-3)

    # e2e: host buffers through the C-ABI host entry point
    xh = torch.from_numpy(prob.x.copy()).pin_memory()
    gh = torch.empty(x.numel(), dtype=torch.float64).pin_memory()
    fh = ctypes.c_double(0.0)
    e2e_ms = []
    for it in range(args.warmup + args.steps):
        flush.fill_(2.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = L.necg_outprod_host(eng.h, prob.K, xh.data_ptr(), ctypes.addressof(fh), gh.data_ptr(),
                                 stream.cuda_stream)
        e1.record(stream)
        _lib.check(rc, "necg_outprod_host")
        e1.synchronize()
        if it >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_t = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps / (float(e2e_t.item()) * 1e-3)
    assert abs(fh.value - E) <= 1e-12 * abs(E), (fh.value, E)
    assert np.array_equal(gh.numpy(), g.cpu().numpy())

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    K, nst, n = prob.K, prob.nst, prob.n
    tf = term_flops(n)
    frozen = FROZEN_FLOPS.get(n, {})
    mode = int(tiles.get("sym", 0))
    unordered = (K * (K + 1) // 2) * nst
    ph = np.array(phases)
    ph_mean = ph.mean(axis=0)
    energy_flops = unordered * tf["energy"]
    if mode == 2:  # one pass over unordered pairs: H, S and both gradients
        block = int(tiles.get("minw_s", 8)) >= 200  # lockstep blocks
        kname, per_term = (f"fsym_block_kernel<{n}>" if block else f"fsym_kernel<{n}>"), "fused"
        kern_flops, kern_ms = unordered * tf["fused"], float(ph_mean[1])
        eval_flops = kern_flops
    elif mode == 1:  # energy pass + unordered pairs with bra and ket gradients
        kname, per_term = f"gsym_kernel<{n}>", "sym"
        kern_flops, kern_ms = unordered * tf["sym"], float(ph_mean[3])
        eval_flops = kern_flops + energy_flops
    else:  # energy pass + ordered pairs (the reference's loop structure)
        kname, per_term = f"grad_kernel<{n}>", "grad"
        kern_flops, kern_ms = K * K * nst * tf["grad"], float(ph_mean[3])
        eval_flops = kern_flops + energy_flops
    ordered_equiv = K * K * nst * tf["grad"] + energy_flops
    # the roofline's FLOPs: the frozen per-term count (the current one is reported beside it)
    per_frozen = frozen.get(per_term, tf[per_term])
    terms_launch = kern_flops // tf[per_term]
    achieved_current = kern_flops / (kern_ms * 1e-3) / 1e12
    kern_flops_frozen = terms_launch * per_frozen
    achieved = kern_flops_frozen / (kern_ms * 1e-3) / 1e12
    traffic, traffic_src = None, None
    tpath = os.path.join(HERE, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath))
            traffic = tj.get(f"{kname}|{args.workload}")
            traffic_src = tj.get("_source")
        except (OSError, ValueError):
            traffic = None
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_port_rate(prob, args.cpu_seconds)
    dropin = None
    if world == 1 and not args.no_dropin:
        dropin = dropin_figures(prob, e2e_value)
    batched = None
    if world == 1 and not args.no_batched:
        batched = batched_figures()
    served = None
    if world == 1 and args.serve_runs > 0:
        served = serving_figures(args.serve_runs, args.serve_maxfun, args.serve_procs)
    out = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, oldquit.dat layout; no public dataset exists)",
        "config": bench_config(args, world),
        "tuning": {"pair_pass": ("fused energy + gradient, unordered pairs" if mode == 2 else
                                 "energy pass + gradient over unordered pairs" if mode == 1 else
                                 "energy pass + gradient over ordered pairs"),
                   "tiles": {k: tiles.get(k, 1) for k in ("lc_e", "minb_e", "lc_g", "minb_g", "sym", "lc_s", "minw_s",
                                                          "npc")
                             if k in tiles}},
        "parity": parity,
        "pair_elements_per_s": value * prob.pairs,
        "energy": E,
        "phase_ms": dict(zip(PHASES, [round(float(v), 4) for v in ph_mean])),
        "roofline": {"bound": "fp64", "kernel": kname, "achieved": achieved, "peak": peak.value,
                     "unit": "TFLOP/s", "frac": achieved / peak.value, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "flops_per_term_frozen": per_frozen,
                     "achieved_at_current_count": achieved_current,
                     "frac_at_current_count": achieved_current / peak.value,
                     "kernel_ms": kern_ms,
                     "peak_source": "measured now by the FP64 FMA probe (necg_fp64_peak); "
                                    "MEASURED_PEAKS.json has no FP64 figure; nominal B200 FP64 = 37 TFLOP/s",
                     "flops_per_launch": kern_flops_frozen, "flops_per_term": tf[per_term],
                     "special_per_term": tf[per_term + "_special"],
                     "energy_kernel": (None if mode == 2 else
                                       {"achieved": energy_flops / (float(ph_mean[1]) * 1e-3) / 1e12,
                                        "flops_per_launch": energy_flops}),
                     "whole_eval_tflops": eval_flops / (total_ms / args.steps * 1e-3) / 1e12,
                     "reference_loop_equivalent_tflops": ordered_equiv / (total_ms / args.steps * 1e-3) / 1e12},
        "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": int(prob.x.nbytes),
                "d2h_bytes_per_step": int(prob.x.nbytes) + 8,
                "path": "necg_outprod_host (pinned host x -> f, g)"},
        # status reset, 2 prep, pair pass(es), rows + finalize, partial sum(s), reduce
        "gpu_launches": launches_per_eval(prob, tiles, mode) * args.steps,
        "cpu_baseline": (dict(cpu, python_reference=python_reference_timing()) if cpu else None),
        "dropin": dropin,
        "batched": batched,
        "clocks": clk,
        "served": served,
    }
    print(json.dumps(out), flush=True)


def launches_per_eval(prob, tiles: dict, mode: int) -> int:
    """Library kernels one evaluation launches: status reset, bra and ket
    records, the pair pass(es), H C / S C rows, finalize, partial sum(s) and the
    reduce to the parameter layout; in the fused pass also the fix-up of the
    lockstep queue's split tail, or the sum of split H, S of one-warp tiles."""
    import torch
    K, nst = prob.K, prob.nst
    if mode != 2:
        return 9 if mode == 1 or (K + tiles["lc_g"] - 1) // tiles["lc_g"] > 1 else 8
    n = 8
    minw, lc = int(tiles.get("minw_s", 8)), int(tiles.get("lc_s", 2))
    if minw >= 200:  # lockstep groups: the tail is split when the last round is partial
        gw = 12 if minw in (222, 232) else 8
        groups = sum(-(-(min(kb * 32 + 31, K - 1) // lc + 1) // gw) for kb in range((K + 31) // 32))
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        tail = groups % sms
        if tail and min(4, nst, sms // tail) >= 2:
            n += 1
    elif int(tiles.get("npc", 1)) > 1:
        n += 1
    return n


def batched_figures(steps: int = 10) -> dict:
    """The 64-instance mixed batch (16 He with K log-uniform 32-512, 24 H2 and 24
    LiH with K 64-1024; seeds 3000 + i): one batched step (a persistent launch
    over every instance's tiles, replayed as a CUDA graph) against the same
    instances evaluated one after another through the per-call path, each with
    its autotuned setting; x resident on the device, CUDA events on the stream."""
    import torch

    from nbo_correlatedgaussians_b200 import _lib, synth
    from nbo_correlatedgaussians_b200.batch import BatchEngine
    probs = synth.workload("mixed64")
    be = BatchEngine(probs, tune=True)
    L = _lib.lib()
    stream = torch.cuda.current_stream()
    be.plan()

    def timed(fn) -> float:
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    def per_call():
        for i, eng in enumerate(be.engines):
            _lib.check(L.necg_outprod(eng.h, probs[i].K, be.x[i].data_ptr(), be.f[i].data_ptr(), be.g[i].data_ptr(),
                                      None, None, stream.cuda_stream), "necg_outprod")

    batch_ms = timed(lambda: be.step(graph=True))
    be.check()
    call_ms = timed(per_call)
    n = len(probs)
    be.close()
    return {"workload": "mixed64: 16 He (K 32-512), 24 H2 and 24 LiH (K 64-1024), seeds 3000+i", "instances": n,
            "batched_ms_per_step": batch_ms, "batched_evals_per_s": n / (batch_ms * 1e-3),
            "per_call_ms_per_round": call_ms, "per_call_evals_per_s": n / (call_ms * 1e-3),
            "batched_vs_per_call": call_ms / batch_ms}


def dropin_figures(prob, e2e_value: float, calls: int = 20) -> dict:
    """evals/s through the drop-in module API (shared module state + outprod,
    the call python/necg.py:159-171 hands to the optimiser), host wall clock
    around each call, with and without H and S copied back into shared."""
    import tempfile

    from nbo_correlatedgaussians_b200 import shared as sh
    from nbo_correlatedgaussians_b200.outprod import outprod
    from nbo_correlatedgaussians_b200.problem import write_oldquit
    from nbo_correlatedgaussians_b200.read_input import read_input
    with tempfile.TemporaryDirectory() as td:
        fn = os.path.join(td, "oldquit.dat")
        write_oldquit(prob, fn)
        read_input(fn)
    x = np.concatenate([sh.iv, sh.C])
    out = {"path": "nbo_correlatedgaussians_b200.outprod.outprod (pageable numpy x in, f and g out)",
           "calls": calls}
    for sync in (False, True):
        sh.sync_matrices = sync
        for _ in range(3):
            outprod(x)
        t0 = time.perf_counter()
        for _ in range(calls):
            outprod(x)
        rate = calls / (time.perf_counter() - t0)
        out["sync_matrices" if sync else "no_sync_matrices"] = {"evals_per_s": rate,
                                                              "vs_host_entry_e2e": rate / e2e_value}
    sh.sync_matrices = True
    return out


def serving_figures(nruns: int, maxfun: int, procs: int = -1) -> dict:
    """The served form on a prefix of the 256-run stream (n uniform over He, H2,
    LiH; K log-uniform 16-2048; seeds 4000 + j): each run is a truncated-Newton
    client making at most ``maxfun`` evaluations.  Three ways through the same
    runs: plain (one after another through the per-call host entry point),
    served with every run admitted at t = 0 (the capacity), and served with
    Poisson arrivals at 20/s (the latency figures).  Host wall clock, setup
    (engine creation, tuning) excluded from plain and from the capacity run.  The
    served clients run in ``procs`` client processes (their SciPy work then
    spreads over host cores) and, for comparison, as threads of this process."""
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.loadgen import plain_stream, served_stream
    if procs < 0:
        cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        procs = max(1, min(12, cores - 2))
    probs = synth.workload("serve256")[:nruns]
    plain = plain_stream(probs, maxfun)
    sat = served_stream(probs, maxfun, rate=0.0, procs=procs)
    poi = served_stream(probs, maxfun, rate=20.0, seed=4, procs=procs)
    sat_thr = served_stream(probs, maxfun, rate=0.0) if procs > 0 else sat
    keep = ("evals", "wall_s", "evals_per_s", "p50_ms", "p99_ms")
    more = ("gpu_step_s", "gpu_idle_between_steps_s", "mean_batch")
    return {"workload": f"first {nruns} runs of the 256-run TN stream, maxfun {maxfun}",
            "client_procs": procs,
            "plain": {k: plain[k] for k in keep},
            "served_capacity": {k: sat[k] for k in keep + more},
            "served_poisson_20_per_s": {k: poi[k] for k in keep + more},
            "served_capacity_thread_clients": {k: sat_thr[k] for k in keep + more},
            "capacity_vs_plain": sat["evals_per_s"] / plain["evals_per_s"]}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
