"""Seeded synthetic inputs in the reference's problem layout.

The reference publishes no benchmark inputs; its only LiH input is the 12-term
oldquit.dat, and its generator (input_file_generation/generate_lih_input.py)
samples new bases from that file's statistics and sets C_k = 1/K
(generate_lih_input.py:245).  These generators follow the distributions the
engine is measured on:

* L_k lower triangular, diagonal uniform[0.2, 3.0] (LiH) or [0.1, 4.0]
  (He, H2), off-diagonal normal(0, 0.3), packed column-major as vech
  (python/matel.py:59-66);
* shifts s_k normal(0, 0.05) in 3n components (x, y, z per particle);
* C_k = 1/K;
* efs = -2e-4 for LiH (the field of oldquit.dat), 0 for He and H2.

Named workloads (seeds fixed):
  lih_k12      LiH,  K=12,   seed 0
  lih_k1024    LiH,  K=1024, seed 1
  h2_k2048     H2,   K=2048, seed 2
  mixed64      16 He (K log-uniform 32..512), 24 H2 and 24 LiH (K 64..1024), seeds 3000+i
  serve256     256 runs, n from {He, H2, LiH}, K log-uniform 16..2048, seeds 4000+j
"""
from __future__ import annotations

import numpy as np

from .problem import Problem
from .symmetry import particles, symmetry_set

DIAG_RANGE = {"He": (0.1, 4.0), "H2": (0.1, 4.0), "LiH": (0.2, 3.0)}
EFS = {"He": 0.0, "H2": 0.0, "LiH": -2.0e-4}


def make_problem(system: str, K: int, seed: int, efs: float | None = None) -> Problem:
    rng = np.random.default_rng(seed)
    n, mass, ncv = particles(system)
    sml, sms, w = symmetry_set(system)
    lo, hi = DIAG_RANGE[system]
    svh, skp = n * (n + 1) // 2, 3 * n
    blocks = np.empty((K, svh + skp))
    for k in range(K):
        L = np.zeros((n, n))
        for j in range(n):
            for i in range(j, n):
                L[i, j] = rng.uniform(lo, hi) if i == j else rng.normal(0.0, 0.3)
        idx = 0
        for j in range(n):
            for i in range(j, n):
                blocks[k, idx] = L[i, j]
                idx += 1
        blocks[k, svh:] = rng.normal(0.0, 0.05, skp)
    C = np.full(K, 1.0 / K)
    p = Problem(n, K, EFS[system] if efs is None else float(efs), mass, ncv, w / len(w), sml, sms,
                blocks.reshape(-1).copy(), C, name=f"{system}_K{K}_seed{seed}")
    p.validate()
    return p


def log_uniform_int(rng, lo: int, hi: int) -> int:
    return int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))


def workload(name: str):
    """Return a Problem (single-instance workloads) or a list of Problems."""
    if name == "lih_k12":
        return make_problem("LiH", 12, 0)
    if name == "lih_k1024":
        return make_problem("LiH", 1024, 1)
    if name == "h2_k2048":
        return make_problem("H2", 2048, 2)
    if name == "mixed64":
        out = []
        rng = np.random.default_rng(3)
        specs = [("He", 32, 512)] * 16 + [("H2", 64, 1024)] * 24 + [("LiH", 64, 1024)] * 24
        for i, (sysname, lo, hi) in enumerate(specs):
            out.append(make_problem(sysname, log_uniform_int(rng, lo, hi), 3000 + i))
        return out
    if name == "serve256":
        rng = np.random.default_rng(4)
        out = []
        for j in range(256):
            sysname = ("He", "H2", "LiH")[int(rng.integers(0, 3))]
            out.append(make_problem(sysname, log_uniform_int(rng, 16, 2048), 4000 + j))
        return out
    raise ValueError(f"unknown workload {name!r}")
