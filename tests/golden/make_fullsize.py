"""Generate the full-size parity fixtures in this directory with the CPU oracle.

The reference Python needs about 22 core-hours for one LiH K=1024 evaluation,
so the full-size fixtures come from the oracle (oracle/necg_oracle.c, the C
restatement of python/outprod.py:20-76, python/make_grad.py:18-90,
python/matel.py:28-210 and python/gradel.py:27-392), which
tests/test_oracle_golden.py pins to fixtures made by executing the reference
itself.  No reference checkout is needed:

    python tests/golden/make_fullsize.py [name ...]

Fixtures (npz, FP64; the problems are regenerated from their seeds by
nbo_correlatedgaussians_b200.synth, and each fixture stores the sum and the
SHA-256 of the x it was made from so a test can tell that it has the same x):
  fullsize_lih_k1024.npz  LiH n=5, K=1024, nst=24, seed 1 (the benchmarked
                          workload): f and g at C = 1/K and at a random C
                          (seed 101), and 8192 sampled H and S entries.
  fullsize_h2_k2048.npz   H2 n=3, K=2048, nst=4, seed 2: f and g at C = 1/K,
                          and 8192 sampled H and S entries.
  fullsize_lih_k731.npz   the largest LiH instance of the 64-instance mixed
                          batch (K=731, seed 3000 + index): f and g at C = 1/K.
  fullsize_serve_lih.npz, fullsize_serve_he.npz
                          the largest LiH run (K=1928) and the largest He run
                          (K=2032) of the 256-run serving stream: f and g at
                          C = 1/K.
The oracle runs on every host core; the whole set takes about half an hour on
8 cores (most of it the LiH K=1928 run).
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from nbo_correlatedgaussians_b200 import synth  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

NSAMPLE = 8192
THREADS = os.cpu_count() or 1


def x_digest(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()


def random_c(K: int, seed: int) -> np.ndarray:
    """A dense random coefficient vector (no symmetry between basis functions)."""
    return np.random.default_rng(seed).normal(0.0, 1.0, K) / np.sqrt(K)


def sample_pairs(K: int, seed: int) -> np.ndarray:
    """NSAMPLE (i, j) entries: the diagonal ends, the first and last rows, then random."""
    rng = np.random.default_rng(seed)
    fixed = [(0, 0), (K - 1, K - 1), (K - 1, 0), (0, K - 1), (K // 2, K // 2 - 1)]
    rnd = rng.integers(0, K, size=(NSAMPLE - len(fixed), 2))
    return np.concatenate([np.array(fixed), rnd]).astype(np.int32)


def evaluate(p, C=None, hs=False):
    x = p.x.copy()
    if C is not None:
        x[p.siv:] = C
    t = time.time()
    out = Oracle.from_problem(p).outprod(x, nthreads=THREADS, return_hs=hs)
    print(f"  {p.name} {'C=1/K' if C is None else 'random C'}: f = {out[0]:.15f} ({time.time() - t:.1f} s)",
          flush=True)
    return x, out


def gen_lih_k1024():
    p = synth.workload("lih_k1024")
    x, (f, g, H, S) = evaluate(p, hs=True)
    C = random_c(p.K, 101)
    xr, (fr, gr) = evaluate(p, C)
    ij = sample_pairs(p.K, 7)
    np.savez_compressed(os.path.join(HERE, "fullsize_lih_k1024.npz"), workload="lih_k1024", K=p.K, n=p.n,
                        x_sum=float(x.sum()), x_sha=x_digest(x), f=f, g=g, C_rand=C, xr_sha=x_digest(xr), f_rand=fr,
                        g_rand=gr, ij=ij, H=H[ij[:, 0], ij[:, 1]], S=S[ij[:, 0], ij[:, 1]])


def gen_h2_k2048():
    p = synth.workload("h2_k2048")
    x, (f, g, H, S) = evaluate(p, hs=True)
    ij = sample_pairs(p.K, 8)
    np.savez_compressed(os.path.join(HERE, "fullsize_h2_k2048.npz"), workload="h2_k2048", K=p.K, n=p.n,
                        x_sum=float(x.sum()), x_sha=x_digest(x), f=f, g=g, ij=ij, H=H[ij[:, 0], ij[:, 1]],
                        S=S[ij[:, 0], ij[:, 1]])


def largest_mixed_lih():
    """(index, Problem) of the largest LiH instance of the mixed 64-instance batch."""
    insts = synth.workload("mixed64")
    i = max((j for j, q in enumerate(insts) if q.n == 5), key=lambda j: insts[j].K)
    return i, insts[i]


def gen_lih_k731():
    i, p = largest_mixed_lih()
    x, (f, g) = evaluate(p)
    np.savez_compressed(os.path.join(HERE, f"fullsize_lih_k{p.K}.npz"), workload="mixed64", index=i, K=p.K,
                        n=p.n, x_sum=float(x.sum()), x_sha=x_digest(x), f=f, g=g)


def largest_serve_run(n: int):
    """(index, Problem) of the largest run with n particles in the 256-run serving stream."""
    runs = synth.workload("serve256")
    j = max((i for i, q in enumerate(runs) if q.n == n), key=lambda i: runs[i].K)
    return j, runs[j]


def gen_serve(n: int, tag: str):
    j, p = largest_serve_run(n)
    x, (f, g) = evaluate(p)
    np.savez_compressed(os.path.join(HERE, f"fullsize_serve_{tag}.npz"), workload="serve256", index=j, K=p.K,
                        n=p.n, x_sum=float(x.sum()), x_sha=x_digest(x), f=f, g=g)


GENERATORS = {"lih_k1024": gen_lih_k1024, "h2_k2048": gen_h2_k2048, "lih_k731": gen_lih_k731,
              "serve_he": lambda: gen_serve(2, "he"), "serve_lih": lambda: gen_serve(5, "lih")}

if __name__ == "__main__":
    for name in sys.argv[1:] or list(GENERATORS):
        print(name, flush=True)
        GENERATORS[name]()
