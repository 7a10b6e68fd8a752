"""Parity at the full benchmark sizes: the sm_100a path (through the C ABI)
against oracle fixtures made by tests/golden/make_fullsize.py.

  LiH n=5, K=1024, nst=24, seed 1   the benchmarked workload: C = 1/K and a
                                    random C; every pair pass
  H2 n=3, K=2048, nst=4, seed 2     C = 1/K; tuned and ordered passes
  LiH K=731 (largest LiH instance   per call and inside the 64-instance
  of the mixed batch)               batched step
  the largest LiH (K=1928) and He   per call and together in one batched step
  (K=2032) runs of the serving stream

Tolerances (the reference's own quantities, python/outprod.py:20-76 and
python/make_grad.py:18-90): E within 1e-10 Eh absolute; g within 1e-9
norm-wise (max|g - g_ref| / max|g_ref|); sampled H and S entries within 1e-12
of the largest sampled entry (an entry far below that scale is a sum of
cancelling terms and its own relative error says nothing about the kernel).
Each test prints its measured errors on a line that starts with PARITY.
"""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from _util import TOL_E, TOL_ELEM, TOL_G, golden, normwise  # noqa: E402

# (mode, ket chunk, variant): ordered pairs (the reference's loop structure),
# symmetric gradient pass, fused pass one-warp, fused pass lockstep blocks
PASSES = {"ordered": (0, 4, 8), "symmetric": (1, 2, 8), "fused_1warp": (2, 2, 118), "fused_lockstep": (2, 2, 228)}


def _sha(x) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()


def _hs_err(Hd, d, key):
    ij = d["ij"]
    ref = d[key]
    got = Hd[ij[:, 0], ij[:, 1]]
    return float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))


def _eval(eng, x, K, with_hs=True):
    import torch
    xt = torch.from_numpy(np.ascontiguousarray(x)).to(eng.device)
    H = S = None
    if with_hs:
        H = torch.empty((K, K), dtype=torch.float64, device=eng.device)
        S = torch.empty_like(H)
    f, g = eng.outprod_device(xt, K, H=H, S=S)
    torch.cuda.synchronize()
    eng.raise_status("outprod")
    out = [float(f.item()), g.cpu().numpy()]
    if with_hs:
        out += [H.cpu().numpy(), S.cpu().numpy()]
    return out


def _set_pass(eng, name, x, K):
    from nbo_correlatedgaussians_b200 import _lib, autotune
    if name == "tuned":
        autotune.tuned(eng, x, K)
        return
    mode, lc, minw = PASSES[name]
    assert eng.L.necg_set_symmetric(eng.h, mode, lc, minw) == _lib.NECG_OK
    assert eng.L.necg_set_splits(eng.h, 1) == _lib.NECG_OK


@pytest.fixture(scope="module")
def lih1024():
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.engine import Engine
    d = golden("fullsize_lih_k1024.npz")
    p = synth.workload("lih_k1024")
    assert _sha(p.x) == str(d["x_sha"]), "the seeded LiH K=1024 input differs from the fixture's"
    eng = Engine(p)
    yield p, d, eng
    eng.close()


@pytest.mark.parametrize("name", ["tuned"] + list(PASSES))
def test_lih_k1024_every_pass(lih1024, name):
    p, d, eng = lih1024
    _set_pass(eng, name, p.x, p.K)
    f, g, H, S = _eval(eng, p.x, p.K)
    dE, dg = abs(f - float(d["f"])), normwise(g, d["g"])
    eH, eS = _hs_err(H, d, "H"), _hs_err(S, d, "S")
    print(f"PARITY lih_k1024 {name}: |dE|={dE:.2e} Eh g={dg:.2e} H={eH:.2e} S={eS:.2e}")
    assert dE < TOL_E and dg < TOL_G
    assert eH < TOL_ELEM and eS < TOL_ELEM


@pytest.mark.parametrize("name", ["tuned", "ordered"])
def test_lih_k1024_random_coefficients(lih1024, name):
    p, d, eng = lih1024
    x = p.x.copy()
    x[p.siv:] = d["C_rand"]
    assert _sha(x) == str(d["xr_sha"])
    _set_pass(eng, name, p.x, p.K)
    f, g = _eval(eng, x, p.K, with_hs=False)
    dE, dg = abs(f - float(d["f_rand"])), normwise(g, d["g_rand"])
    print(f"PARITY lih_k1024 random C {name}: |dE|={dE:.2e} Eh g={dg:.2e}")
    assert dE < TOL_E and dg < TOL_G


def test_lih_k1024_host_entry_point(lih1024):
    """necg_outprod_host (the call the bench's end-to-end figure times)."""
    from nbo_correlatedgaussians_b200 import autotune
    p, d, eng = lih1024
    autotune.tuned(eng, p.x, p.K)
    f, g = eng.outprod(p.x)
    dE, dg = abs(f - float(d["f"])), normwise(g, d["g"])
    print(f"PARITY lih_k1024 host entry: |dE|={dE:.2e} Eh g={dg:.2e}")
    assert dE < TOL_E and dg < TOL_G


@pytest.mark.parametrize("name", ["tuned", "ordered"])
def test_h2_k2048(name):
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.engine import Engine
    d = golden("fullsize_h2_k2048.npz")
    p = synth.workload("h2_k2048")
    assert _sha(p.x) == str(d["x_sha"])
    eng = Engine(p)
    _set_pass(eng, name, p.x, p.K)
    f, g, H, S = _eval(eng, p.x, p.K)
    dE, dg = abs(f - float(d["f"])), normwise(g, d["g"])
    eH, eS = _hs_err(H, d, "H"), _hs_err(S, d, "S")
    print(f"PARITY h2_k2048 {name}: |dE|={dE:.2e} Eh g={dg:.2e} H={eH:.2e} S={eS:.2e}")
    eng.close()
    assert dE < TOL_E and dg < TOL_G
    assert eH < TOL_ELEM and eS < TOL_ELEM


def test_mixed_batch_largest_lih():
    """The largest LiH instance of the 64-instance mixed batch, per call and
    inside one batched step over all 64 instances."""
    import torch
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.batch import BatchEngine
    from nbo_correlatedgaussians_b200.engine import Engine
    insts = synth.workload("mixed64")
    d = golden("fullsize_lih_k731.npz")
    i = int(d["index"])
    p = insts[i]
    assert p.K == int(d["K"]) and _sha(p.x) == str(d["x_sha"])
    eng = Engine(p)
    _set_pass(eng, "tuned", p.x, p.K)
    f1, g1 = _eval(eng, p.x, p.K, with_hs=False)
    eng.close()
    be = BatchEngine(insts, tune=False)
    be.plan()
    be.step()
    torch.cuda.synchronize()
    be.check()
    f2, g2 = be.results(i)
    be.close()
    dE1, dg1 = abs(f1 - float(d["f"])), normwise(g1, d["g"])
    dE2, dg2 = abs(f2 - float(d["f"])), normwise(g2, d["g"])
    print(f"PARITY mixed64 LiH K={p.K} per call: |dE|={dE1:.2e} Eh g={dg1:.2e}; "
          f"batched: |dE|={dE2:.2e} Eh g={dg2:.2e}")
    assert dE1 < TOL_E and dg1 < TOL_G
    assert dE2 < TOL_E and dg2 < TOL_G


def test_serving_stream_largest_runs():
    """The largest LiH run (K=1928) and the largest He run (K=2032) of the
    256-run serving stream, per call with the tuned pass and together in one
    batched step (the step the serving loop runs)."""
    import torch
    from nbo_correlatedgaussians_b200 import synth
    from nbo_correlatedgaussians_b200.batch import BatchEngine
    from nbo_correlatedgaussians_b200.engine import Engine
    runs = synth.workload("serve256")
    fixtures = [golden("fullsize_serve_lih.npz"), golden("fullsize_serve_he.npz")]
    probs = []
    for d in fixtures:
        p = runs[int(d["index"])]
        assert p.K == int(d["K"]) and _sha(p.x) == str(d["x_sha"])
        probs.append(p)
        eng = Engine(p)
        _set_pass(eng, "tuned", p.x, p.K)
        f, g = _eval(eng, p.x, p.K, with_hs=False)
        eng.close()
        dE, dg = abs(f - float(d["f"])), normwise(g, d["g"])
        print(f"PARITY serve256 run {int(d['index'])} (n={p.n}, K={p.K}) per call: |dE|={dE:.2e} Eh g={dg:.2e}")
        assert dE < TOL_E and dg < TOL_G
    be = BatchEngine(probs, tune=True)
    be.plan()
    be.step()
    torch.cuda.synchronize()
    be.check()
    for i, d in enumerate(fixtures):
        f, g = be.results(i)
        dE, dg = abs(f - float(d["f"])), normwise(g, d["g"])
        print(f"PARITY serve256 run {int(d['index'])} batched: |dE|={dE:.2e} Eh g={dg:.2e}")
        assert dE < TOL_E and dg < TOL_G
    be.close()
