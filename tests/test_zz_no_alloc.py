"""necg_outprod_noalloc: the evaluation for callers that cannot allocate device
memory (their own fixed memory pool, no tolerance for an allocation's implicit
synchronisation, or a foreign-language host with no device allocator).  It
uses only the library's fixed scratch array; these tests call it through the C
ABI and compare each result with the handle-based necg_outprod at the
tolerances of the other parity tests: twice in a row, at the largest sizes the
array accepts, across calls whose scratch layouts differ, and on the
non-positive-definite status path.  The free device memory is checked to be
unchanged across a call.  The file sorts last so that a run stopping at its
first failure has already run every other test; it also passes on its own in a
fresh process (the first call sets up the scratch address)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_E = 1e-10
TOL_G = 1e-9
# the largest K whose intermediates fit the 32 MiB array, per system (n, nst)
K_LIMIT = {"LiH": 779, "H2": 1143, "He": 1247}


def _noalloc(L, p, x, f, g):
    c = [np.ascontiguousarray(a, dtype=np.float64) for a in (p.mass, p.ncv, p.scvv, p.sml, p.sms)]
    return L.necg_outprod_noalloc(p.n, p.nst, p.K, float(p.efs), *[a.ctypes.data for a in c], x.data_ptr(),
                                  f.data_ptr(), g.data_ptr(), None)


def _problem(system, K, seed):
    from nbo_correlatedgaussians_b200 import synth
    p = synth.make_problem(system, K, seed)
    p.C = np.random.default_rng(seed).normal(size=K)
    return p


def _handle_result(p):
    import torch
    from nbo_correlatedgaussians_b200.engine import Engine
    x = torch.from_numpy(p.x).cuda()
    eng = Engine(p)
    f, g = eng.outprod_device(x, p.K)
    torch.cuda.synchronize()
    out = float(f.item()), g.cpu().numpy()
    eng.close()
    return x, out


def _check_against(L, p, x, ref):
    import torch
    from nbo_correlatedgaussians_b200 import _lib
    f = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    g = torch.full_like(x, np.nan)
    assert _noalloc(L, p, x, f, g) == _lib.NECG_OK
    gn = g.cpu().numpy()
    assert abs(float(f.item()) - ref[0]) < TOL_E
    assert np.max(np.abs(gn - ref[1])) / np.max(np.abs(ref[1])) < TOL_G


@pytest.mark.parametrize("system,K", [("He", 70), ("H2", 150), ("LiH", 96)])
def test_noalloc_matches_handle_path_twice(system, K):
    from nbo_correlatedgaussians_b200 import _lib
    L = _lib.lib()
    p = _problem(system, K, 41 + K)
    x, ref = _handle_result(p)
    for _ in range(2):
        _check_against(L, p, x, ref)


def test_noalloc_allocates_no_device_memory():
    """Free device memory is the same before and after a call (the second one:
    the first may load the library's kernels, which lazy module loading places
    in device memory)."""
    import torch
    from nbo_correlatedgaussians_b200 import _lib
    L = _lib.lib()
    p = _problem("LiH", 200, 5)
    x = torch.from_numpy(p.x).cuda()
    f = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = torch.zeros_like(x)
    assert _noalloc(L, p, x, f, g) == _lib.NECG_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert _noalloc(L, p, x, f, g) == _lib.NECG_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


@pytest.mark.parametrize("system", ["LiH", "H2", "He"])
def test_noalloc_largest_accepted_size(system):
    """The largest K each system's layout fits in the array matches the handle
    path; one more basis function is refused with NECG_ERR_CAPACITY and writes
    nothing."""
    import torch
    from nbo_correlatedgaussians_b200 import _lib
    L = _lib.lib()
    K = K_LIMIT[system]
    p = _problem(system, K, 7 + K)
    x, ref = _handle_result(p)
    _check_against(L, p, x, ref)
    q = _problem(system, K + 1, 8 + K)
    xq = torch.from_numpy(q.x).cuda()
    f = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = torch.zeros_like(xq)
    assert _noalloc(L, q, xq, f, g) == _lib.NECG_ERR_CAPACITY
    torch.cuda.synchronize()
    assert torch.count_nonzero(g).item() == 0 and f.item() == 0.0


def test_noalloc_layouts_change_between_calls():
    """LiH K=96, then He K=70 (another scratch layout), then LiH K=96 again in one
    process: what an earlier call left in the shared array must not leak into a
    later one."""
    from nbo_correlatedgaussians_b200 import _lib
    L = _lib.lib()
    lih, he = _problem("LiH", 96, 31), _problem("He", 70, 32)
    x1, r1 = _handle_result(lih)
    x2, r2 = _handle_result(he)
    for p, x, r in ((lih, x1, r1), (he, x2, r2), (lih, x1, r1), (he, x2, r2)):
        _check_against(L, p, x, r)


def test_noalloc_not_positive_definite_then_recovers():
    """A basis function with L = 0 makes A_k + A_k' singular: the call returns
    NECG_ERR_NOT_PD (the reference's np.linalg.inv raises LinAlgError,
    python/matel.py:93); the next call on a good input is correct."""
    import torch
    from nbo_correlatedgaussians_b200 import _lib
    L = _lib.lib()
    p = _problem("LiH", 40, 9)
    x, ref = _handle_result(p)
    bad = p.copy()
    bad.iv[2 * p.blk:2 * p.blk + p.svh] = 0.0
    xb = torch.from_numpy(bad.x).cuda()
    f = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = torch.zeros_like(xb)
    assert _noalloc(L, bad, xb, f, g) == _lib.NECG_ERR_NOT_PD
    _check_against(L, p, x, ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from nbo_correlatedgaussians_b200 import _lib, synth
    L = _lib.lib()
    p = synth.make_problem("LiH", 1024, 1)
    x = torch.from_numpy(p.x).cuda()
    f = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = torch.zeros_like(x)
    assert _noalloc(L, p, x, f, g) == _lib.NECG_ERR_CAPACITY
    assert torch.count_nonzero(g).item() == 0
