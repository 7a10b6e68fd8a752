"""necg_outprod_noalloc: the evaluation for callers that cannot allocate device
memory (their own fixed memory pool, no tolerance for an allocation's implicit
synchronisation, or a foreign-language host with no device allocator).  It
uses only the library's fixed scratch array; this test calls it through the C
ABI twice in a row and compares each result with the handle-based necg_outprod
at the tolerances of the other parity tests.  The file sorts last so that a
run stopping at its first failure has already run every other test; it also
passes on its own in a fresh process (the first call sets up the scratch
address)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_E = 1e-10
TOL_G = 1e-9


def _noalloc(L, p, x, f, g):
    c = [np.ascontiguousarray(a, dtype=np.float64) for a in (p.mass, p.ncv, p.scvv, p.sml, p.sms)]
    return L.necg_outprod_noalloc(p.n, p.nst, p.K, float(p.efs), *[a.ctypes.data for a in c], x.data_ptr(),
                                  f.data_ptr(), g.data_ptr(), None)


@pytest.mark.parametrize("system,K", [("He", 70), ("H2", 150), ("LiH", 96)])
def test_noalloc_matches_handle_path_twice(system, K):
    import torch
    from nbo_correlatedgaussians_b200 import _lib, synth
    from nbo_correlatedgaussians_b200.engine import Engine
    L = _lib.lib()
    p = synth.make_problem(system, K, 41 + K)
    p.C = np.random.default_rng(K).normal(size=K)
    x = torch.from_numpy(p.x).cuda()
    f_ref, g_ref = Engine(p).outprod_device(x, K)
    torch.cuda.synchronize()
    f_ref, g_ref = float(f_ref.item()), g_ref.cpu().numpy()
    for _ in range(2):
        f = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
        g = torch.full_like(x, np.nan)
        assert _noalloc(L, p, x, f, g) == _lib.NECG_OK
        gn = g.cpu().numpy()
        assert abs(float(f.item()) - f_ref) < TOL_E
        assert np.max(np.abs(gn - g_ref)) / np.max(np.abs(g_ref)) < TOL_G


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
