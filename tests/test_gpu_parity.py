"""Parity of the sm_100a kernels (through the C ABI) with the reference's golden
vectors and with the CPU oracle.

Tolerances: elements 1e-12 relative; E 1e-10 Eh absolute; gradients 1e-9
relative norm-wise (max|g - g_ref| / max|g_ref|).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from oracle.oracle import Oracle  # noqa: E402
from _util import TOL_E, TOL_ELEM, TOL_G, elem_rel, golden, normwise, problem_from  # noqa: E402


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def _engine(p, K_max=None):
    from nbo_correlatedgaussians_b200.engine import Engine
    return Engine(p, K_max=K_max or p.K)


def test_f0_df0(torch_cuda):
    from nbo_correlatedgaussians_b200.engine import boys_f0
    d = golden("f0.npz")
    f, df = boys_f0(d["z"])
    assert np.max(np.abs(f - d["f0"]) / np.abs(d["f0"])) < 1e-14
    assert np.max(np.abs(df - d["df0"]) / np.abs(d["df0"])) < 1e-13


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_matel_gradel_elements(torch_cuda, system):
    d = golden(f"elements_{system}.npz")
    p = problem_from(d)
    eng = _engine(p)
    mat = eng.matel(p.iv, d["terms"])
    err = elem_rel(mat, d["matel"], efs=p.efs)
    assert err.max() < TOL_ELEM, err.max(axis=0)
    tg, tgs = eng.gradel(p.iv, d["terms"])
    assert normwise(tg, d["tgvl"]) < 1e-12
    assert normwise(tgs, d["tgvls"]) < 1e-12


def test_f0_branch_edge(torch_cuda):
    d = golden("f0_edge.npz")
    for tag in ("below", "above"):
        p = problem_from(d, iv=d[f"iv_{tag}"])
        eng = _engine(p)
        m = eng.matel(p.iv, [(1, 2, 1)])
        assert elem_rel(m, d[f"matel_{tag}"][None]).max() < TOL_ELEM
        tg, tgs = eng.gradel(p.iv, [(1, 2, 1)])
        assert normwise(tg[0], d[f"tgvl_{tag}"]) < 1e-12
        assert normwise(tgs[0], d[f"tgvls_{tag}"]) < 1e-12


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_outprod_golden(torch_cuda, system):
    d = golden(f"outprod_{system}.npz")
    p = problem_from(d)
    f, g = _engine(p).outprod(p.x)
    assert abs(f - float(d["E"])) < TOL_E
    assert normwise(g, d["g"]) < TOL_G


def test_oldquit_file_and_eigen_coefficients(torch_cuda):
    d = golden("oldquit.npz")
    p = problem_from(d)
    eng = _engine(p)
    f, g = eng.outprod(p.x)
    assert abs(f - 4.296758204100342) < TOL_E
    assert normwise(g, d["g"]) < TOL_G
    f2, g2 = eng.outprod(np.concatenate([p.iv, d["C_eig"]]))
    assert abs(f2 - (-7.023692395001888)) < TOL_E
    assert normwise(g2, d["g_eig"]) < TOL_G
    H, S, Kin, Pot, fb = eng.build_matrices(p.iv, p.C)
    assert normwise(H.cpu().numpy(), d["H"]) < 1e-12
    assert normwise(S.cpu().numpy(), d["S"]) < 1e-12
    assert abs(float(fb[0].item()) - 4.296758204100342) < TOL_E


@pytest.mark.parametrize("system,K", [("He", 64), ("H2", 64), ("LiH", 40)])
def test_outprod_vs_oracle(torch_cuda, system, K):
    from nbo_correlatedgaussians_b200 import synth
    p = synth.make_problem(system, K, 100 + K)
    p.C = np.random.default_rng(K).normal(size=K)  # general coefficients
    fo, go, Ho, So = Oracle.from_problem(p).outprod(p.x, nthreads=8, return_hs=True)
    eng = _engine(p)
    f, g = eng.outprod(p.x)
    assert abs(f - fo) < TOL_E
    assert normwise(g, go) < TOL_G
    H, S, Kin, Pot, _ = eng.build_matrices(p.iv)
    assert normwise(H.cpu().numpy(), Ho) < 1e-12
    assert normwise(S.cpu().numpy(), So) < 1e-12
    Hk, Sk, Ko, Po = Oracle.from_problem(p).build_matrices(p.iv, nthreads=8)
    assert normwise(Kin.cpu().numpy(), Ko) < 1e-12
    assert normwise(Pot.cpu().numpy(), Po) < 1e-12


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_edge_sizes_every_pass(torch_cuda, system):
    """One basis function, two, and the sizes either side of a 32-row block, in a
    handle made for a larger K_max: every pair pass (ordered, symmetric, fused
    with one-warp tiles, split terms and lockstep blocks) against the oracle."""
    from nbo_correlatedgaussians_b200 import _lib, synth
    from nbo_correlatedgaussians_b200.engine import Engine
    for K in (1, 2, 31, 32, 33):
        p = synth.make_problem(system, K, 900 + K)
        p.C = np.random.default_rng(K).normal(size=K)
        fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
        eng = Engine(p, K_max=40)
        L = eng.L
        for mode, lc, minw, npc in [(0, 4, 8, 1), (1, 2, 8, 1), (2, 2, 118, 1), (2, 1, 118, p.nst),
                                    (2, 2, 228, 1), (2, 1, 248, 1), (2, 2, 258, 1), (2, 1, 268, 1)]:
            assert L.necg_set_symmetric(eng.h, mode, lc, minw) == _lib.NECG_OK
            assert L.necg_set_splits(eng.h, npc) == _lib.NECG_OK
            f, g = eng.outprod(p.x)
            assert abs(f - fo) < TOL_E, (K, mode, minw, npc)
            assert normwise(g, go) < TOL_G, (K, mode, minw, npc)
        eng.close()


def test_make_grad_matches_outprod_gradient(torch_cuda):
    from nbo_correlatedgaussians_b200 import synth
    p = synth.make_problem("H2", 48, 7)
    eng = _engine(p)
    f, g = eng.outprod(p.x)
    H, S, _, _, _ = eng.build_matrices(p.iv, parts=False)
    Hn, Sn = H.cpu().numpy(), S.cpu().numpy()
    norm = 1.0 / float(p.C @ Sn @ p.C)
    g2 = eng.make_grad(p.iv, p.C, Hn, Sn, f, norm).cpu().numpy()
    assert normwise(g2, g) < 1e-13


def test_drop_in_modules(torch_cuda, tmp_path):
    """read_input -> matel / gradel / outprod / make_grad with the reference's
    module-level calling convention."""
    from nbo_correlatedgaussians_b200 import shared as sh
    from nbo_correlatedgaussians_b200.gradel import gradel
    from nbo_correlatedgaussians_b200.make_grad import make_grad
    from nbo_correlatedgaussians_b200.matel import matel
    from nbo_correlatedgaussians_b200.outprod import outprod
    from nbo_correlatedgaussians_b200.problem import write_oldquit
    from nbo_correlatedgaussians_b200.read_input import read_input
    from nbo_correlatedgaussians_b200.utils import df0, f0
    d = golden("oldquit.npz")
    fn = tmp_path / "oldquit.dat"
    write_oldquit(problem_from(d), str(fn))
    read_input(str(fn))
    e = golden("elements_LiH.npz")  # different basis: only check self-consistency here
    x = np.concatenate([sh.iv, sh.C])
    f, g = outprod(x)
    assert abs(f - 4.296758204100342) < TOL_E and normwise(g, d["g"]) < TOL_G
    assert normwise(sh.H, d["H"]) < 1e-12 and np.array_equal(sh.grad, g)
    make_grad(f, 1.0 / float(sh.C @ sh.S @ sh.C))
    assert normwise(sh.grad, g) < 1e-13
    o = Oracle.from_problem(problem_from(d))
    for t in [(1, 1, 1), (5, 3, 7), (24, 12, 4), (11, 6, 6)]:
        ref = np.array(o.matel(sh.iv, *t))
        assert elem_rel(np.array(matel(*t))[None], ref[None], efs=sh.efs).max() < TOL_ELEM
        tg, tgs = gradel(*t)
        rg, rgs = o.gradel(sh.iv, *t)
        # the bra gradient of the identity self-overlap is analytically zero, so
        # both sides are rounding noise there: floor the scale at the overlap
        scale = max(np.abs(rgs).max(), abs(ref[0]))
        assert normwise(tg, rg) < 1e-12 and np.abs(tgs - rgs).max() < 1e-12 * scale
    assert abs(f0(0.5) - o.f0(0.5)) < 1e-15 and abs(df0(20.0) - o.df0(20.0)) < 1e-15
    del e


def test_full_size_properties(torch_cuda):
    """LiH K=1024 (the benchmark workload): properties that hold at any size.
    E is invariant under C -> a C, so g_C . C = 0; the directional derivative
    of E along a random unit direction matches g . u (5-point stencil)."""
    torch = torch_cuda
    from nbo_correlatedgaussians_b200 import synth
    p = synth.workload("lih_k1024")
    eng = _engine(p)
    x = torch.from_numpy(p.x).cuda()
    f, g = eng.outprod_device(x, p.K)
    eng.raise_status("outprod")
    f = float(f.item())
    g = g.cpu().numpy()
    assert np.isfinite(f) and np.isfinite(g).all()
    gC = g[p.siv:]
    assert abs(gC @ p.C) < 1e-10 * np.abs(gC).sum() * np.abs(p.C).max() + 1e-15
    f3, _ = eng.outprod_device(torch.from_numpy(np.concatenate([p.iv, 3.0 * p.C])).cuda(), p.K)
    assert abs(float(f3.item()) - f) < 1e-12 * abs(f)
    u = np.random.default_rng(0).normal(size=p.x.size)
    u /= np.linalg.norm(u)
    h = 1e-4
    vals = []
    for s in (-2, -1, 1, 2):
        fs, _ = eng.outprod_device(torch.from_numpy(p.x + s * h * u).cuda(), p.K)
        vals.append(float(fs.item()))
    fd = (vals[0] - 8 * vals[1] + 8 * vals[2] - vals[3]) / (12 * h)
    assert abs(fd - g @ u) < 1e-6 * max(abs(g @ u), np.abs(g).max())
    # deterministic: the same call twice gives identical bits
    f_a, g_a = eng.outprod_device(x, p.K)
    f_b, g_b = eng.outprod_device(x, p.K)
    assert torch.equal(g_a, g_b) and torch.equal(f_a, f_b)


def test_errors(torch_cuda):
    from nbo_correlatedgaussians_b200 import _lib, synth
    p = synth.make_problem("He", 8, 3)
    eng = _engine(p)
    with pytest.raises(_lib.NecgError):
        eng.outprod_device(np.zeros(9 * 9 + 9), 9)  # K > K_max
    bad = p.copy()
    bad.iv[2 * p.blk:2 * p.blk + p.svh] = 0.0  # L_3 = 0: A_3 + A_3' singular
    with pytest.raises(np.linalg.LinAlgError):
        eng.outprod(bad.x)
    # the handle stays usable after the error
    f, g = eng.outprod(p.x)
    assert np.isfinite(f)


@pytest.mark.parametrize("system,K", [("He", 80), ("H2", 90), ("LiH", 70)])
def test_symmetric_and_ordered_gradient_passes_agree(torch_cuda, system, K):
    """The unordered-pair gradient pass (bra and ket gradient per term) against
    the ordered pass of the reference's loop structure and against the oracle."""
    from nbo_correlatedgaussians_b200 import _lib, synth
    p = synth.make_problem(system, K, 5 * K)
    p.C = np.random.default_rng(K).normal(size=K)
    eng = _engine(p)
    L = eng.L
    assert L.necg_set_symmetric(eng.h, 1, 4, 8) == _lib.NECG_OK
    fs, gs = eng.outprod(p.x)
    assert L.necg_set_symmetric(eng.h, 1, 7, 12) == _lib.NECG_OK
    fs2, gs2 = eng.outprod(p.x)
    assert L.necg_set_symmetric(eng.h, 0, 4, 8) == _lib.NECG_OK
    fo, go = eng.outprod(p.x)
    fr, gr = Oracle.from_problem(p).outprod(p.x, nthreads=8)
    assert fs == fo == fs2  # the energy pass is shared
    assert normwise(gs, gr) < TOL_G and normwise(gs2, gr) < TOL_G and normwise(go, gr) < TOL_G
    assert normwise(gs, go) < 1e-12


@pytest.mark.parametrize("system,K,lc", [("He", 80, 3), ("H2", 90, 2), ("LiH", 70, 4), ("LiH", 101, 16)])
def test_fused_pass_matches_oracle(torch_cuda, system, K, lc):
    """Mode 2: one pass over unordered pairs writes H and S and the H and S
    gradients; E, g, H and S against the oracle for each register variant, and
    the gradient against the two-pass symmetric mode."""
    import torch
    from nbo_correlatedgaussians_b200 import _lib, synth
    p = synth.make_problem(system, K, 7 * K)
    p.C = np.random.default_rng(K).normal(size=K)
    eng = _engine(p)
    L = eng.L
    assert L.necg_set_symmetric(eng.h, 1, lc, 8) == _lib.NECG_OK
    f1, g1 = eng.outprod(p.x)
    fr, gr, Hr, Sr = Oracle.from_problem(p).outprod(p.x, nthreads=8, return_hs=True)
    for minw in (8, 12, 16, 108, 112, 118, 122, 208, 218, 228, 222, 232, 248, 258, 268):
        rc = L.necg_set_symmetric(eng.h, 2, lc, minw)
        if rc == _lib.NECG_ERR_UNSUPPORTED and minw in (222, 232) and p.n == 5:
            continue  # 12 warps of n = 5 do not fit in shared memory
        assert rc == _lib.NECG_OK
        H = torch.empty((K, K), dtype=torch.float64, device=eng.device)
        S = torch.empty_like(H)
        fd, gd = eng.outprod_device(torch.from_numpy(p.x), K, H=H, S=S)
        torch.cuda.synchronize()
        eng.raise_status("outprod")
        f2, g2 = eng.outprod(p.x)
        assert float(fd.item()) == f2 and np.array_equal(gd.cpu().numpy(), g2)
        assert abs(f2 - fr) < TOL_E and normwise(g2, gr) < TOL_G
        assert abs(f2 - f1) < TOL_E and normwise(g2, g1) < 1e-12
        Hn, Sn = H.cpu().numpy(), S.cpu().numpy()
        assert np.array_equal(Hn, Hn.T) and np.array_equal(Sn, Sn.T)
        assert np.max(np.abs(Hn - Hr)) <= TOL_ELEM * max(1.0, np.max(np.abs(Hr)))
        assert np.max(np.abs(Sn - Sr)) <= TOL_ELEM * max(1.0, np.max(np.abs(Sr)))


@pytest.mark.parametrize("system,K,lc", [("He", 40, 2), ("H2", 33, 1), ("LiH", 12, 2), ("LiH", 70, 4)])
def test_fused_pass_split_terms(torch_cuda, system, K, lc):
    """The fused pass with the symmetry terms of each tile split over npc warps
    (necg_set_splits): E, g, H and S against the oracle and against the unsplit
    pass for every split count, one-warp variants; lockstep variants ignore
    the setting."""
    import torch
    from nbo_correlatedgaussians_b200 import _lib, synth
    p = synth.make_problem(system, K, 5 * K + 1)
    p.C = np.random.default_rng(K + 1).normal(size=K)
    eng = _engine(p)
    L = eng.L
    fr, gr, Hr, Sr = Oracle.from_problem(p).outprod(p.x, nthreads=8, return_hs=True)
    for minw in (8, 118, 122):
        assert L.necg_set_symmetric(eng.h, 2, lc, minw) == _lib.NECG_OK
        assert L.necg_set_splits(eng.h, 1) == _lib.NECG_OK
        f1, g1 = eng.outprod(p.x)
        for npc in sorted({q for q in (2, 3, p.nst // 2, p.nst) if 1 <= q <= p.nst}):
            assert L.necg_set_splits(eng.h, npc) == _lib.NECG_OK
            H = torch.empty((K, K), dtype=torch.float64, device=eng.device)
            S = torch.empty_like(H)
            fd, gd = eng.outprod_device(torch.from_numpy(p.x), K, H=H, S=S)
            torch.cuda.synchronize()
            eng.raise_status("outprod")
            f2, g2 = float(fd.item()), gd.cpu().numpy()
            assert abs(f2 - fr) < TOL_E and normwise(g2, gr) < TOL_G
            assert abs(f2 - f1) < 1e-12 * max(1.0, abs(f1)) and normwise(g2, g1) < 1e-12
            Hn, Sn = H.cpu().numpy(), S.cpu().numpy()
            assert np.array_equal(Hn, Hn.T) and np.array_equal(Sn, Sn.T)
            assert np.max(np.abs(Hn - Hr)) <= TOL_ELEM * max(1.0, np.max(np.abs(Hr)))
            assert np.max(np.abs(Sn - Sr)) <= TOL_ELEM * max(1.0, np.max(np.abs(Sr)))
            f3, g3 = eng.outprod(p.x)  # deterministic: fixed summation order
            assert f3 == f2 and np.array_equal(g3, g2)
    assert L.necg_set_splits(eng.h, 0) == _lib.NECG_ERR_ARG
    assert L.necg_set_splits(eng.h, p.nst + 1) == _lib.NECG_ERR_ARG
    assert L.necg_set_symmetric(eng.h, 2, lc, 218) == _lib.NECG_OK
    assert L.necg_set_splits(eng.h, 1) == _lib.NECG_OK
    fb, gb = eng.outprod(p.x)
    assert L.necg_set_splits(eng.h, 2) == _lib.NECG_OK
    fb2, gb2 = eng.outprod(p.x)
    assert fb2 == fb and np.array_equal(gb2, gb)
    # the pair-status path with splits: the first failing pair and a usable handle
    assert L.necg_set_symmetric(eng.h, 2, lc, 118) == _lib.NECG_OK
    assert L.necg_set_splits(eng.h, min(4, p.nst)) == _lib.NECG_OK
    bad = p.copy()
    bad.iv[2 * p.blk:2 * p.blk + p.svh] = 0.0
    with pytest.raises(np.linalg.LinAlgError):
        eng.outprod(bad.x)
    assert eng.status()[1] == 2 * K + 2
    f4, g4 = eng.outprod(p.x)
    assert abs(f4 - fr) < TOL_E and normwise(g4, gr) < TOL_G


@pytest.mark.parametrize("minw", [8, 118, 208, 228, 248, 258, 268])
def test_fused_pass_oldquit_and_errors(torch_cuda, minw):
    """The fused mode on the reference's input file, and the pair-status path
    (a singular A_k + A_l') leaving the handle usable, for one-warp and lockstep
    blocks."""
    from nbo_correlatedgaussians_b200 import _lib
    d = golden("oldquit.npz")
    p = problem_from(d)
    eng = _engine(p)
    assert eng.L.necg_set_symmetric(eng.h, 2, 4, minw) == _lib.NECG_OK
    f, g = eng.outprod(p.x)
    assert abs(f - 4.296758204100342) < TOL_E and normwise(g, d["g"]) < TOL_G
    bad = p.copy()
    bad.iv[2 * p.blk:2 * p.blk + p.svh] = 0.0
    with pytest.raises(np.linalg.LinAlgError):
        eng.outprod(bad.x)
    rc, pair = eng.status()
    assert rc == _lib.NECG_ERR_NOT_PD and pair == 2 * p.K + 2  # the pair (3, 3), 1-based
    f2, g2 = eng.outprod(p.x)
    assert f2 == f and np.array_equal(g2, g)


def test_symmetric_pass_unavailable_without_inverse_closure(torch_cuda):
    from nbo_correlatedgaussians_b200 import _lib, synth
    p = synth.make_problem("H2", 20, 4)
    keep = [0, 2]  # identity and the proton swap: closed
    q = p.copy()
    q.sml, q.sms, q.scvv = p.sml[[0, 1]], p.sms[[0, 1]], p.scvv[[0, 1]]
    assert _engine(q).L.necg_set_symmetric(_engine(q).h, 1, 4, 8) == _lib.NECG_OK
    r = p.copy()  # a lone non-involutory map has no inverse in the set
    M = np.array([[1.0, 0, 0], [0, 0, 1.0], [0, 1.0, 0]]) @ np.array([[1.0, 0, 0], [1.0, 1.0, 0], [0, 0, 1.0]])
    r.sml = np.stack([np.eye(3), M])
    r.sms = np.stack([np.eye(9), np.kron(np.linalg.inv(M), np.eye(3))])
    r.scvv = np.array([0.5, 0.5])
    e = _engine(r)
    assert e.L.necg_set_symmetric(e.h, 1, 4, 8) == _lib.NECG_ERR_UNSUPPORTED
    f, g = e.outprod(r.x)  # ordered pass still works
    fo, go = Oracle.from_problem(r).outprod(r.x, nthreads=4)
    assert abs(f - fo) < TOL_E and normwise(g, go) < TOL_G
    del keep


def _lockstep_tail_parts(K, lc, nst, sms, gw=8):
    """Parts the host splits each of the lockstep queue's last groups into (the
    rule of the library's tile builder): G groups, T = G mod SMs of them split
    into min(4, nst, SMs // T) parts, capped so the units fit the tile slots."""
    G = tiles = 0
    for kb in range((K + 31) // 32):
        t = min(kb * 32 + 31, K - 1) // lc + 1
        tiles += t
        G += -(-t // gw)
    T = G % sms
    if not T:
        return 1
    parts = min(8, nst, sms // T)
    return min(parts, 1 + (tiles - G) // T)


def test_lockstep_queue_tail_split(torch_cuda):
    """The lockstep pass (variant 258) splits the groups of its queue's last,
    partial round over the symmetry terms and adds the parts in a fix-up
    kernel.  At LiH sizes whose tails split 2, 1 (not at all), 8 and 3 ways on a
    148-SM B200, E, g, H and S must match the one-warp pass (variant 118, which
    has no queue) to rounding: a lost or doubled part would be an O(1) error."""
    import torch
    from nbo_correlatedgaussians_b200 import _lib, synth
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    seen = set()
    for K in (200, 257, 353, 545):
        p = synth.make_problem("LiH", K, 60 + K)
        p.C = np.random.default_rng(K).normal(size=K)
        eng = _engine(p)
        res = {}
        for minw in (118, 258):
            assert eng.L.necg_set_symmetric(eng.h, 2, 2, minw) == _lib.NECG_OK
            assert eng.L.necg_set_splits(eng.h, 1) == _lib.NECG_OK
            H = torch.empty((K, K), dtype=torch.float64, device=eng.device)
            S = torch.empty_like(H)
            f, g = eng.outprod_device(torch.from_numpy(p.x), K, H=H, S=S)
            torch.cuda.synchronize()
            eng.raise_status("outprod")
            res[minw] = (float(f.item()), g.cpu().numpy(), H.cpu().numpy(), S.cpu().numpy())
        eng.close()
        seen.add(_lockstep_tail_parts(K, 2, p.nst, sms))
        (f1, g1, H1, S1), (f2, g2, H2, S2) = res[118], res[258]
        assert abs(f2 - f1) <= 1e-12 * abs(f1), K
        assert normwise(g2, g1) < 1e-11, K
        assert np.max(np.abs(H2 - H1)) <= 1e-13 * np.max(np.abs(H1)), K
        assert np.max(np.abs(S2 - S1)) <= 1e-13 * np.max(np.abs(S1)), K
        assert np.array_equal(H2, H2.T) and np.array_equal(S2, S2.T)
    if sms == 148:
        assert seen == {1, 2, 3, 8}


@pytest.mark.parametrize("minw,npc", [(258, 1), (118, 4)])
def test_fused_graph_replay(torch_cuda, minw, npc):
    """A call that repeats the previous call's buffers, K and settings replays
    the fused pass's launch sequence as a captured CUDA graph (from the third
    such call on).  Its results must be bitwise those of eager launches, it must
    read new contents of the same x buffer, and a settings change must leave it."""
    import torch
    from nbo_correlatedgaussians_b200 import _lib, synth
    p = synth.make_problem("LiH", 40, 11)
    p.C = np.random.default_rng(3).normal(size=40)
    eng = _engine(p)
    L = eng.L
    assert L.necg_set_symmetric(eng.h, 2, 2, minw) == _lib.NECG_OK
    assert L.necg_set_splits(eng.h, npc) == _lib.NECG_OK
    x = torch.from_numpy(p.x).cuda()
    g = torch.empty_like(x)
    f = torch.empty(1, dtype=torch.float64, device="cuda")
    outs = []
    for _ in range(5):  # eager, eager + capture, then replays
        eng.outprod_device(x, p.K, g=g, f=f)
        torch.cuda.synchronize()
        eng.raise_status("outprod")
        outs.append((float(f.item()), g.cpu().numpy().copy()))
    for fo, go in outs[1:]:
        assert fo == outs[0][0] and np.array_equal(go, outs[0][1])
    fr, gr = Oracle.from_problem(p).outprod(p.x, nthreads=8)
    assert abs(outs[0][0] - fr) < TOL_E and normwise(outs[0][1], gr) < TOL_G
    # new contents in the same buffer: the replay reads them
    q = p.copy()
    q.iv = q.iv * 1.01
    x.copy_(torch.from_numpy(q.x))
    eng.outprod_device(x, p.K, g=g, f=f)
    torch.cuda.synchronize()
    f2, g2 = float(f.item()), g.cpu().numpy().copy()
    fe, ge = eng.outprod_device(torch.from_numpy(q.x).cuda(), p.K)  # other buffers: eager
    torch.cuda.synchronize()
    assert f2 == float(fe.item()) and np.array_equal(g2, ge.cpu().numpy())
    # a non-positive-definite input through the replay, then a good one
    bad = p.copy()
    bad.iv[2 * p.blk:2 * p.blk + p.svh] = 0.0
    x.copy_(torch.from_numpy(bad.x))
    eng.outprod_device(x, p.K, g=g, f=f)
    with pytest.raises(np.linalg.LinAlgError):
        eng.raise_status("outprod")
    x.copy_(torch.from_numpy(p.x))
    eng.outprod_device(x, p.K, g=g, f=f)
    torch.cuda.synchronize()
    eng.raise_status("outprod")
    assert float(f.item()) == outs[0][0] and np.array_equal(g.cpu().numpy(), outs[0][1])
    eng.close()
