"""The kernels' per-thread bodies, run on the host by the test emulator
(tests/emu), against the golden vectors and the oracle.  This checks the device
algorithm -- tile and lane ranges, ket records, reductions, the A-space to
vech(L) mapping -- on CPU; the GPU parity tests check the compiled kernels."""
import numpy as np
import pytest

from emu import emu
from oracle.oracle import Oracle
from nbo_correlatedgaussians_b200 import synth
from _util import TOL_E, TOL_ELEM, TOL_G, elem_rel, golden, normwise, problem_from, rrms_rel


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_elements_vs_golden(system):
    d = golden(f"elements_{system}.npz")
    p = problem_from(d)
    rc, mat, tg, tgs = emu.elements(p, d["terms"])
    assert rc == 0
    assert elem_rel(mat, d["matel"], efs=p.efs).max() < TOL_ELEM
    assert normwise(tg, d["tgvl"]) < 1e-12
    assert normwise(tgs, d["tgvls"]) < 1e-12


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_outprod_vs_golden(system):
    d = golden(f"outprod_{system}.npz")
    p = problem_from(d)
    rc, f, g, H, S = emu.outprod(p)
    assert rc == 0
    assert abs(f - float(d["E"])) < TOL_E
    assert normwise(g, d["g"]) < TOL_G
    assert normwise(H, d["H"]) < 1e-12 and normwise(S, d["S"]) < 1e-12


def test_oldquit():
    d = golden("oldquit.npz")
    p = problem_from(d)
    rc, f, g, H, S = emu.outprod(p)
    assert rc == 0 and abs(f - 4.296758204100342) < TOL_E and normwise(g, d["g"]) < TOL_G


@pytest.mark.parametrize("system,K,lc_e,lc_g", [("He", 45, 1, 4), ("He", 45, 7, 5), ("H2", 37, 3, 9),
                                                ("H2", 70, 8, 16), ("LiH", 33, 4, 4), ("LiH", 33, 64, 64)])
def test_outprod_vs_oracle_ragged_tiles(system, K, lc_e, lc_g):
    """K not a multiple of the warp width, tile widths that do not divide K."""
    p = synth.make_problem(system, K, 7 * K)
    p.C = np.random.default_rng(K).normal(size=K)
    fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
    rc, f, g, H, S = emu.outprod(p, lc_e, lc_g)
    assert rc == 0
    assert abs(f - fo) < TOL_E
    assert normwise(g, go) < TOL_G


def test_single_basis_function():
    p = synth.make_problem("H2", 1, 3)
    fo, go = Oracle.from_problem(p).outprod(p.x)
    rc, f, g, H, S = emu.outprod(p, 1, 4)
    assert rc == 0 and abs(f - fo) < TOL_E and normwise(g, go) < TOL_G


def test_not_positive_definite_flag():
    p = synth.make_problem("He", 5, 3)
    p.iv[2 * p.blk:2 * p.blk + p.svh] = 0.0
    rc, f, g, H, S = emu.outprod(p)
    assert rc & 1


@pytest.mark.parametrize("system,K,lc_s", [("He", 45, 1), ("He", 45, 6), ("H2", 37, 3), ("H2", 70, 8),
                                           ("LiH", 33, 4), ("LiH", 40, 7)])
def test_symmetric_pass_vs_oracle(system, K, lc_s):
    """Unordered pairs with bra and ket gradients from one term, ket gradients
    mapped back through each symmetry term's inverse frame."""
    p = synth.make_problem(system, K, 11 * K)
    p.C = np.random.default_rng(K + 1).normal(size=K)
    fo, go = Oracle.from_problem(p).outprod(p.x, nthreads=8)
    rc, f, g, H, S = emu.outprod_sym(p, 4, lc_s)
    assert rc == 0
    assert abs(f - fo) < TOL_E
    assert normwise(g, go) < TOL_G


def test_symmetric_pass_oldquit():
    d = golden("oldquit.npz")
    p = problem_from(d)
    rc, f, g, H, S = emu.outprod_sym(p, 4, 4)
    assert rc == 0 and abs(f - 4.296758204100342) < TOL_E and normwise(g, d["g"]) < TOL_G


@pytest.mark.parametrize("system,K,lc_s", [("He", 45, 1), ("He", 45, 6), ("H2", 37, 3), ("H2", 70, 8),
                                           ("LiH", 33, 4), ("LiH", 40, 7)])
def test_fused_pass_vs_oracle(system, K, lc_s):
    """One pass over unordered pairs for H, S and the split H and S gradients,
    combined as g_H - E g_S once E is known."""
    p = synth.make_problem(system, K, 11 * K)
    p.C = np.random.default_rng(K + 1).normal(size=K)
    fo, go, Ho, So = Oracle.from_problem(p).outprod(p.x, nthreads=8, return_hs=True)
    rc, f, g, H, S = emu.outprod_fused(p, lc_s)
    assert rc == 0
    assert abs(f - fo) < TOL_E
    assert normwise(g, go) < TOL_G
    assert np.max(np.abs(H - Ho)) <= TOL_ELEM * max(1.0, np.max(np.abs(Ho)))
    assert np.max(np.abs(S - So)) <= TOL_ELEM * max(1.0, np.max(np.abs(So)))


def test_fused_pass_oldquit():
    d = golden("oldquit.npz")
    p = problem_from(d)
    rc, f, g, H, S = emu.outprod_fused(p, 4)
    assert rc == 0 and abs(f - 4.296758204100342) < TOL_E and normwise(g, d["g"]) < TOL_G


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_rrms_terms_vs_golden(system):
    d = golden(f"rrms_{system}.npz")
    rc, out = emu.rrms(problem_from(d), d["terms"])
    assert rc == 0 and rrms_rel(out, d["rrms"]).max() < TOL_ELEM


@pytest.mark.parametrize("system,K,lc", [("He", 45, 2), ("H2", 37, 3), ("LiH", 20, 4)])
def test_dipole_vs_oracle(system, K, lc):
    """The dipole tiles (lower triangle, nst^2 symmetry pairs, C contracted on
    the fly) against the oracle's matrices of python/necg.py:200-244."""
    p = synth.make_problem(system, K, 17 * K)
    p.C = np.random.default_rng(K).normal(size=K)
    comps_o, dip_o = Oracle.from_problem(p).dipole(p.iv, p.C, nthreads=8)
    rc, comps, dip = emu.dipole(p, lc)
    assert rc == 0
    scale = max(np.max(np.abs(comps_o)), 1e-300)
    assert np.max(np.abs(comps - comps_o)) <= 1e-11 * scale
    assert np.max(np.abs(dip - dip_o)) <= 1e-11 * max(np.max(np.abs(dip_o)), scale)


def test_dipole_oldquit_optimum():
    d = golden("driver_oldquit.npz")
    p = problem_from(golden("oldquit.npz"))
    x = d["x_opt"]
    p.iv, p.C = x[:p.K * p.blk].copy(), x[p.K * p.blk:].copy()
    rc, comps, dip = emu.dipole(p, 4)
    assert rc == 0 and np.max(np.abs(comps - d["dip_comps"])) < 1e-12 and np.max(np.abs(dip - d["dipole"])) < 1e-12
