"""The CPU oracle (oracle/necg_oracle.c) against golden vectors produced by
executing the reference Python package (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from _util import TOL_E, TOL_ELEM, elem_rel, golden, normwise, problem_from, rrms_rel


def test_f0_df0():
    d = golden("f0.npz")
    o = Oracle(2, 1, 0.0, np.eye(2), np.zeros(3), np.ones(1), np.eye(2)[None], np.eye(6)[None])
    f = np.array([o.f0(z) for z in d["z"]])
    df = np.array([o.df0(z) for z in d["z"]])
    assert np.max(np.abs(f - d["f0"]) / np.abs(d["f0"])) < 1e-15
    assert np.max(np.abs(df - d["df0"]) / np.abs(d["df0"])) < 1e-14


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_elements(system):
    d = golden(f"elements_{system}.npz")
    p = problem_from(d)
    o = Oracle.from_problem(p)
    mat = np.array([o.matel(p.iv, *t) for t in d["terms"]])
    assert elem_rel(mat, d["matel"], efs=p.efs).max() < TOL_ELEM
    tg = np.stack([o.gradel(p.iv, *t)[0] for t in d["terms"]])
    tgs = np.stack([o.gradel(p.iv, *t)[1] for t in d["terms"]])
    assert normwise(tg, d["tgvl"]) < 1e-12
    assert normwise(tgs, d["tgvls"]) < 1e-12


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_outprod_small(system):
    d = golden(f"outprod_{system}.npz")
    p = problem_from(d)
    f, g, H, S = Oracle.from_problem(p).outprod(p.x, nthreads=2, return_hs=True)
    assert abs(f - float(d["E"])) < 1e-12
    assert normwise(g, d["g"]) < 1e-12
    assert normwise(H, d["H"]) < 1e-13 and normwise(S, d["S"]) < 1e-13


def test_oldquit():
    d = golden("oldquit.npz")
    p = problem_from(d)
    o = Oracle.from_problem(p)
    f, g = o.outprod(p.x, nthreads=4)
    assert abs(f - float(d["E"])) < TOL_E
    assert abs(f - 4.296758204100342) < 1e-12
    assert normwise(g, d["g"]) < 1e-12
    f2, g2 = o.outprod(np.concatenate([p.iv, d["C_eig"]]), nthreads=4)
    assert abs(f2 - float(d["E_eig"])) < 1e-12
    assert abs(f2 - (-7.023692395001888)) < 1e-10
    assert normwise(g2, d["g_eig"]) < 1e-11


def test_f0_edge():
    d = golden("f0_edge.npz")
    assert d["z_below"] < 16.3578 < d["z_above"]
    assert 16.3578 - d["z_below"] < 1e-6 and d["z_above"] - 16.3578 < 1e-6
    for tag in ("below", "above"):
        p = problem_from(d, iv=d[f"iv_{tag}"])
        o = Oracle.from_problem(p)
        m = np.array(o.matel(p.iv, 1, 2, 1))
        assert elem_rel(m[None], d[f"matel_{tag}"][None]).max() < TOL_ELEM
        tg, tgs = o.gradel(p.iv, 1, 2, 1)
        assert normwise(tg, d[f"tgvl_{tag}"]) < 1e-12 and normwise(tgs, d[f"tgvls_{tag}"]) < 1e-12
    # the two sides of the branch differ by the Pade / asymptotic jump
    assert abs(d["matel_below"][2] - d["matel_above"][2]) > 0


def test_threaded_equals_serial():
    d = golden("outprod_H2.npz")
    p = problem_from(d)
    o = Oracle.from_problem(p)
    f1, g1 = o.outprod(p.x, nthreads=1)
    f3, g3 = o.outprod(p.x, nthreads=3)
    assert abs(f1 - f3) < 1e-13 and normwise(g3, g1) < 1e-13


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_rrms(system):
    """rrms (python/rrms.py:21) on 400 terms, symmetry maps on both sides."""
    d = golden(f"rrms_{system}.npz")
    p = problem_from(d)
    o = Oracle.from_problem(p)
    out = np.array([o.rrms(p.iv, *t) for t in d["terms"]])
    assert rrms_rel(out, d["rrms"]).max() < TOL_ELEM


def test_driver_steps_oldquit():
    """The matrices, eigenpair and energetics of python/necg.py:main on
    oldquit.dat, and the dipole at the reference's L-BFGS-B optimum."""
    d = golden("driver_oldquit.npz")
    q = golden("oldquit.npz")
    p = problem_from(q)
    o = Oracle.from_problem(p)
    H, S, Kin, Pot = o.build_matrices(p.iv, nthreads=4)
    for got, ref in ((H, d["H0"]), (S, d["S0"]), (Kin, d["Kin0"]), (Pot, d["Pot0"])):
        assert np.max(np.abs(got - ref)) <= TOL_ELEM * np.max(np.abs(ref))
    K = p.K
    x = d["x_opt"]
    comps, dip = o.dipole(x[:K * p.blk], x[K * p.blk:], nthreads=4)
    assert np.max(np.abs(comps - d["dip_comps"])) < 1e-12
    assert np.max(np.abs(dip - d["dipole"])) < 1e-12
