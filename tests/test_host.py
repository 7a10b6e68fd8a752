"""Host-side logic: input format, symmetry sets, synthetic workloads, vech."""
import os

import numpy as np
import pytest

from nbo_correlatedgaussians_b200 import shared as sh
from nbo_correlatedgaussians_b200 import synth
from nbo_correlatedgaussians_b200.problem import read_oldquit, write_oldquit
from nbo_correlatedgaussians_b200.read_input import read_input
from nbo_correlatedgaussians_b200.symmetry import inverse_map, mass_matrix, particles, symmetry_set
from nbo_correlatedgaussians_b200.utils import vech
from _util import golden, problem_from


def _as_set(sml, w):
    return sorted((tuple(np.round(m, 12).ravel()), float(x)) for m, x in zip(sml, w))


def test_lih_symmetry_matches_reference_file():
    d = golden("oldquit.npz")
    sml, sms, w = symmetry_set("LiH")
    assert _as_set(sml, w / len(w)) == _as_set(d["sml"], d["scvv"])
    for s in range(len(w)):
        assert np.array_equal(sms[s], np.kron(sml[s].T, np.eye(3)))


def test_lih_particles_match_reference_file():
    d = golden("oldquit.npz")
    n, M, ncv = particles("LiH")
    assert n == 5
    # oldquit.dat was written with m(Li) = 12786.3935 and m(p) = 1836.15267; the
    # synthetic workloads use 12786.39 and 1836.15, hence ~1e-6 relative
    np.testing.assert_allclose(M, d["mass"], rtol=2e-6)
    np.testing.assert_array_equal(ncv, d["ncv"])


@pytest.mark.parametrize("system,nst", [("He", 2), ("H2", 4), ("LiH", 24)])
def test_symmetry_sets_closed_under_inverse(system, nst):
    sml, sms, w = symmetry_set(system)
    assert len(sml) == nst
    inv = inverse_map(sml)
    assert (inv >= 0).all()
    np.testing.assert_array_equal(w[inv], w)
    for m in sml:
        assert abs(abs(np.linalg.det(m)) - 1.0) < 1e-12


@pytest.mark.parametrize("system", ["He", "H2", "LiH"])
def test_symmetry_sets_make_H_bra_ket_symmetric(system):
    """The reference's gradient (python/make_grad.py:61-79) assumes H_ij computed
    with bra i equals H_ji computed with bra j; a symmetry set whose shift maps
    do not match its coordinate maps breaks that.  Checked with the oracle."""
    from oracle.oracle import Oracle
    p = synth.make_problem(system, 5, 3)
    o = Oracle.from_problem(p)
    for i in range(2, 6):
        for j in range(1, i):
            a = sum(w * np.array(o.matel(p.iv, s + 1, i, j)) for s, w in enumerate(p.scvv))
            b = sum(w * np.array(o.matel(p.iv, s + 1, j, i)) for s, w in enumerate(p.scvv))
            assert abs(a[0] - b[0]) < 1e-12 * abs(a[0])
            ha, hb = a[1] + a[2] - a[3], b[1] + b[2] - b[3]
            assert abs(ha - hb) < 1e-11 * abs(ha)


def test_shift_maps_are_inverse_coordinate_maps():
    for system in ("He", "H2", "LiH"):
        sml, sms, _ = symmetry_set(system)
        for P, Sm in zip(sml, sms):
            np.testing.assert_allclose(Sm, np.kron(np.linalg.inv(P), np.eye(3)), atol=1e-15)


def test_h2_proton_swap_is_involution():
    sml, _, _ = symmetry_set("H2")
    for m in sml:
        np.testing.assert_allclose(m @ m, np.eye(3), atol=1e-15)


def test_mass_matrix_convention():
    M = mass_matrix(10.0, [2.0, 1.0])
    np.testing.assert_allclose(M, [[0.5 / 2 + 0.05, 0.05], [0.05, 0.5 + 0.05]])


def test_oldquit_roundtrip(tmp_path):
    p = problem_from(golden("oldquit.npz"))
    f = tmp_path / "rt.dat"
    write_oldquit(p, str(f))
    q = read_oldquit(str(f))
    assert (q.n, q.K, q.nst) == (p.n, p.K, p.nst) and q.efs == p.efs
    for k in ("mass", "ncv", "scvv", "sml", "sms", "iv", "C"):
        np.testing.assert_array_equal(getattr(q, k), getattr(p, k), err_msg=k)


def test_read_input_populates_shared_like_reference(tmp_path):
    d = golden("oldquit.npz")
    p = problem_from(d)
    f = tmp_path / "oldquit.dat"
    write_oldquit(p, str(f))
    read_input(str(f))
    assert (sh.M, sh.ne, sh.nst, sh.svh, sh.skp, sh.siv) == (12, 5, 24, 15, 15, 360)
    assert sh.sml.shape == (5, 5, 24) and sh.sms.shape == (15, 15, 24)
    np.testing.assert_array_equal(sh.sml[:, :, 3], d["sml"][3])
    np.testing.assert_array_equal(sh.sms[:, :, 7], d["sms"][7])
    np.testing.assert_array_equal(sh.iv, d["iv"])
    np.testing.assert_allclose(sh.scvv * sh.nst, d["scvv"] * 24)


def test_read_input_fortran_exponent_and_missing_file(tmp_path):
    p = synth.make_problem("He", 3, 0)
    f = tmp_path / "in.dat"
    write_oldquit(p, str(f))
    txt = f.read_text().replace("e-", "d-")
    f.write_text(txt)
    q = read_oldquit(str(f))
    np.testing.assert_allclose(q.iv, p.iv, rtol=0, atol=0)
    with pytest.raises(OSError):
        read_input(str(tmp_path / "absent.dat"))
    g = tmp_path / "short.dat"
    g.write_text("\n".join(f.read_text().split("\n")[:20]))
    with pytest.raises(ValueError):
        read_oldquit(str(g))


def test_vech_column_major():
    A = np.arange(16.0).reshape(4, 4)
    expect = [A[i, j] for j in range(4) for i in range(j, 4)]
    np.testing.assert_array_equal(vech(A, 4), expect)


@pytest.mark.parametrize("system,lo,hi", [("LiH", 0.2, 3.0), ("H2", 0.1, 4.0), ("He", 0.1, 4.0)])
def test_synthetic_distributions(system, lo, hi):
    p = synth.make_problem(system, 300, 1)
    p.validate()
    blocks = p.iv.reshape(p.K, p.blk)
    diag = [j * p.n - j * (j - 1) // 2 for j in range(p.n)]
    d = blocks[:, diag]
    assert d.min() >= lo and d.max() <= hi
    off = np.delete(blocks[:, :p.svh], diag, axis=1)
    assert abs(off.std() - 0.3) < 0.03
    assert abs(blocks[:, p.svh:].std() - 0.05) < 0.005
    np.testing.assert_array_equal(p.C, np.full(300, 1.0 / 300))
    q = synth.make_problem(system, 300, 1)
    np.testing.assert_array_equal(p.iv, q.iv)


def test_named_workloads():
    assert synth.workload("lih_k12").K == 12
    mixed = synth.workload("mixed64")
    assert len(mixed) == 64
    assert sum(p.n == 2 for p in mixed) == 16 and sum(p.n == 5 for p in mixed) == 24
    assert all(32 <= p.K <= 512 for p in mixed if p.n == 2)
    assert all(64 <= p.K <= 1024 for p in mixed if p.n != 2)
