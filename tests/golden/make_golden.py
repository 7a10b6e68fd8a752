"""Generate the golden fixtures in this directory by executing the reference
Python package (MauricioCafiero/NBO_CorrelatedGaussians, python/).

Run in a checkout where the reference is available:
    NECG_REF=/path/to/NBO_CorrelatedGaussians python tests/golden/make_golden.py

Fixtures (npz, all FP64):
  oldquit.npz     the reference's own LiH input (K=12, n=5, nst=24): problem
                  arrays, E and g of outprod at the file's C, H and S, and the
                  lowest eigenpair of (H, S) with E at that C.
  elements_<sys>.npz  for He, H2, LiH (K=6 synthetic bases): 400 random
                  (stf, ii, jj) terms incl. ii == jj with matel outputs and
                  gradel outputs.
  outprod_<sys>.npz   outprod (E, g, H, S) on small synthetic bases.
  f0.npz          f0 / df0 at z on both sides of the 16.3578 branch point and near 0.
  f0_edge.npz     a He problem whose Coulomb argument z sits within 1e-6 of the
                  branch point, with matel / gradel outputs.
  rrms_<sys>.npz  for He, H2, LiH (K=6): 400 random (stfe, stf, ii, jj, n1)
                  terms with the rrms outputs (ov, tk).
  driver_oldquit.npz  the steps of python/necg.py:main on oldquit.dat: the
                  initial H, S, Kinetic, Potential, lowest eigenpair and
                  energetics, the L-BFGS-B result (20 iterations, main's
                  options), the energetics at the optimum and the dipole
                  components.
  driver_tnc_oldquit.npz  the same start point optimised with SciPy's TNC
                  (truncated Newton) for at most 50 iterations through the
                  reference's outprod: iterate count, final E and x.
Select generators by name on the command line (default: all).
The reference is imported only by this script; the tests read the npz files.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
REF = os.environ.get("NECG_REF")
if not REF:
    sys.exit("set NECG_REF to a checkout of MauricioCafiero/NBO_CorrelatedGaussians")
sys.path.insert(0, os.path.join(REF, "python"))

import shared as sh  # noqa: E402  (reference module)
from gradel import gradel  # noqa: E402
from matel import matel  # noqa: E402
from outprod import outprod  # noqa: E402
from rrms import rrms  # noqa: E402
from read_input import read_input  # noqa: E402
from utils import df0, f0  # noqa: E402
from scipy import linalg  # noqa: E402

from nbo_correlatedgaussians_b200 import synth  # noqa: E402
from nbo_correlatedgaussians_b200.problem import Problem  # noqa: E402


def load_into_reference(p: Problem) -> None:
    """Set the reference's shared state from a Problem (same as its read_input)."""
    sh.M, sh.ne, sh.nst, sh.efs = p.K, p.n, p.nst, p.efs
    sh.skp, sh.svh = 3 * p.n, p.n * (p.n + 1) // 2
    sh.siv = sh.M * (sh.svh + sh.skp)
    sh.mass = p.mass.copy()
    sh.ncv = p.ncv.copy()
    sh.iv = p.iv.copy()
    sh.C = p.C.copy()
    sh.scvv = p.scvv.copy()
    sh.sml = np.ascontiguousarray(np.transpose(p.sml, (1, 2, 0)))
    sh.sms = np.ascontiguousarray(np.transpose(p.sms, (1, 2, 0)))
    for name in ("H", "S", "Kinetic", "Potential", "ki", "po", "hh", "ss"):
        setattr(sh, name, np.zeros((sh.M, sh.M)))
    sh.grad = np.zeros(sh.siv + sh.M)


def problem_arrays(p: Problem) -> dict:
    return dict(n=p.n, K=p.K, efs=p.efs, mass=p.mass, ncv=p.ncv, scvv=p.scvv, sml=p.sml, sms=p.sms,
                iv=p.iv, C=p.C)


def build_hs():
    H = np.zeros((sh.M, sh.M))
    S = np.zeros((sh.M, sh.M))
    for i in range(1, sh.M + 1):
        for j in range(1, i + 1):
            for stf in range(1, sh.nst + 1):
                ov, tk, ert, zht = matel(stf, i, j)
                H[i - 1, j - 1] += sh.scvv[stf - 1] * (tk + ert - zht)
                S[i - 1, j - 1] += sh.scvv[stf - 1] * ov
    H = np.tril(H) + np.tril(H, -1).T
    S = np.tril(S) + np.tril(S, -1).T
    return H, S


def gen_oldquit():
    read_input(os.path.join(REF, "oldquit.dat"))
    p = Problem(sh.ne, sh.M, sh.efs, sh.mass.copy(), sh.ncv.copy(), sh.scvv.copy(),
                np.ascontiguousarray(np.transpose(sh.sml, (2, 0, 1))),
                np.ascontiguousarray(np.transpose(sh.sms, (2, 0, 1))), sh.iv.copy(), sh.C.copy())
    x = np.concatenate([sh.iv, sh.C])
    E, g = outprod(x)
    H, S = sh.H.copy(), sh.S.copy()
    ev, evec = linalg.eigh(H, S)
    C0 = evec[:, 0].copy()
    x2 = np.concatenate([p.iv, C0])
    E2, g2 = outprod(x2)
    np.savez(os.path.join(HERE, "oldquit.npz"), E=E, g=g, H=H, S=S, eig0=ev[0], C_eig=C0, E_eig=E2,
             g_eig=g2, **problem_arrays(p))
    print("oldquit: E", E, "E_eig", E2)


def gen_elements(system: str, K: int = 6, nterms: int = 400, seed: int = 11):
    p = synth.make_problem(system, K, seed)
    load_into_reference(p)
    rng = np.random.default_rng(seed)
    terms = np.stack([rng.integers(1, p.nst + 1, nterms), rng.integers(1, K + 1, nterms),
                      rng.integers(1, K + 1, nterms)], axis=1).astype(np.int32)
    terms[:40, 2] = terms[:40, 1]  # diagonal terms (ii == jj)
    mat = np.array([matel(*map(int, t)) for t in terms])
    gr = [gradel(*map(int, t)) for t in terms]
    np.savez(os.path.join(HERE, f"elements_{system}.npz"), terms=terms, matel=mat,
             tgvl=np.stack([a for a, _ in gr]), tgvls=np.stack([b for _, b in gr]), **problem_arrays(p))
    print("elements", system, mat.shape)


def gen_outprod(system: str, K: int, seed: int):
    p = synth.make_problem(system, K, seed)
    load_into_reference(p)
    E, g = outprod(p.x)
    np.savez(os.path.join(HERE, f"outprod_{system}.npz"), E=E, g=g, H=sh.H.copy(), S=sh.S.copy(),
             **problem_arrays(p))
    print("outprod", system, K, E)


def gen_f0():
    zs = [0.0, 1e-300, 1e-12, 1e-6, 0.01, 0.5, 1.0, 3.0, 7.5, 12.0, 16.0, 16.3578 - 1e-6, 16.3578,
          16.3578 + 1e-6, 16.36, 20.0, 50.0, 1e3, 1e6]
    z = np.array(zs)
    np.savez(os.path.join(HERE, "f0.npz"), z=z, f0=np.array([f0(v) for v in z]),
             df0=np.array([df0(v) for v in z]))


def gen_f0_edge():
    """He, K=2: scale the shift of basis 2 until the nucleus-electron-1 Coulomb
    argument of term (stf=1, 2, 1) lands within 1e-6 of the Pade branch point,
    then record a term just below and one just above it."""
    base = synth.make_problem("He", 2, 5)
    base.iv[0 * base.blk:0 * base.blk + base.svh] = [1.0, 0.1, 0.9]
    base.iv[1 * base.blk:1 * base.blk + base.svh] = [1.1, -0.2, 1.0]

    def z_of(lam):
        p = base.copy()
        p.iv[base.blk + base.svh:2 * base.blk] = lam * np.array([0.0, 0.0, 1.0, 0.0, 0.0, 0.3])
        p.iv[base.svh:base.blk] = 0.0
        n = p.n
        L1 = np.array([[1.0, 0.0], [0.1, 0.9]])
        L2 = np.array([[1.1, 0.0], [-0.2, 1.0]])
        A1, A2 = L1 @ L1.T, L2 @ L2.T
        Bi = np.linalg.inv(A1 + A2)
        s2 = p.iv[base.blk + base.svh:2 * base.blk].reshape(n, 3)
        T = Bi @ (A2 @ s2)
        return T[0] @ T[0] / Bi[0, 0], p

    lo, hi = 0.0, 1.0
    while z_of(hi)[0] < 16.3578:
        hi *= 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if z_of(mid)[0] < 16.3578:
            lo = mid
        else:
            hi = mid
    out = {}
    for tag, lam in (("below", lo * (1 - 2e-8)), ("above", hi * (1 + 2e-8))):
        z, p = z_of(lam)
        load_into_reference(p)
        out[f"z_{tag}"] = z
        out[f"iv_{tag}"] = p.iv.copy()
        out[f"matel_{tag}"] = np.array(matel(1, 2, 1))
        tg, tgs = gradel(1, 2, 1)
        out[f"tgvl_{tag}"] = tg
        out[f"tgvls_{tag}"] = tgs
    np.savez(os.path.join(HERE, "f0_edge.npz"), **{k: v for k, v in problem_arrays(base).items() if k != "iv"},
             **out)
    print("f0 edge z", out["z_below"], out["z_above"])


def gen_rrms(system: str, K: int = 6, nterms: int = 400, seed: int = 13):
    p = synth.make_problem(system, K, seed)
    load_into_reference(p)
    rng = np.random.default_rng(seed)
    terms = np.stack([rng.integers(1, p.nst + 1, nterms), rng.integers(1, p.nst + 1, nterms),
                      rng.integers(1, K + 1, nterms), rng.integers(1, K + 1, nterms),
                      rng.integers(1, 3 * p.n + 1, nterms)], 1).astype(np.int32)
    terms[:20, 3] = terms[:20, 2]  # diagonal pairs
    out = np.array([rrms(*map(int, t)) for t in terms])
    np.savez(os.path.join(HERE, f"rrms_{system}.npz"), terms=terms, rrms=out, **problem_arrays(p))
    print("rrms", system, out[:2])


def _energetics():
    cHc, cSc = sh.C @ sh.H @ sh.C, sh.C @ sh.S @ sh.C
    cKc, cPc = sh.C @ sh.Kinetic @ sh.C, sh.C @ sh.Potential @ sh.C
    return np.array([cHc / cSc, cKc / cSc, cPc / cSc, -2.0 * cKc / cPc])


def gen_driver(maxiter: int = 20):
    """python/necg.py:main on oldquit.dat, step by step, through the reference's
    own functions (its _build_matrices, scipy's eigh and L-BFGS-B with main's
    options, its rrms)."""
    import necg as ref_necg  # noqa: E402  (reference module)
    from scipy.optimize import minimize
    read_input(os.path.join(REF, "oldquit.dat"))
    ref_necg._build_matrices()
    H0, S0, K0, P0 = sh.H.copy(), sh.S.copy(), sh.Kinetic.copy(), sh.Potential.copy()
    ev, evec = linalg.eigh(sh.H, sh.S)
    sh.C[:] = evec[:, 0]
    C0 = sh.C.copy()
    en0 = _energetics()
    hiv = np.concatenate([sh.iv.copy(), sh.C.copy()])
    fvals = []

    def fun(x):
        f, g = outprod(x)
        fvals.append(f)
        return f, g

    eps = 2.220446649250313e-16
    res = minimize(fun, hiv, method="L-BFGS-B", jac=True,
                   options={"maxiter": maxiter, "maxfun": 150 * (sh.siv + sh.M), "ftol": eps,
                            "gtol": np.sqrt(eps)})
    sh.iv[:] = res.x[:sh.siv]
    sh.C[:] = res.x[sh.siv:]
    ref_necg._build_matrices()
    en1 = _energetics()
    # dipole: the loop of python/necg.py:200-244 over its rrms
    M, nst = sh.M, sh.nst
    dip = np.zeros(3)
    den = None
    comps = np.zeros(3 * sh.ne)
    for kk in range(1, 3 * sh.ne + 1):
        hd = np.zeros((M, M))
        sd = np.zeros((M, M))
        for stfe in range(1, nst + 1):
            for stf in range(1, nst + 1):
                w = sh.scvv[stf - 1] * sh.scvv[stfe - 1]
                for i in range(1, M + 1):
                    for j in range(i, M + 1):
                        ov_r, tk_r = rrms(stfe, stf, j, i, kk)
                        hd[j - 1, i - 1] += w * tk_r
                        sd[j - 1, i - 1] += w * ov_r
        hd = np.tril(hd) + np.tril(hd, -1).T
        sd = np.tril(sd) + np.tril(sd, -1).T
        den = sh.C @ sd @ sh.C
        comps[kk - 1] = (sh.C @ hd @ sh.C) / den if den != 0.0 else 0.0
        dip[(kk - 1) % 3] += sh.ncv[(kk - 1) // 3 + 1] * comps[kk - 1]
    np.savez(os.path.join(HERE, "driver_oldquit.npz"), H0=H0, S0=S0, Kin0=K0, Pot0=P0, eig0=ev[0], C0=C0,
             en0=en0, x_opt=res.x, f_opt=res.fun, nit=res.nit, nfev=res.nfev, fvals=np.array(fvals),
             en1=en1, dip_comps=comps, dipole=dip, maxiter=maxiter)
    print("driver: eig0", ev[0], "en0", en0, "f_opt", res.fun, "nit", res.nit, "en1", en1, "dipole", dip)


class _Cap(Exception):
    pass


def gen_driver_tnc(maxiter: int = 50):
    from scipy.optimize import minimize
    d = np.load(os.path.join(HERE, "driver_oldquit.npz"))
    read_input(os.path.join(REF, "oldquit.dat"))
    x0 = np.concatenate([sh.iv.copy(), d["C0"]])
    last = {"x": x0.copy(), "it": 0}

    def cb(xk):
        last["x"] = np.array(xk)
        last["it"] += 1
        if last["it"] >= maxiter:
            raise _Cap

    try:
        r = minimize(outprod, x0, method="TNC", jac=True, callback=cb, options={"maxfun": 1000 * maxiter})
        x, f, nit = r.x, float(r.fun), int(r.nit)
    except _Cap:
        x, nit = last["x"], last["it"]
        f = float(outprod(x)[0])
    np.savez(os.path.join(HERE, "driver_tnc_oldquit.npz"), x_opt=x, f_opt=f, nit=nit, maxiter=maxiter)
    print("driver TNC: f", f, "nit", nit)


if __name__ == "__main__":
    want = set(sys.argv[1:]) or {"f0", "f0_edge", "oldquit", "elements", "outprod", "rrms", "driver",
                                 "driver_tnc"}
    if "f0" in want:
        gen_f0()
    if "f0_edge" in want:
        gen_f0_edge()
    if "oldquit" in want:
        gen_oldquit()
    if "elements" in want:
        for system in ("He", "H2", "LiH"):
            gen_elements(system)
    if "outprod" in want:
        gen_outprod("He", 16, 21)
        gen_outprod("H2", 12, 22)
        gen_outprod("LiH", 6, 23)
    if "rrms" in want:
        for system in ("He", "H2", "LiH"):
            gen_rrms(system)
    if "driver" in want:
        gen_driver()
    if "driver_tnc" in want:
        gen_driver_tnc()
