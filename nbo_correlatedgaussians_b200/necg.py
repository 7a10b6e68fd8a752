"""Drop-in driver with the flow of python/necg.py:main (itself the analogue of
source/necg.f90): read the input, build H, S, Kinetic and Potential, solve the
generalised eigenproblem for the initial C, minimise E over x = [iv, C] with
L-BFGS-B on ``outprod``, rebuild at the optimum and compute the dipole.

Everything after ``read_input`` stays on the GPU except the optimiser itself
(SciPy, as in the reference): the matrix build and the dipole run in the CUDA
library, and the eigenproblem H v = lambda S v is solved on the device
(Cholesky of S, then the symmetric eigenproblem of L^-1 H L^-T) instead of
scipy.linalg.eigh on the host (python/necg.py:129-134).

Usage:  python -m nbo_correlatedgaussians_b200.necg [input_file]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np
import torch
from scipy.optimize import minimize

from . import _state
from . import shared as sh
from .outprod import outprod
from .read_input import read_input
from .utils import biout, get_current_time

DEBYE = 2.541765e0  # python/necg.py:235


def _build_matrices() -> None:
    """H, S, Kinetic, Potential from the current iv into ``shared``
    (python/necg.py:36-58), built by the energy tiles on the device."""
    eng = _state.engine()
    H, S, Kin, Pot, _ = eng.build_matrices(sh.iv, K=sh.M, parts=True)
    sh.H, sh.S = H.cpu().numpy(), S.cpu().numpy()
    sh.Kinetic, sh.Potential = Kin.cpu().numpy(), Pot.cpu().numpy()


def _rayleigh_quotient() -> tuple[float, float, float, float]:
    """(energy, kinetic, potential, virial) at the current C (python/necg.py:61-71)."""
    C = sh.C
    cHc, cSc = float(C @ sh.H @ C), float(C @ sh.S @ C)
    cKc, cPc = float(C @ sh.Kinetic @ C), float(C @ sh.Potential @ C)
    return cHc / cSc, cKc / cSc, cPc / cSc, -2.0 * (cKc / cSc) / (cPc / cSc)


def _print_energetics(energy: float, kin: float, pot: float, virial: float) -> None:
    print("*" * 69)
    print()
    print(f"Rayleigh Quotient: {energy:25.15f}")
    print()
    print(f"Average Kinetic  : {kin:25.15f}")
    print()
    print(f"Average Potential: {pot:25.15f}")
    print()
    print(f"Virial Coef.     : {virial:25.15f}")
    print()
    print("*" * 69)


def generalized_eigh(H, S, device=None) -> tuple[np.ndarray, np.ndarray]:
    """All eigenpairs of H v = lambda S v on the GPU, eigenvalues ascending and
    eigenvectors S-orthonormal (the output of scipy.linalg.eigh(H, S) /
    LAPACK DSYGV, up to the sign of each vector).  Raises
    numpy.linalg.LinAlgError if S is not positive definite."""
    dev = device or _state.engine().device
    Ht = torch.as_tensor(np.asarray(H), dtype=torch.float64, device=dev)
    St = torch.as_tensor(np.asarray(S), dtype=torch.float64, device=dev)
    Lc, info = torch.linalg.cholesky_ex(St)
    if int(info.item()) != 0:
        raise np.linalg.LinAlgError("S is not positive definite")
    A = torch.linalg.solve_triangular(Lc, Ht, upper=False)            # L^-1 H
    A = torch.linalg.solve_triangular(Lc, A.T.contiguous(), upper=False)  # L^-1 (L^-1 H)^T
    A = 0.5 * (A + A.T)
    w, V = torch.linalg.eigh(A)
    X = torch.linalg.solve_triangular(Lc.T.contiguous(), V, upper=True)  # L^-T V
    return w.cpu().numpy(), X.cpu().numpy()


def dipole() -> tuple[np.ndarray, np.ndarray]:
    """(components, dipole) at the current iv, C: the 3n component expectation
    values and (d_x, d_y, d_z) in atomic units (python/necg.py:200-244)."""
    return _state.engine().dipole(sh.iv, sh.C)


class _IterationCap(Exception):
    pass


def optimise(fun, x0: np.ndarray, method: str = "L-BFGS-B", maxiter: int = 20, nvar: int | None = None,
             hessp=None):
    """Minimise fun (returning (f, g)) from x0.  L-BFGS-B with the options of
    python/necg.py:159-171; "TNC" (SciPy's truncated Newton, the analogue of
    the Fortran driver's LMQN, source/tn.f) stopped after ``maxiter``
    iterations; or "Newton-CG" with ``hessp(x, v)`` (the Hessian-vector product
    of the truncated-Newton inner loop, source/tn.f:1301-1327).  Returns (x, f,
    nit, message)."""
    eps = 2.220446649250313e-16
    nvar = nvar or x0.size
    if method == "L-BFGS-B":
        r = minimize(fun, x0, method="L-BFGS-B", jac=True,
                     options={"maxiter": maxiter, "maxfun": 150 * nvar, "ftol": eps, "gtol": np.sqrt(eps)})
        return r.x, float(r.fun), int(r.nit), str(r.message)
    if method == "Newton-CG":
        if hessp is None:
            raise ValueError("Newton-CG needs hessp")
        r = minimize(fun, x0, method="Newton-CG", jac=True, hessp=hessp, options={"maxiter": maxiter})
        return r.x, float(r.fun), int(r.nit), str(r.message)
    if method != "TNC":
        raise ValueError(f"unknown method {method!r}")
    last = {"x": x0.copy(), "it": 0}

    def cb(xk):  # TNC has no iteration limit of its own
        last["x"] = np.array(xk, dtype=np.float64)
        last["it"] += 1
        if last["it"] >= maxiter:
            raise _IterationCap

    try:
        r = minimize(fun, x0, method="TNC", jac=True, callback=cb, options={"maxfun": 1000 * maxiter})
        return r.x, float(r.fun), int(r.nit), str(r.message)
    except _IterationCap:
        f, _ = fun(last["x"])
        return last["x"], float(f), last["it"], f"stopped after {maxiter} iterations"


def write_restart(filename: str) -> None:
    """The current basis (iv, C) and problem in the oldquit.dat layout, so a run
    can resume from it (the restart writer of the Fortran driver,
    source/btn.f:335-363, kept there as a comment)."""
    from .problem import write_oldquit
    write_oldquit(_state.problem_from_shared(), filename)


def main(input_file: str = "oldquit.dat", maxiter: int = 20, output: str | None = None,
         method: str = "L-BFGS-B", restart: str | None = None) -> dict:
    """Run the driver; returns the quantities it prints (for tests and callers).
    method "L-BFGS-B" is python/necg.py's optimiser; "TNC" runs ``maxiter``
    truncated-Newton iterations instead; "Newton-CG" uses Hessian-vector
    products from two gradients evaluated in one batched step.  ``restart``:
    write the optimised basis there in the oldquit.dat layout."""
    if output is None:
        output = "necg.out"
    from . import utils
    utils._OUTPUT_FILE = output
    if os.path.exists(output):
        os.remove(output)
    biout("N-particle Non-Born-Oppenheimer Correlated Gaussians")
    biout("=" * 68)
    biout(":PROGRAM BEGINS:")
    td, tt, tz = get_current_time()
    biout(f"Date: {td} | Time: {tt} / {tz} gmt")

    read_input(input_file)
    print(f"M, NE, NST = {sh.M}, {sh.ne}, {sh.nst}")
    print(f"Electric Field = {sh.efs}")
    print(f"OUTPUT FILENAME = {output}")
    res: dict = {}

    t0 = time.perf_counter()
    _build_matrices()
    res["t_matrices"] = time.perf_counter() - t0
    print(f"Time for matrix calc. is {res['t_matrices']:.3f} seconds")

    try:
        w, X = generalized_eigh(sh.H, sh.S)
        print(f"Eigenvalue = {w[0]:.15f}")
        sh.C[:] = X[:, 0]
        res["eig0"] = float(w[0])
    except np.linalg.LinAlgError as exc:
        print(f"Warning: generalised eigenvalue problem failed: {exc}")
        res["eig0"] = None
    res["C0"] = sh.C.copy()
    print()
    print("***** The Input Vectors *****")
    print(sh.C)
    print("***** End Input Vectors *****")
    print()
    res["en0"] = _rayleigh_quotient()
    _print_energetics(*res["en0"])

    hiv = np.concatenate([sh.iv.copy(), sh.C.copy()])
    fvals = []

    def fun(x):
        f, g = outprod(x)
        fvals.append(f)
        return f, g

    hv = None
    if method == "Newton-CG":
        from .hessian import HessianVector
        hv = HessianVector(_state.problem_from_shared())
    t0 = time.perf_counter()
    x_opt, f_opt, nit, message = optimise(fun, hiv, method, maxiter, sh.siv + sh.M,
                                          hessp=(lambda x, v: hv(x, v)) if hv else None)
    if hv is not None:
        res["hessp_calls"] = hv.count
        hv.close()
    res["t_optimise"] = time.perf_counter() - t0
    print(f"Time for energy/gradient calc. is {res['t_optimise']:.3f} seconds")
    print(f"Energy is {f_opt:.15f} hartree")
    print(f"Optimiser message: {message}")
    res.update(f_opt=f_opt, x_opt=x_opt.copy(), nit=nit, nfev=len(fvals), fvals=np.array(fvals))

    sh.iv[:] = x_opt[:sh.siv]
    sh.C[:] = x_opt[sh.siv:]
    print()
    print("***** The Output Vectors *****")
    print(sh.C)
    print()
    print("***** End Output Vectors *****")
    print()
    if restart:
        write_restart(restart)
    _build_matrices()
    res["en1"] = _rayleigh_quotient()
    _print_energetics(*res["en1"])

    t0 = time.perf_counter()
    comps, dip = dipole()
    res["t_dipole"] = time.perf_counter() - t0
    res["dip_comps"], res["dipole"] = comps, dip
    print()
    for name, d in zip("xyz", dip):
        print(f"Dipole {name}-component = {d:.15f}  ( {d * DEBYE:.6f} Debye )")
        print()
    print("*" * 69)
    biout("PROGRAM TERMINATES")
    td, tt, tz = get_current_time()
    biout(f"Date: {td} | Time: {tt} / {tz} gmt")
    return res


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "oldquit.dat")
