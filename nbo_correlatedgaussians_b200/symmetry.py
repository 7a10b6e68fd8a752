"""Particle sets and symmetry-projector sets for the three systems the engine
is exercised on (He, H2, LiH in non-Born-Oppenheimer internal coordinates).

A symmetry term is a coordinate map ``sml`` (n x n, acting on the internal
coordinates of the ket, python/matel.py:76-77), its shift map ``sms``
(python/matel.py:87) and a weight ``scvv``.  The reference's Gaussians are
centred, exp(-(r - s)^T (A x I3) (r - s)) (python/matel.py:125-136), so
evaluating one at P r moves A to P^T A P and the centre s to P^-1 s: the shift
map is kron(P^-1, I3).  For the permutations of oldquit.dat P^-1 = P^T, which
is the kron(sml^T, I3) stored there.  The
reference reads these from the input file (python/read_input.py:139-157) and
ships them only for LiH (``oldquit.dat``); the He and H2 sets here are built
the same way.

LiH: the 24 = 4! permutations of the four electrons (internal particles 2..5,
particle 1 is the proton, the Li nucleus is the reference).  The weights are
the coefficients of Y Y^dagger for the Young operator Y = A S of the [2,2]
tableau with rows {e1, e2}, {e3, e4}: S symmetrises the rows, A antisymmetrises
the columns {e1, e3}, {e2, e4}.  This reproduces the weights stored in the
reference's oldquit.dat (16, 8, -8, -16) term for term.
He: identity and the electron swap, weights +1 (spatially symmetric singlet).
H2: identity, electron swap, proton swap and both, weights +1.  With the first
proton as the reference, swapping the protons maps internal coordinates
(r_p, r_e1, r_e2) to (-r_p, r_e1 - r_p, r_e2 - r_p).
"""
from __future__ import annotations

import itertools

import numpy as np

# masses in electron masses, charges in e
M_PROTON = 1836.15
M_LI7 = 12786.39
M_HE4 = 7294.30

SYSTEMS = {
    # name: (reference-nucleus mass, reference-nucleus charge, [(mass, charge), ...])
    "He": (M_HE4, 2.0, [(1.0, -1.0), (1.0, -1.0)]),
    "H2": (M_PROTON, 1.0, [(M_PROTON, 1.0), (1.0, -1.0), (1.0, -1.0)]),
    "LiH": (M_LI7, 3.0, [(M_PROTON, 1.0)] + [(1.0, -1.0)] * 4),
}


def mass_matrix(m0: float, masses) -> np.ndarray:
    """mass_ij = (delta_ij / m_i + 1 / m_0) / 2, the convention of oldquit.dat."""
    n = len(masses)
    M = np.full((n, n), 0.5 / m0)
    for i, m in enumerate(masses):
        M[i, i] += 0.5 / m
    return M


def _sms_from_sml(sml: np.ndarray) -> np.ndarray:
    """Shift maps kron(P^-1, I3) of the coordinate maps P (see the module doc)."""
    return np.stack([np.kron(np.linalg.inv(p), np.eye(3)) for p in sml])


def _perm_matrix(n: int, perm) -> np.ndarray:
    """Row i of the map has a one in column perm[i]."""
    P = np.zeros((n, n))
    for i, j in enumerate(perm):
        P[i, j] = 1.0
    return P


def _young_22_weights():
    """Group-algebra coefficients of Y Y^dagger for Y = A S on S4, tableau rows
    {0,1},{2,3}, columns {0,2},{1,3}.  Returns {perm tuple: integer weight}."""
    e = (0, 1, 2, 3)

    def comp(a, b):
        return tuple(a[b[i]] for i in range(4))

    def inv(a):
        r = [0] * 4
        for i, x in enumerate(a):
            r[x] = i
        return tuple(r)

    def tr(i, j):
        p = list(e)
        p[i], p[j] = p[j], p[i]
        return tuple(p)

    def mul(X, Y):
        Z = {}
        for a, ca in X.items():
            for b, cb in Y.items():
                c = comp(a, b)
                Z[c] = Z.get(c, 0) + ca * cb
        return Z

    S = mul({e: 1, tr(0, 1): 1}, {e: 1, tr(2, 3): 1})
    A = mul({e: 1, tr(0, 2): -1}, {e: 1, tr(1, 3): -1})
    Y = mul(A, S)
    Yd = {inv(k): v for k, v in Y.items()}
    return {k: v for k, v in mul(Y, Yd).items() if v != 0}


def symmetry_set(system: str):
    """Return (sml (nst,n,n), sms (nst,3n,3n), weights (nst,)) with the raw
    (undivided) weights as they appear in an input file."""
    if system == "He":
        sml = np.stack([_perm_matrix(2, (0, 1)), _perm_matrix(2, (1, 0))])
        w = np.array([1.0, 1.0])
    elif system == "H2":
        I = np.eye(3)
        E = _perm_matrix(3, (0, 2, 1))
        Pp = np.array([[-1.0, 0, 0], [-1.0, 1.0, 0], [-1.0, 0, 1.0]])
        sml = np.stack([I, E, Pp, Pp @ E])
        w = np.ones(4)
    elif system == "LiH":
        coef = _young_22_weights()
        mats, ws = [], []
        for perm in itertools.permutations(range(4)):
            mats.append(_perm_matrix(5, (0,) + tuple(p + 1 for p in perm)))
            ws.append(float(coef.get(perm, 0)))
        sml = np.stack(mats)
        w = np.array(ws)
    else:
        raise ValueError(f"unknown system {system!r}")
    return sml, _sms_from_sml(sml), w


def particles(system: str):
    """Return (n, mass matrix, ncv) for a system."""
    m0, q0, parts = SYSTEMS[system]
    masses = [m for m, _ in parts]
    ncv = np.array([q0] + [q for _, q in parts])
    return len(parts), mass_matrix(m0, masses), ncv


def inverse_map(sml: np.ndarray, atol: float = 1e-12) -> np.ndarray:
    """Index of the inverse of each symmetry map within the set, -1 if absent."""
    out = np.full(len(sml), -1, dtype=np.int64)
    for a, P in enumerate(sml):
        Pi = np.linalg.inv(P)
        for b, Q in enumerate(sml):
            if np.allclose(Pi, Q, atol=atol):
                out[a] = b
                break
    return out
