"""Problem description and the oldquit.dat input format.

``Problem`` holds what the reference keeps in its ``shared`` module after
``read_input`` (python/shared.py:15-66, python/read_input.py:78-157):

* ``n``     particles in internal coordinates (``shared.ne``)
* ``K``     basis functions (``shared.M``)
* ``nst``   symmetry terms
* ``efs``   electric-field strength
* ``mass``  (n, n) inverse-mass tensor
* ``ncv``   (n+1,) charges, reference nucleus first
* ``scvv``  (nst,) symmetry weights ALREADY divided by nst (python/read_input.py:141)
* ``sml``   (nst, n, n) coordinate maps; ``sml[s]`` is ``shared.sml[:, :, s]``
* ``sms``   (nst, 3n, 3n) shift maps; ``sms[s]`` is ``shared.sms[:, :, s]``
* ``iv``    (K * blk,) packed [vech(L_k), s_k] blocks, blk = n(n+1)/2 + 3n
* ``C``     (K,) linear coefficients

The parser and writer follow the token layout of python/read_input.py:16-157
(whitespace separated, Fortran ``d`` exponents accepted).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Problem:
    n: int
    K: int
    efs: float
    mass: np.ndarray
    ncv: np.ndarray
    scvv: np.ndarray
    sml: np.ndarray
    sms: np.ndarray
    iv: np.ndarray
    C: np.ndarray
    name: str = ""

    @property
    def nst(self) -> int:
        return int(len(self.scvv))

    @property
    def svh(self) -> int:
        return self.n * (self.n + 1) // 2

    @property
    def skp(self) -> int:
        return 3 * self.n

    @property
    def blk(self) -> int:
        return self.svh + self.skp

    @property
    def siv(self) -> int:
        return self.K * self.blk

    @property
    def x(self) -> np.ndarray:
        """The optimiser vector [iv, C] (python/outprod.py:40-41)."""
        return np.concatenate([self.iv, self.C])

    @property
    def pairs(self) -> int:
        """Unordered (k, l) basis pairs, k >= l."""
        return self.K * (self.K + 1) // 2

    def copy(self) -> "Problem":
        return Problem(self.n, self.K, self.efs, self.mass.copy(), self.ncv.copy(), self.scvv.copy(),
                       self.sml.copy(), self.sms.copy(), self.iv.copy(), self.C.copy(), self.name)

    def validate(self) -> None:
        n, K, nst = self.n, self.K, self.nst
        if n < 1 or K < 1 or nst < 1:
            raise ValueError("n, K and nst must be positive")
        shapes = {"mass": (n, n), "ncv": (n + 1,), "scvv": (nst,), "sml": (nst, n, n),
                  "sms": (nst, 3 * n, 3 * n), "iv": (K * self.blk,), "C": (K,)}
        for k, shp in shapes.items():
            a = getattr(self, k)
            if a.shape != shp:
                raise ValueError(f"{k} has shape {a.shape}, expected {shp}")


def _tokens(filename: str):
    with open(filename, "r", encoding="utf-8") as fh:
        return fh.read().split()


def read_oldquit(filename: str) -> Problem:
    """Parse an oldquit.dat-format file (python/read_input.py:61-157)."""
    toks = _tokens(filename)
    pos = 0

    def nxt_i():
        nonlocal pos
        v = int(toks[pos])
        pos += 1
        return v

    def nxt_f(count=None):
        nonlocal pos
        if count is None:
            v = float(toks[pos].lower().replace("d", "e"))
            pos += 1
            return v
        vals = [float(t.lower().replace("d", "e")) for t in toks[pos:pos + count]]
        if len(vals) != count:
            raise ValueError(f"{filename}: truncated input (wanted {count} values at token {pos})")
        pos += count
        return np.array(vals, dtype=np.float64)

    K = nxt_i()
    n = nxt_i()
    nst = nxt_i()
    efs = nxt_f()
    svh, skp = n * (n + 1) // 2, 3 * n
    mass = nxt_f(n * n).reshape(n, n)
    ncv = nxt_f(n + 1)
    iv = nxt_f(K * (svh + skp))
    C = nxt_f(K)
    scvv = nxt_f(nst) / nst
    sml = nxt_f(nst * n * n).reshape(nst, n, n)
    sms = nxt_f(nst * skp * skp).reshape(nst, skp, skp)
    p = Problem(n, K, efs, mass, ncv, scvv, sml, sms, iv, C, name=filename)
    p.validate()
    return p


def _f(v: float) -> str:
    return repr(float(v))


def write_oldquit(p: Problem, filename: str) -> None:
    """Write ``p`` in the oldquit.dat token layout (python/read_input.py:20-53),
    with full round-trip precision."""
    lines = [str(p.K), str(p.n), str(p.nst), _f(p.efs), ""]
    for row in p.mass:
        lines.append(" ".join(_f(v) for v in row))
    lines.append("")
    lines += [_f(v) for v in p.ncv]
    lines.append("")
    for k in range(p.K):
        lines += ["   " + _f(v) for v in p.iv[k * p.blk:(k + 1) * p.blk]]
        lines.append("")
    lines += ["  " + _f(v) for v in p.C]
    lines.append("")
    lines += [_f(v) for v in p.scvv * p.nst]
    lines.append("")
    for s in range(p.nst):
        for row in p.sml[s]:
            lines.append(" ".join(_f(v) for v in row))
        lines.append("")
    for s in range(p.nst):
        for row in p.sms[s]:
            lines.append(" ".join(_f(v) for v in row))
        lines.append("")
    with open(filename, "w", encoding="utf-8") as fh:
        fh.write("\n".join(lines) + "\n")
