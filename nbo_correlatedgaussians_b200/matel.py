"""Drop-in ``matel(stf, ii, jj)`` (python/matel.py:28-210): overlap, kinetic,
Coulomb and Stark elements of one (bra ii, symmetry stf on ket jj) term,
1-based, computed by the CUDA library from the parameters in ``shared``."""
from __future__ import annotations

from . import _state
from . import shared as sh


def matel(stf: int, ii: int, jj: int) -> tuple[float, float, float, float]:
    out = _state.engine().matel(sh.iv, [(stf, ii, jj)], K=sh.M)[0]
    return float(out[0]), float(out[1]), float(out[2]), float(out[3])


def matel_batch(terms):
    """Vectorised form: (nterms, 4) array for 1-based (stf, ii, jj) rows."""
    return _state.engine().matel(sh.iv, terms, K=sh.M)
