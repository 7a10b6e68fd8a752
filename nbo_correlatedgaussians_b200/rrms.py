"""Drop-in ``rrms(stfe, stf, ii, jj, n1) -> (ov, tk)`` (python/rrms.py:21-120):
the overlap and the n1-th Cartesian component of the position vector times
the overlap, for bra ii under symmetry term stfe and ket jj under stf (all
1-based), evaluated by the CUDA library from the module state in ``shared``.
``rrms_batch`` evaluates many terms in one launch."""
from __future__ import annotations

import numpy as np

from . import _state
from . import shared as sh


def rrms_batch(terms) -> np.ndarray:
    """(nterms, 2) array of (ov, tk) for 1-based (stfe, stf, ii, jj, n1) rows."""
    return _state.engine().rrms(sh.iv, terms, K=sh.M)


def rrms(stfe: int, stf: int, ii: int, jj: int, n1: int) -> tuple[float, float]:
    out = rrms_batch(np.array([[stfe, stf, ii, jj, n1]], dtype=np.int32))
    return float(out[0, 0]), float(out[0, 1])
