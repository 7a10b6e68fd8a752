"""Drop-in ``gradel(stf, ii, jj)`` (python/gradel.py:27-392): derivatives of
H_ii,jj and S_ii,jj for one symmetry term with respect to the bra block
[vech(L_ii), s_ii], doubled when ii == jj, from the CUDA library."""
from __future__ import annotations

from . import _state
from . import shared as sh


def gradel(stf: int, ii: int, jj: int):
    tg, tgs = _state.engine().gradel(sh.iv, [(stf, ii, jj)], K=sh.M)
    return tg[0], tgs[0]


def gradel_batch(terms):
    return _state.engine().gradel(sh.iv, terms, K=sh.M)
