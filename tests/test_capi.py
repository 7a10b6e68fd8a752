"""The C-ABI library: it builds, loads without a GPU and exports every entry
point that include/necg.h declares; argument errors return codes."""
import ctypes
import os
import re

import pytest

from nbo_correlatedgaussians_b200 import _lib
from nbo_correlatedgaussians_b200.build import build

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "necg.h")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(necg_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def L():
    build()
    return _lib.load()


def test_every_declared_symbol_is_exported(L):
    names = _declared()
    assert len(names) >= 14
    for name in names:
        assert hasattr(L, name), name


def test_bindings_cover_header():
    assert sorted(n for n, _, _ in _lib.SIGNATURES) == _declared()


def test_status_strings(L):
    for code in range(8):
        s = L.necg_status_string(code)
        assert isinstance(s, bytes) and len(s) >= 2
    assert L.necg_status_string(0) == b"ok"


def test_create_rejects_bad_arguments_without_touching_a_device(L):
    h = ctypes.c_void_p()
    one = (ctypes.c_double * 64)(*([1.0] * 64))
    assert L.necg_create(7, 1, 4, 0.0, one, one, one, one, one, ctypes.byref(h)) == _lib.NECG_ERR_UNSUPPORTED
    assert L.necg_create(0, 1, 4, 0.0, one, one, one, one, one, ctypes.byref(h)) == _lib.NECG_ERR_UNSUPPORTED
    assert L.necg_create(2, 0, 4, 0.0, one, one, one, one, one, ctypes.byref(h)) == _lib.NECG_ERR_ARG
    assert L.necg_create(2, 1, 4, 0.0, None, one, one, one, one, ctypes.byref(h)) == _lib.NECG_ERR_ARG
    assert L.necg_create(2, 1, 4, 0.0, one, one, one, one, one, None) == _lib.NECG_ERR_ARG
    assert L.necg_destroy(None) == _lib.NECG_ERR_ARG
    assert L.necg_f0(None, -1, None, None, None) == _lib.NECG_ERR_ARG
    assert L.necg_f0(None, 0, None, None, None) == _lib.NECG_OK


def test_term_flops_counter(L):
    s = ctypes.c_longlong()
    prev = 0
    for n in range(1, 7):
        e = L.necg_term_flops(n, 0, ctypes.byref(s))
        g = L.necg_term_flops(n, 1, ctypes.byref(s))
        assert 0 < e < g and g > prev
        assert s.value == 2 * n * (n + 1) // 2 + n + 1  # 2 rsqrt per Coulomb pair, n rsqrt, 1 exp
        prev = g
    # the current count of an ordered n = 5 gradient term (3337 before the
    # Coulomb derivative coefficients shared one product per pair, 3307 before
    # the factor -4 of Z's update moved into the ket record, 3292 before tau's
    # trace and quadratic form used the symmetric packed forms, 3222 before the
    # Boys function evaluated both of its branches' last products on every lane,
    # 3267 before it took 1/a from a reciprocal for n > 3, 3237 before F0'/F0's
    # numerator became one polynomial)
    assert L.necg_term_flops(5, 1, None) == 3222
    for n in range(1, 7):
        e, g, y, f = (L.necg_term_flops(n, w, None) for w in range(4))
        # an unordered term carries both gradients, so it costs less than two
        # ordered terms; the fused term adds the H and S elements and the split
        # S gradient, less than a separate energy term
        assert g < y < 2 * g
        assert y < f < y + e
    assert L.necg_term_flops(9, 1, None) == -1
