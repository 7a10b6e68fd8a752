"""ctypes binding of libnecg_b200.so (the C ABI of include/necg.h).

There is no fallback: if the library is missing or no CUDA device is present,
``lib()`` raises, so the product path never silently runs elsewhere.
"""
from __future__ import annotations

import ctypes
import os

from .build import LIB

NECG_OK = 0
NECG_ERR_ARG = 1
NECG_ERR_NOT_PD = 2
NECG_ERR_NONFINITE = 3
NECG_ERR_CUDA = 4
NECG_ERR_ALLOC = 5
NECG_ERR_UNSUPPORTED = 6
NECG_ERR_CAPACITY = 7

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_ll = ctypes.c_longlong

# (name, restype, argtypes) for every entry point of include/necg.h
SIGNATURES = [
    ("necg_create", _i, [_i, _i, _i, _d, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    ("necg_destroy", _i, [_vp]),
    ("necg_workspace_bytes", _ll, [_vp]),
    ("necg_set_tiles", _i, [_vp, _i, _i]),
    ("necg_set_variant", _i, [_vp, _i, _i]),
    ("necg_set_symmetric", _i, [_vp, _i, _i, _i]),
    ("necg_set_splits", _i, [_vp, _i]),
    ("necg_outprod", _i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("necg_outprod_host", _i, [_vp, _i, _vp, _vp, _vp, _vp]),
    ("necg_build_matrices", _i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("necg_make_grad", _i, [_vp, _i, _vp, _vp, _vp, _vp, _d, _d, _vp, _vp]),
    ("necg_make_grad_dev", _i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("necg_matel", _i, [_vp, _i, _vp, _i, _vp, _vp, _vp]),
    ("necg_gradel", _i, [_vp, _i, _vp, _i, _vp, _vp, _vp, _vp]),
    ("necg_rrms", _i, [_vp, _i, _vp, _i, _vp, _vp, _vp]),
    ("necg_shard_tiles", _i, [_vp, _i, _vp]),
    ("necg_shard_pairs", _i, [_vp, _i, _vp, _i, _i, _vp, _vp]),
    ("necg_shard_grad", _i, [_vp, _i, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp]),
    ("necg_shard_finish", _i, [_vp, _i, _vp, _vp, _vp, _vp]),
    ("necg_dipole", _i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    ("necg_f0", _i, [_vp, _i, _vp, _vp, _vp]),
    ("necg_outprod_noalloc", _i, [_i, _i, _i, _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("necg_status", _i, [_vp, ctypes.POINTER(_ll)]),
    ("necg_batch_create", _i, [_i, _i, ctypes.POINTER(_vp)]),
    ("necg_batch_destroy", _i, [_vp]),
    ("necg_batch_plan", _i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("necg_batch_step", _i, [_vp, _vp]),
    ("necg_batch_graph", _i, [_vp, _vp]),
    ("necg_batch_replay", _i, [_vp, _vp]),
    ("necg_batch_status", _i, [_vp, _vp, _vp]),
    ("necg_batch_status_async", _i, [_vp, _vp, _vp]),
    ("necg_status_string", ctypes.c_char_p, [_i]),
    ("necg_profile", _i, [_vp, _i]),
    ("necg_fp64_peak", _i, [_i, _dp, _vp]),
    ("necg_phase_ms", _i, [_vp, _dp]),
    ("necg_term_flops", _ll, [_i, _i, ctypes.POINTER(_ll)]),
]

_lib = None


class NecgError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        msg = _status_text(code)
        super().__init__(f"{where}: {msg} (code {code})" if where else f"{msg} (code {code})")


def _status_text(code: int) -> str:
    try:
        return lib().necg_status_string(code).decode()
    except Exception:  # library not loadable: still report the code
        return f"status {code}"


def load(path: str | None = None):
    """Load the library (no CUDA device needed to load it)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: run `python -m nbo_correlatedgaussians_b200.build` "
                          "(needs nvcc) before using the CUDA engine")
    L = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def lib():
    return load()


def check(code: int, where: str = "") -> None:
    if code != NECG_OK:
        raise NecgError(code, where)
