"""ctypes wrapper around the CPU oracle (``necg_oracle.c``).

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it as the checker.  The product package
never imports it.

The oracle restates the reference Python path (python/matel.py:28-210,
python/gradel.py:27-392, python/outprod.py:20-76, python/make_grad.py:18-90,
python/utils.py:78-106, python/rrms.py:21-120 and the dipole loop of
python/necg.py:200-244) in C; see the header of ``necg_oracle.c``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class _Problem(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("nst", ctypes.c_int), ("K", ctypes.c_int),
        ("efs", ctypes.c_double),
        ("mass", _dp), ("ncv", _dp), ("scvv", _dp), ("sml", _dp), ("sms", _dp),
    ]


def build(force: bool = False) -> str:
    """Compile liboracle.so with gcc (no GPU needed)."""
    src = os.path.join(_HERE, "necg_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE], stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_f0.restype = ctypes.c_double
        L.oracle_f0.argtypes = [ctypes.c_double]
        L.oracle_df0.restype = ctypes.c_double
        L.oracle_df0.argtypes = [ctypes.c_double]
        P = ctypes.POINTER(_Problem)
        L.oracle_matel.argtypes = [P, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        L.oracle_gradel.argtypes = [P, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.oracle_build_matrices.argtypes = [P, _dp, ctypes.c_int, _dp, _dp, _dp, _dp]
        L.oracle_outprod.argtypes = [P, _dp, ctypes.c_int, _dp, _dp, _dp, _dp]
        L.oracle_rrms.argtypes = [P, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  _dp]
        L.oracle_dipole.argtypes = [P, _dp, _dp, ctypes.c_int, _dp, _dp]
        L.oracle_sample_terms.restype = ctypes.c_double
        L.oracle_sample_terms.argtypes = [P, _dp, ctypes.c_int, _ip, ctypes.c_int, _ip]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_dp)


class Oracle:
    """One problem (particles, symmetry set, basis size) for the oracle.

    ``sml`` is (nst, n, n) with ``sml[s] == shared.sml[:, :, s]`` of the
    reference, ``sms`` is (nst, 3n, 3n), ``scvv`` is already divided by nst.
    """

    def __init__(self, n, K, efs, mass, ncv, scvv, sml, sms):
        self.n, self.K = int(n), int(K)
        self.nst = len(scvv)
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (mass, ncv, scvv, sml, sms)]
        m, q, w, s1, s2 = self._keep
        self.blk = self.n * (self.n + 1) // 2 + 3 * self.n
        self.siv = self.K * self.blk
        self._p = _Problem(self.n, self.nst, self.K, float(efs), _ptr(m), _ptr(q), _ptr(w), _ptr(s1), _ptr(s2))

    @classmethod
    def from_problem(cls, prob):
        """Build from any object with n, K, efs, mass, ncv, scvv, sml, sms."""
        return cls(prob.n, prob.K, prob.efs, prob.mass, prob.ncv, prob.scvv, prob.sml, prob.sms)

    def f0(self, z):
        return lib().oracle_f0(float(z))

    def df0(self, z):
        return lib().oracle_df0(float(z))

    def matel(self, iv, stf, ii, jj):
        iv = np.ascontiguousarray(iv, dtype=np.float64)
        out = np.zeros(4)
        rc = lib().oracle_matel(ctypes.byref(self._p), _ptr(iv), int(stf), int(ii), int(jj), _ptr(out))
        if rc:
            raise np.linalg.LinAlgError("singular matrix in oracle matel")
        return tuple(out)

    def gradel(self, iv, stf, ii, jj):
        iv = np.ascontiguousarray(iv, dtype=np.float64)
        tg = np.zeros(self.blk)
        tgs = np.zeros(self.blk)
        rc = lib().oracle_gradel(ctypes.byref(self._p), _ptr(iv), int(stf), int(ii), int(jj), _ptr(tg), _ptr(tgs))
        if rc:
            raise np.linalg.LinAlgError("singular matrix in oracle gradel")
        return tg, tgs

    def rrms(self, iv, stfe, stf, ii, jj, n1):
        iv = np.ascontiguousarray(iv, dtype=np.float64)
        out = np.zeros(2)
        rc = lib().oracle_rrms(ctypes.byref(self._p), _ptr(iv), int(stfe), int(stf), int(ii), int(jj), int(n1),
                               _ptr(out))
        if rc:
            raise np.linalg.LinAlgError("singular matrix in oracle rrms")
        return tuple(out)

    def dipole(self, iv, C, nthreads=1):
        """(comps (3n,), dipole (3,)) of the dipole loop of python/necg.py:200-244."""
        iv = np.ascontiguousarray(iv, dtype=np.float64)
        C = np.ascontiguousarray(C, dtype=np.float64)
        comps = np.zeros(3 * self.n)
        dip = np.zeros(3)
        rc = lib().oracle_dipole(ctypes.byref(self._p), _ptr(iv), _ptr(C), int(nthreads), _ptr(comps), _ptr(dip))
        if rc:
            raise np.linalg.LinAlgError("oracle dipole failed")
        return comps, dip

    def build_matrices(self, iv, nthreads=1):
        iv = np.ascontiguousarray(iv, dtype=np.float64)
        K = self.K
        H, S, Kin, Pot = (np.zeros((K, K)) for _ in range(4))
        rc = lib().oracle_build_matrices(ctypes.byref(self._p), _ptr(iv), int(nthreads), _ptr(H), _ptr(S), _ptr(Kin), _ptr(Pot))
        if rc:
            raise np.linalg.LinAlgError("oracle build failed")
        return H, S, Kin, Pot

    def outprod(self, x, nthreads=1, return_hs=False):
        x = np.ascontiguousarray(x, dtype=np.float64)
        K = self.K
        f = ctypes.c_double(0.0)
        g = np.zeros(self.siv + K)
        H = np.zeros((K, K))
        S = np.zeros((K, K))
        rc = lib().oracle_outprod(ctypes.byref(self._p), _ptr(x), int(nthreads), ctypes.cast(ctypes.byref(f), _dp), _ptr(g), _ptr(H), _ptr(S))
        if rc:
            raise np.linalg.LinAlgError("oracle outprod failed")
        if return_hs:
            return f.value, g, H, S
        return f.value, g

    def sample_terms(self, iv, mat_terms, grad_terms):
        """Evaluate a list of (stf, ii, jj) matel terms and gradel terms; returns a checksum."""
        iv = np.ascontiguousarray(iv, dtype=np.float64)
        mt = np.ascontiguousarray(mat_terms, dtype=np.int32).reshape(-1, 3)
        gt = np.ascontiguousarray(grad_terms, dtype=np.int32).reshape(-1, 3)
        return lib().oracle_sample_terms(ctypes.byref(self._p), _ptr(iv), len(mt), mt.ctypes.data_as(_ip), len(gt), gt.ctypes.data_as(_ip))
