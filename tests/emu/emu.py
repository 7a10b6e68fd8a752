"""TEST INFRASTRUCTURE: ctypes wrapper of libnecg_emu.so, the host emulator that
runs the kernels' per-thread bodies (necg_lanes.cuh) tile by tile and lane by
lane on the CPU."""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "necg_emu.cu")
LIB = os.path.join(HERE, "libnecg_emu.so")
CSRC = os.path.join(os.path.dirname(os.path.dirname(HERE)), "nbo_correlatedgaussians_b200", "csrc")
_lib = None


def build() -> str:
    deps = [SRC] + [os.path.join(CSRC, f) for f in ("necg_lanes.cuh", "necg_math.cuh", "necg_hostscalar.cuh")]
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    subprocess.check_call([nvcc, "-O1", "-std=c++17", "-Xcompiler", "-fPIC", "--shared",
                           "-Wno-deprecated-gpu-targets", "-o", LIB + ".tmp", SRC])
    os.replace(LIB + ".tmp", LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
    return _lib


def _p(a):
    return a.ctypes.data


def _consts(p):
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (p.mass, p.ncv, p.scvv, p.sml, p.sms)]
    return arrs


def outprod(p, lc_e=4, lc_g=4):
    L = lib()
    c = _consts(p)
    x = np.ascontiguousarray(p.x)
    f = np.zeros(1)
    g = np.zeros(x.size)
    H = np.zeros((p.K, p.K))
    S = np.zeros((p.K, p.K))
    fn = L.emu_outprod
    fn.restype = ctypes.c_int
    rc = fn(ctypes.c_int(p.n), ctypes.c_int(p.nst), ctypes.c_int(p.K), ctypes.c_double(p.efs),
            *[ctypes.c_void_p(_p(a)) for a in c], ctypes.c_void_p(_p(x)), ctypes.c_int(lc_e), ctypes.c_int(lc_g),
            ctypes.c_void_p(_p(f)), ctypes.c_void_p(_p(g)), ctypes.c_void_p(_p(H)), ctypes.c_void_p(_p(S)))
    return rc, float(f[0]), g, H, S


def outprod_sym(p, lc_e=4, lc_s=4):
    """The symmetric gradient pass (unordered pairs) emulated on the host."""
    L = lib()
    c = _consts(p)
    x = np.ascontiguousarray(p.x)
    f = np.zeros(1)
    g = np.zeros(x.size)
    H = np.zeros((p.K, p.K))
    S = np.zeros((p.K, p.K))
    fn = L.emu_outprod_sym
    fn.restype = ctypes.c_int
    rc = fn(ctypes.c_int(p.n), ctypes.c_int(p.nst), ctypes.c_int(p.K), ctypes.c_double(p.efs),
            *[ctypes.c_void_p(_p(a)) for a in c], ctypes.c_void_p(_p(x)), ctypes.c_int(lc_e), ctypes.c_int(lc_s),
            ctypes.c_void_p(_p(f)), ctypes.c_void_p(_p(g)), ctypes.c_void_p(_p(H)), ctypes.c_void_p(_p(S)))
    return rc, float(f[0]), g, H, S


def outprod_fused(p, lc_s=4):
    """The fused energy + symmetric gradient pass emulated on the host."""
    L = lib()
    c = _consts(p)
    x = np.ascontiguousarray(p.x)
    f = np.zeros(1)
    g = np.zeros(x.size)
    H = np.zeros((p.K, p.K))
    S = np.zeros((p.K, p.K))
    fn = L.emu_outprod_fused
    fn.restype = ctypes.c_int
    rc = fn(ctypes.c_int(p.n), ctypes.c_int(p.nst), ctypes.c_int(p.K), ctypes.c_double(p.efs),
            *[ctypes.c_void_p(_p(a)) for a in c], ctypes.c_void_p(_p(x)), ctypes.c_int(lc_s),
            ctypes.c_void_p(_p(f)), ctypes.c_void_p(_p(g)), ctypes.c_void_p(_p(H)), ctypes.c_void_p(_p(S)))
    return rc, float(f[0]), g, H, S


def rrms(p, terms):
    L = lib()
    c = _consts(p)
    t = np.ascontiguousarray(terms, dtype=np.int32).reshape(-1, 5)
    out = np.zeros((len(t), 2))
    fn = L.emu_rrms
    fn.restype = ctypes.c_int
    rc = fn(ctypes.c_int(p.n), ctypes.c_int(p.nst), ctypes.c_int(p.K), ctypes.c_double(p.efs),
            *[ctypes.c_void_p(_p(a)) for a in c], ctypes.c_void_p(_p(np.ascontiguousarray(p.iv))),
            ctypes.c_int(len(t)), ctypes.c_void_p(_p(t)), ctypes.c_void_p(_p(out)))
    return rc, out


def dipole(p, lc=2):
    L = lib()
    c = _consts(p)
    comps = np.zeros(3 * p.n)
    dip = np.zeros(3)
    fn = L.emu_dipole
    fn.restype = ctypes.c_int
    rc = fn(ctypes.c_int(p.n), ctypes.c_int(p.nst), ctypes.c_int(p.K), ctypes.c_double(p.efs),
            *[ctypes.c_void_p(_p(a)) for a in c], ctypes.c_void_p(_p(np.ascontiguousarray(p.iv))),
            ctypes.c_void_p(_p(np.ascontiguousarray(p.C))), ctypes.c_int(lc), ctypes.c_void_p(_p(comps)),
            ctypes.c_void_p(_p(dip)))
    return rc, comps, dip


def elements(p, terms):
    L = lib()
    c = _consts(p)
    t = np.ascontiguousarray(terms, dtype=np.int32).reshape(-1, 3)
    mat = np.zeros((len(t), 4))
    tg = np.zeros((len(t), p.blk))
    tgs = np.zeros((len(t), p.blk))
    fn = L.emu_elements
    fn.restype = ctypes.c_int
    rc = fn(ctypes.c_int(p.n), ctypes.c_int(p.nst), ctypes.c_int(p.K), ctypes.c_double(p.efs),
            *[ctypes.c_void_p(_p(a)) for a in c], ctypes.c_void_p(_p(np.ascontiguousarray(p.iv))),
            ctypes.c_int(len(t)), ctypes.c_void_p(_p(t)), ctypes.c_void_p(_p(mat)), ctypes.c_void_p(_p(tg)),
            ctypes.c_void_p(_p(tgs)))
    return rc, mat, tg, tgs
