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
    tmp = f"{LIB}.{os.getpid()}.tmp"  # processes started together may build at the same time
    subprocess.check_call([nvcc, "-O1", "-std=c++17", "-Xcompiler", "-fPIC", "--shared",
                           "-Wno-deprecated-gpu-targets", "-o", tmp, SRC])
    os.replace(tmp, LIB)
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


class EmuShardOps:
    """The shard steps of ``nbo_correlatedgaussians_b200.shard.DeviceShardOps``
    run by the host emulation of the kernels, on CPU tensors, so that the
    sharded orchestration (tile ranges, the two all-reduces, E and GRADC from
    the summed rows) can be tested on CPU ranks with the gloo backend."""

    def __init__(self, p, lc_s=2):
        import torch
        self.torch = torch
        self.p = p
        self.lc = int(lc_s)
        self.n, self.blk = p.n, p.blk
        self.ps = p.n * (p.n + 1) // 2 + 1 + 3 * p.n
        self.device = torch.device("cpu")
        self._sumH = self._sumS = None
        self._status = 0

    def _call_pairs(self, x, K, t0, t1):
        L = lib()
        c = _consts(self.p)
        rows = np.zeros(2 * K)
        sH = np.zeros(self.ps * K)
        sS = np.zeros(self.ps * K)
        nt = ctypes.c_int(0)
        fn = L.emu_shard_pairs
        fn.restype = ctypes.c_int
        rc = fn(ctypes.c_int(self.p.n), ctypes.c_int(self.p.nst), ctypes.c_int(K), ctypes.c_double(self.p.efs),
                *[ctypes.c_void_p(_p(a)) for a in c], ctypes.c_void_p(_p(x)), ctypes.c_int(self.lc),
                ctypes.c_int(t0), ctypes.c_int(t1), ctypes.c_void_p(_p(rows)), ctypes.c_void_p(_p(sH)),
                ctypes.c_void_p(_p(sS)), ctypes.byref(nt))
        return rc, rows, sH, sS, nt.value

    def tiles(self, K):
        x = np.ascontiguousarray(self.p.x)
        rc, _, _, _, nt = self._call_pairs(x, K, 0, 0)
        assert rc >= 0
        return nt

    def pairs(self, x, K, t0, t1):
        xn = np.ascontiguousarray(x.numpy())
        rc, rows, self._sumH, self._sumS, _ = self._call_pairs(xn, K, t0, t1)
        assert rc >= 0
        self._status = 2 if rc & 1 else (3 if rc & 2 else 0)
        return self.torch.from_numpy(rows)

    def grad(self, x, K, rows, t0, t1):
        # the finalize kernel: E, norm and GRADC from the summed rows
        xn = x.numpy()
        C = xn[K * self.blk:]
        r = rows.numpy()
        cHc, cSc = float(C @ r[:K]), float(C @ r[K:])
        E, norm = cHc / cSc, 1.0 / cSc
        g = np.zeros(K * self.blk + K)
        g[K * self.blk:] = 2.0 * norm * (r[:K] - E * r[K:])
        self._norm = norm
        sums = self._sumH - E * self._sumS
        return (self.torch.tensor([E], dtype=self.torch.float64), self.torch.from_numpy(g),
                self.torch.from_numpy(sums))

    def finish(self, x, K, sums, g):
        L = lib()
        c = _consts(self.p)
        gn = np.ascontiguousarray(g.numpy()).copy()
        fn = L.emu_shard_finish
        fn.restype = ctypes.c_int
        fn(ctypes.c_int(self.p.n), ctypes.c_int(self.p.nst), ctypes.c_int(K), ctypes.c_double(self.p.efs),
           *[ctypes.c_void_p(_p(a)) for a in c], ctypes.c_void_p(_p(np.ascontiguousarray(x.numpy()))),
           ctypes.c_void_p(_p(np.ascontiguousarray(sums.numpy()))), ctypes.c_double(self._norm),
           ctypes.c_void_p(_p(gn)))
        return self.torch.from_numpy(gn)

    def status(self):
        return self._status
