"""Device-resident evaluation engine over the C ABI (include/necg.h).

``Engine`` owns one ``necg_handle`` (problem constants + device workspace) and
PyTorch-allocated device buffers.  PyTorch is used only for device memory and
streams; all arithmetic runs in libnecg_b200.so.

Entry points mirror the reference's hot path:
  outprod(x)                python/outprod.py:20-76   -> (f, g) host arrays
  outprod_device(x)         same, on device tensors (no host copies)
  build_matrices(iv, C)     python/necg.py:36-58      -> H, S, Kinetic, Potential
  make_grad(...)            python/make_grad.py:18-90
  matel(terms), gradel(terms)  python/matel.py:28, python/gradel.py:27 (batched)
  rrms(terms), dipole(iv, C)   python/rrms.py:21, python/necg.py:200-244
Errors are raised like the reference raises them: a basis pair whose A_k + A_l'
is not positive definite raises numpy.linalg.LinAlgError (np.linalg.inv does the
same in python/matel.py:93).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .problem import Problem


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("nbo_correlatedgaussians_b200 needs a CUDA device; none is visible")
    return torch.device("cuda", torch.cuda.current_device())


class Engine:
    """One particle system + symmetry set on one GPU, for bases of up to ``K_max``."""

    def __init__(self, prob: Problem, K_max: int | None = None, device=None):
        self.L = _lib.lib()
        self.device = torch.device(device) if device is not None else require_cuda()
        self.n, self.nst, self.efs = prob.n, prob.nst, float(prob.efs)
        self.K_max = int(K_max or prob.K)
        self.blk = prob.blk
        self._consts = [np.ascontiguousarray(a, dtype=np.float64)
                        for a in (prob.mass, prob.ncv, prob.scvv, prob.sml, prob.sms)]
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            rc = self.L.necg_create(self.n, self.nst, self.K_max, self.efs,
                                    *[a.ctypes.data for a in self._consts], ctypes.byref(h))
        _lib.check(rc, "necg_create")
        self.h = h
        dev = self.device
        self._f = torch.zeros(2, dtype=torch.float64, device=dev)
        self._x = None
        self._g = None

    # ------------------------------------------------------------------ util
    def close(self, sync: bool = True) -> None:
        """Release the handle.  necg_destroy returns the workspace to the
        library's device pool without waiting for the GPU, so no work that uses
        it may still be running: by default the device is synchronised first;
        a caller that knows its work has completed passes sync=False."""
        if getattr(self, "h", None):
            if sync:
                torch.cuda.synchronize(self.device)
            self.L.necg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def workspace_bytes(self) -> int:
        return int(self.L.necg_workspace_bytes(self.h))

    def prepare_fused(self, K: int) -> int:
        """Build the fused pass's tile list and partial buffers for bases of K
        functions now (else the first batched step does it); returns the tile
        count, or 0 when the symmetry set does not allow the fused pass."""
        n = ctypes.c_int(0)
        rc = self.L.necg_shard_tiles(self.h, int(K), ctypes.byref(n))
        if rc == _lib.NECG_ERR_UNSUPPORTED:
            return 0
        _lib.check(rc, "necg_shard_tiles")
        return n.value

    def set_tiles(self, lc_energy: int, lc_grad: int) -> None:
        _lib.check(self.L.necg_set_tiles(self.h, int(lc_energy), int(lc_grad)), "necg_set_tiles")

    def status(self) -> tuple[int, int]:
        bad = ctypes.c_longlong(-1)
        rc = self.L.necg_status(self.h, ctypes.byref(bad))
        return rc, bad.value

    def raise_status(self, where: str) -> None:
        rc, bad = self.status()
        if rc == _lib.NECG_OK:
            return
        if rc == _lib.NECG_ERR_NOT_PD:
            raise np.linalg.LinAlgError(f"{where}: A_k + A_l' is not positive definite (first pair index {bad})")
        raise _lib.NecgError(rc, where)

    def _len(self, K: int) -> int:
        return K * self.blk + K

    def _tensor(self, a, K=None) -> torch.Tensor:
        if isinstance(a, torch.Tensor):
            t = a
            if t.device != self.device or t.dtype != torch.float64:
                t = t.to(self.device, torch.float64)
            return t.contiguous()
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)

    # -------------------------------------------------------------- outprod
    def outprod_device(self, x: torch.Tensor, K: int, g: torch.Tensor | None = None,
                       f: torch.Tensor | None = None, H: torch.Tensor | None = None,
                       S: torch.Tensor | None = None, stream=None):
        """Evaluate on device tensors; returns (f (1,), g) device tensors.  Asynchronous."""
        x = self._tensor(x)
        if x.numel() != self._len(K):
            raise ValueError(f"x has {x.numel()} entries, expected {self._len(K)}")
        if g is None:
            g = torch.empty(self._len(K), dtype=torch.float64, device=self.device)
        if f is None:
            f = torch.empty(1, dtype=torch.float64, device=self.device)
        rc = self.L.necg_outprod(self.h, K, x.data_ptr(), f.data_ptr(), g.data_ptr(), _ptr(H), _ptr(S),
                                 _stream_ptr(stream))
        _lib.check(rc, "necg_outprod")
        return f, g

    def outprod(self, x: np.ndarray) -> tuple[float, np.ndarray]:
        """python/outprod.py:20 outprod(x) -> (f, g) through the host-pointer entry point."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        K = x.size // (self.blk + 1)
        if K * (self.blk + 1) != x.size:
            raise ValueError(f"x has {x.size} entries, not a multiple of blk+1 = {self.blk + 1}")
        g = np.empty_like(x)
        f = ctypes.c_double(0.0)
        rc = self.L.necg_outprod_host(self.h, K, x.ctypes.data, ctypes.addressof(f), g.ctypes.data,
                                      _stream_ptr(None))
        if rc == _lib.NECG_ERR_NOT_PD:
            raise np.linalg.LinAlgError("outprod: A_k + A_l' is not positive definite for some basis pair")
        _lib.check(rc, "necg_outprod_host")
        return f.value, g

    # ------------------------------------------------------- matrix build
    def build_matrices(self, iv, C=None, K: int | None = None, parts: bool = True, stream=None,
                       check: bool = True):
        """H, S (and Kinetic, Potential when ``parts``) as device tensors; also
        en = [E, norm] with E = C^T H C / C^T S C, norm = 1 / C^T S C when C is
        given (python/necg.py:36-71)."""
        iv = self._tensor(iv)
        K = K or iv.numel() // self.blk
        dev = self.device
        H = torch.empty((K, K), dtype=torch.float64, device=dev)
        S = torch.empty_like(H)
        Kin = torch.empty_like(H) if parts else None
        Pot = torch.empty_like(H) if parts else None
        Ct = self._tensor(C) if C is not None else None
        en = torch.empty(2, dtype=torch.float64, device=dev) if C is not None else None
        rc = self.L.necg_build_matrices(self.h, K, iv.data_ptr(), _ptr(Ct), H.data_ptr(), S.data_ptr(),
                                        _ptr(Kin), _ptr(Pot), _ptr(en), _stream_ptr(stream))
        _lib.check(rc, "necg_build_matrices")
        if check:
            self.raise_status("build_matrices")
        return H, S, Kin, Pot, en

    def make_grad(self, iv, C, H, S, eng: float, norm: float, stream=None) -> torch.Tensor:
        iv, C, H, S = (self._tensor(a) for a in (iv, C, H, S))
        K = C.numel()
        g = torch.empty(self._len(K), dtype=torch.float64, device=self.device)
        rc = self.L.necg_make_grad(self.h, K, iv.data_ptr(), C.data_ptr(), H.data_ptr(), S.data_ptr(),
                                   float(eng), float(norm), g.data_ptr(), _stream_ptr(stream))
        _lib.check(rc, "necg_make_grad")
        self.raise_status("make_grad")
        return g

    def make_grad_dev(self, iv, C, H, S, en, stream=None) -> torch.Tensor:
        """Gradient with E and norm read from the device tensor en = [E, norm]."""
        iv, C, H, S, en = (self._tensor(a) for a in (iv, C, H, S, en))
        K = C.numel()
        g = torch.empty(self._len(K), dtype=torch.float64, device=self.device)
        rc = self.L.necg_make_grad_dev(self.h, K, iv.data_ptr(), C.data_ptr(), H.data_ptr(), S.data_ptr(),
                                       en.data_ptr(), g.data_ptr(), _stream_ptr(stream))
        _lib.check(rc, "necg_make_grad_dev")
        return g

    # ------------------------------------------------------ single terms
    def matel(self, iv, terms, K: int | None = None) -> np.ndarray:
        """(nterms, 4) array of (ov, tk, ert, zht); terms are 1-based (stf, ii, jj)."""
        iv = self._tensor(iv)
        K = K or iv.numel() // self.blk
        t = torch.as_tensor(np.ascontiguousarray(terms, dtype=np.int32).reshape(-1, 3), device=self.device)
        out = torch.empty((t.shape[0], 4), dtype=torch.float64, device=self.device)
        rc = self.L.necg_matel(self.h, K, iv.data_ptr(), t.shape[0], t.data_ptr(), out.data_ptr(),
                               _stream_ptr(None))
        _lib.check(rc, "necg_matel")
        self.raise_status("matel")
        return out.cpu().numpy()

    def rrms(self, iv, terms, K: int | None = None) -> np.ndarray:
        """(nterms, 2) array of (ov, tk) of python/rrms.py:21; terms are 1-based
        (stfe, stf, ii, jj, n1)."""
        iv = self._tensor(iv)
        K = K or iv.numel() // self.blk
        t = torch.as_tensor(np.ascontiguousarray(terms, dtype=np.int32).reshape(-1, 5), device=self.device)
        out = torch.empty((t.shape[0], 2), dtype=torch.float64, device=self.device)
        rc = self.L.necg_rrms(self.h, K, iv.data_ptr(), t.shape[0], t.data_ptr(), out.data_ptr(),
                              _stream_ptr(None))
        _lib.check(rc, "necg_rrms")
        self.raise_status("rrms")
        return out.cpu().numpy()

    def dipole(self, iv, C) -> tuple[np.ndarray, np.ndarray]:
        """(comps, dipole): the 3n component expectation values and the dipole
        (d_x, d_y, d_z) of python/necg.py:200-244, in atomic units."""
        iv, C = self._tensor(iv), self._tensor(C)
        K = C.numel()
        comps = torch.empty(3 * self.n, dtype=torch.float64, device=self.device)
        dip = torch.empty(3, dtype=torch.float64, device=self.device)
        rc = self.L.necg_dipole(self.h, K, iv.data_ptr(), C.data_ptr(), comps.data_ptr(), dip.data_ptr(),
                                _stream_ptr(None))
        _lib.check(rc, "necg_dipole")
        self.raise_status("dipole")
        return comps.cpu().numpy(), dip.cpu().numpy()

    def gradel(self, iv, terms, K: int | None = None):
        """(tgvl, tgvls), each (nterms, blk); terms are 1-based (stf, ii, jj)."""
        iv = self._tensor(iv)
        K = K or iv.numel() // self.blk
        t = torch.as_tensor(np.ascontiguousarray(terms, dtype=np.int32).reshape(-1, 3), device=self.device)
        tg = torch.empty((t.shape[0], self.blk), dtype=torch.float64, device=self.device)
        tgs = torch.empty_like(tg)
        rc = self.L.necg_gradel(self.h, K, iv.data_ptr(), t.shape[0], t.data_ptr(), tg.data_ptr(),
                                tgs.data_ptr(), _stream_ptr(None))
        _lib.check(rc, "necg_gradel")
        self.raise_status("gradel")
        return tg.cpu().numpy(), tgs.cpu().numpy()


def boys_f0(z) -> tuple[np.ndarray, np.ndarray]:
    """F0(z) and F0'(z) on the device (python/utils.py:78-106)."""
    dev = require_cuda()
    zt = torch.as_tensor(np.atleast_1d(np.asarray(z, dtype=np.float64)), device=dev).contiguous()
    f = torch.empty_like(zt)
    df = torch.empty_like(zt)
    _lib.check(_lib.lib().necg_f0(zt.data_ptr(), zt.numel(), f.data_ptr(), df.data_ptr(), _stream_ptr(None)),
               "necg_f0")
    return f.cpu().numpy(), df.cpu().numpy()


def term_flops(n: int) -> dict:
    """Algorithmic FLOPs per (k, l, P) term: energy, ordered gradient, and one
    unordered term of the symmetric ("sym") and fused ("fused") passes."""
    L = _lib.lib()
    out = {}
    for which, name in ((0, "energy"), (1, "grad"), (2, "sym"), (3, "fused")):
        s = ctypes.c_longlong(0)
        tot = L.necg_term_flops(int(n), which, ctypes.byref(s))
        out[name] = int(tot)
        out[name + "_special"] = int(s.value)
    return out
