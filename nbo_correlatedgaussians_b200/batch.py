"""Batched evaluation of many independent instances in one step.

Each instance (a basis of any n <= 5, nst, K) has its own ``Engine`` (handle +
device workspace) with tile widths chosen by the autotuner for its (n, K).  A
``BatchEngine`` plans a step over any subset of its instances: when every
instance's symmetry set is closed under inverse, the pair work of all of them
is one persistent launch of the fused pass over a single queue (instances by
decreasing tile cost, each over its own tile groups; 8-warp lockstep blocks, or
one-warp blocks when the plan is too small to fill the SMs); otherwise one
queue of energy tiles and one of ordered gradient tiles.  The step is a fixed
sequence of kernels with fixed grids, so each mode's step is captured once as
a CUDA graph and replayed for every later plan.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .autotune import tuned
from .engine import Engine, _stream_ptr
from .problem import Problem


class Batch:
    """Thin owner of one necg_batch: plans over any engines and device tensors."""

    def __init__(self, max_instances: int, max_tiles: int = 1 << 20):
        self.L = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(self.L.necg_batch_create(max(1, int(max_instances)), int(max_tiles), ctypes.byref(h)),
                   "necg_batch_create")
        self.b = h
        self.graph_ready = False
        self.count = 0

    def close(self) -> None:
        if getattr(self, "b", None):
            self.L.necg_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def plan(self, engines, Ks, xs, gs, fs, stream=None) -> None:
        n = len(engines)
        arr = lambda typ, vals: (typ * max(1, n))(*vals)  # noqa: E731
        _lib.check(self.L.necg_batch_plan(
            self.b, n, arr(ctypes.c_void_p, [e.h.value for e in engines]), arr(ctypes.c_int, list(Ks)),
            arr(ctypes.c_void_p, [t.data_ptr() for t in xs]), arr(ctypes.c_void_p, [t.data_ptr() for t in gs]),
            arr(ctypes.c_void_p, [t.data_ptr() for t in fs]), _stream_ptr(stream)), "necg_batch_plan")
        self.count = n

    def step(self, graph: bool = True, stream=None) -> None:
        s = _stream_ptr(stream)
        if graph:
            if not self.graph_ready:
                _lib.check(self.L.necg_batch_graph(self.b, s), "necg_batch_graph")
                self.graph_ready = True
            _lib.check(self.L.necg_batch_replay(self.b, s), "necg_batch_replay")
        else:
            _lib.check(self.L.necg_batch_step(self.b, s), "necg_batch_step")

    def status_async(self, flags_host, stream=None) -> None:
        """Enqueue a copy of the last step's raw status words (2 ints per
        instance) into the pinned int32 tensor ``flags_host``."""
        _lib.check(self.L.necg_batch_status_async(self.b, ctypes.c_void_p(flags_host.data_ptr()), _stream_ptr(stream)),
                   "necg_batch_status_async")

    @staticmethod
    def decode(flags) -> list[int]:
        """Status codes from raw flag words (as necg_batch_status returns them)."""
        out = []
        for fl in flags:
            fl = int(fl)
            out.append(_lib.NECG_ERR_NOT_PD if fl & 1 else _lib.NECG_ERR_NONFINITE if fl & 2 else _lib.NECG_OK)
        return out

    def status(self, stream=None) -> list[int]:
        out = (ctypes.c_int * max(1, self.count))()
        self.L.necg_batch_status(self.b, out, _stream_ptr(stream))
        return list(out)[:self.count]


class BatchEngine:
    def __init__(self, problems: list[Problem], tune: bool = True, max_tiles: int = 1 << 20,
                 device=None, K_max: list[int] | None = None):
        self.L = _lib.lib()
        self.problems = list(problems)
        self.engines: list[Engine] = []
        self.x: list[torch.Tensor] = []
        self.g: list[torch.Tensor] = []
        self.f: list[torch.Tensor] = []
        self.tiles: list[dict] = []
        for i, p in enumerate(self.problems):
            if p.n > 5:
                raise ValueError("the batched path supports n <= 5")
            eng = Engine(p, K_max=(K_max[i] if K_max else p.K), device=device)
            x = torch.from_numpy(np.ascontiguousarray(p.x)).to(eng.device)
            self.engines.append(eng)
            self.x.append(x)
            self.g.append(torch.empty_like(x))
            self.f.append(torch.zeros(1, dtype=torch.float64, device=eng.device))
            self.tiles.append(tuned(eng, x, p.K) if tune else {})
        self.batch = Batch(len(self.problems), max_tiles)
        self._active: list[int] = []

    def close(self) -> None:
        if getattr(self, "batch", None):
            self.batch.close()
            self.batch = None
        for e in self.engines:
            e.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_x(self, i: int, x) -> None:
        """Copy new parameters [iv, C] into instance i's device input."""
        self.x[i].copy_(torch.as_tensor(x, dtype=torch.float64), non_blocking=True)

    def plan(self, active: list[int] | None = None, stream=None) -> None:
        """Make the next step evaluate the instances in ``active`` (default: all)."""
        active = list(range(len(self.problems))) if active is None else list(active)
        self.batch.plan([self.engines[i] for i in active], [self.problems[i].K for i in active],
                        [self.x[i] for i in active], [self.g[i] for i in active], [self.f[i] for i in active],
                        stream)
        self._active = active

    def step(self, graph: bool = True, stream=None) -> None:
        """Launch one energy+gradient step of the current plan (asynchronous)."""
        self.batch.step(graph, stream)

    def status_async(self, flags_host, stream=None) -> None:
        """Enqueue a copy of the last step's raw status words (2 ints per
        instance) into the pinned int32 tensor ``flags_host``."""
        _lib.check(self.L.necg_batch_status_async(self.b, ctypes.c_void_p(flags_host.data_ptr()), _stream_ptr(stream)),
                   "necg_batch_status_async")

    @staticmethod
    def decode(flags) -> list[int]:
        """Status codes from raw flag words (as necg_batch_status returns them)."""
        out = []
        for fl in flags:
            fl = int(fl)
            out.append(_lib.NECG_ERR_NOT_PD if fl & 1 else _lib.NECG_ERR_NONFINITE if fl & 2 else _lib.NECG_OK)
        return out

    def status(self, stream=None) -> list[int]:
        return self.batch.status(stream)

    def check(self, stream=None) -> None:
        for i, code in zip(self._active, self.status(stream)):
            if code == _lib.NECG_ERR_NOT_PD:
                raise np.linalg.LinAlgError(f"instance {i}: A_k + A_l' is not positive definite")
            if code != _lib.NECG_OK:
                raise _lib.NecgError(code, f"instance {i}")

    def results(self, i: int):
        """(E, gradient) of instance i from the last step, as host values."""
        return float(self.f[i].item()), self.g[i].cpu().numpy()

    def terms(self, active: list[int] | None = None) -> int:
        """(k, l, P) terms of one step counted with the reference's loop structure
        (energy triangle + ordered gradient square), for throughput figures."""
        ids = range(len(self.problems)) if active is None else active
        return sum((p.K * (p.K + 1) // 2 + p.K * p.K) * p.nst for p in (self.problems[i] for i in ids))
