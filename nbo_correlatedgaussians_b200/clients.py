"""Optimiser clients of the serving loop that run in their own processes.

A truncated-Newton run spends about a millisecond of host time per evaluation
inside SciPy (line search and vector updates over x, which has up to ~60,000
parameters here).  Run as threads of the server's own process, hundreds of such
clients take turns on one interpreter lock and the GPU waits for them between
steps.  Clients in other processes send their requests to the server through
``serve.Endpoint`` instead, over one local socket connection per run:

  open   b"O" + pickle((problem, timeout))    -> b"K" + run id (int64)
  eval   b"E" + x as float64 bytes             -> b"K" + f (float64) + g (float64 bytes)
  close  b"C"                                  -> b"K"
  error reply                                  -> b"X" + pickle((type name, message))

This module does not import torch: client processes need no CUDA context.
"""
from __future__ import annotations

import pickle
import struct
import threading
import time
from multiprocessing.connection import Client as _connect

import numpy as np
from scipy.optimize import minimize

OP_OPEN, OP_EVAL, OP_CLOSE = b"O", b"E", b"C"
REPLY_OK, REPLY_ERR = b"K", b"X"

_ERRORS = {"LinAlgError": np.linalg.LinAlgError, "TimeoutError": TimeoutError, "MemoryError": MemoryError,
           "ValueError": ValueError}


def encode_error(exc: BaseException) -> bytes:
    return REPLY_ERR + pickle.dumps((type(exc).__name__, str(exc)))


def decode_error(msg: bytes) -> BaseException:
    name, text = pickle.loads(msg[1:])
    cls = _ERRORS.get(name)
    return cls(text) if cls is not None else RuntimeError(f"{name}: {text}")


def tn_run(evaluate, x0: np.ndarray, maxfun: int) -> int:
    """One truncated-Newton run (SciPy's TNC, the Python analogue of the
    reference's LMQN, source/tn.f) of at most ``maxfun`` evaluations; returns
    the number of evaluations made."""
    count = [0]

    def fun(x):
        count[0] += 1
        return evaluate(x)

    minimize(fun, x0, method="TNC", jac=True, options={"maxfun": int(maxfun)})
    return count[0]


class RemoteRun:
    """One run on a server in another process: ``evaluate(x) -> (f, g)`` like
    ``Server.evaluate``.  Opening blocks until the server admits the run."""

    def __init__(self, address, authkey: bytes, problem, timeout: float | None = None):
        self.conn = _connect(address, authkey=authkey)
        try:
            rep = self._call(OP_OPEN + pickle.dumps((problem, timeout)))
        except BaseException:
            self.conn.close()
            raise
        self.id = struct.unpack_from("<q", rep, 1)[0]

    def _call(self, msg: bytes) -> bytes:
        self.conn.send_bytes(msg)
        rep = self.conn.recv_bytes()
        if rep[:1] == REPLY_ERR:
            raise decode_error(rep)
        return rep

    def evaluate(self, x: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float64)
        rep = self._call(OP_EVAL + x.tobytes())
        f = struct.unpack_from("<d", rep, 1)[0]
        g = np.frombuffer(rep, dtype=np.float64, offset=9).copy()
        return f, g

    def close(self) -> None:
        if self.conn is None:
            return
        try:
            self._call(OP_CLOSE)
        finally:
            self.conn.close()
            self.conn = None


def client_worker(address, authkey: bytes, jobs: list, maxfun: int, ready, gate, go, t0_epoch, out_q) -> None:
    """Body of one client process: a thread per assigned run (index, problem,
    arrival offset), started once every client process is up (``ready``, a
    multiprocessing Barrier).  With ``gate`` (another Barrier) every run opens
    first and the runs start together once all are admitted; otherwise run j
    waits for ``go`` and opens at t0_epoch + its arrival offset.  Puts one
    dict per process on ``out_q``: evaluations and completion time per run,
    and the errors met."""
    res = {"evals": {}, "t_done": {}, "errors": []}
    ready.wait()
    lock = threading.Lock()

    def one(j, prob, t_arr):
        try:
            if gate is None:
                go.wait()
                dt = t0_epoch.value + t_arr - time.time()
                if dt > 0:
                    time.sleep(dt)
            run = RemoteRun(address, authkey, prob)
            try:
                if gate is not None:
                    gate.wait()
                n = tn_run(run.evaluate, prob.x.copy(), maxfun)
            finally:
                run.close()
            with lock:
                res["evals"][j] = n
                res["t_done"][j] = time.time()
        except Exception as exc:  # noqa: BLE001 -- reported to the parent
            with lock:
                res["errors"].append((j, repr(exc)))
            if gate is not None:
                gate.abort()

    th = [threading.Thread(target=one, args=job, daemon=True) for job in jobs]
    for t in th:
        t.start()
    for t in th:
        t.join()
    out_q.put(res)
