"""Hessian-vector products for the optimiser (the role of GTIMS in
source/tn.f:1301-1327, which differences two gradients inside the truncated-
Newton inner loop).

``HessianVector(problem)(x, v)`` returns H(x) v by central differences of the
analytic gradient, (g(x + e v) - g(x - e v)) / (2 e), with both gradients
evaluated as two instances of one batched step (one graph replay), so a
product costs one step instead of two sequential evaluations.  The step e is
relative to |v| and |x| (e = eps * (1 + |x|) / |v|); the truncation error is
O(e^2) and the rounding error O(eps_machine / e) relative to |g|.
"""
from __future__ import annotations

import numpy as np
import torch

from .batch import BatchEngine
from .problem import Problem


class HessianVector:
    def __init__(self, prob: Problem, eps: float = 1e-5, tune: bool = True, device=None):
        self.prob = prob
        self.eps = float(eps)
        self.be = BatchEngine([prob, prob], tune=tune, device=device)
        self.be.plan([0, 1])
        self.count = 0

    def __call__(self, x: np.ndarray, v: np.ndarray) -> np.ndarray:
        x = np.asarray(x, dtype=np.float64)
        v = np.asarray(v, dtype=np.float64)
        nv = float(np.linalg.norm(v))
        if nv == 0.0:
            return np.zeros_like(x)
        e = self.eps * (1.0 + float(np.linalg.norm(x))) / nv
        self.be.set_x(0, x + e * v)
        self.be.set_x(1, x - e * v)
        self.be.step(graph=True)
        self.be.check()
        _, gp = self.be.results(0)
        _, gm = self.be.results(1)
        self.count += 1
        return (gp - gm) / (2.0 * e)

    def close(self) -> None:
        self.be.close()
