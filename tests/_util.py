"""Shared helpers of the test suite: golden fixtures and tolerances.

Tolerances (FP64, against the reference / oracle):
  matrix elements  1e-12 relative
  energy           1e-10 Eh absolute
  gradient         1e-9 relative, norm-wise: max|g - g_ref| / max|g_ref|
"""
from __future__ import annotations

import os

import numpy as np

from nbo_correlatedgaussians_b200.problem import Problem

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TOL_ELEM = 1e-12
TOL_E = 1e-10
TOL_G = 1e-9


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name))


def problem_from(d, iv=None) -> Problem:
    return Problem(int(d["n"]), int(d["K"]), float(d["efs"]), d["mass"], d["ncv"], d["scvv"], d["sml"],
                   d["sms"], d["iv"] if iv is None else iv, d["C"] if "C" in d else np.full(int(d["K"]), 1.0 / int(d["K"])))


def normwise(a, b) -> float:
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def elem_rel(got, ref, ov_ref=None, efs=0.0) -> np.ndarray:
    """Per-element relative error of (ov, tk, ert, zht) rows.  zht = ov efs sum q_i T_iz
    can cancel to ~0, so its floor is |ov efs| (the size of one field term)."""
    got, ref = np.asarray(got), np.asarray(ref)
    floor = np.full(ref.shape, 1e-300)
    floor[:, 3] = np.maximum(np.abs(ref[:, 0] * efs), 1e-300)
    return np.abs(got - ref) / np.maximum(np.abs(ref), floor)


def rrms_rel(got, ref) -> np.ndarray:
    """Per-element relative error of (ov, tk) rows of rrms.  tk = st[n1] ov, and a
    component of the position vector st can cancel to ~0 (rounding-level values
    of either sign), so the tk floor is 1e-4 |ov| (st components are O(0.1))."""
    got, ref = np.asarray(got), np.asarray(ref)
    floor = np.full(ref.shape, 1e-300)
    floor[:, 1] = np.maximum(1e-4 * np.abs(ref[:, 0]), 1e-300)
    return np.abs(got - ref) / np.maximum(np.abs(ref), floor)
