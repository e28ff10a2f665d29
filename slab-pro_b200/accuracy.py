"""Accuracy measures of a run against an FP64 run of the same scenario.

The bar the FP32 split path is held to: max-flow-height maps within 1 cm or
1 % node by node (on at least 99.5 % of the wet nodes, never more than 5 cm
off), runout within one grid cell, total particle mass unchanged."""
from __future__ import annotations

import numpy as np


def runout(hmax: np.ndarray, dx: float, thresh: float = 0.01, i0: int = 0) -> float:
    """Furthest downslope (+x) node with h_max above thresh, in metres; i0 is
    the map's first row on the terrain."""
    wet = np.nonzero((hmax > thresh).any(axis=1))[0]
    return (wet.max() + i0) * dx if len(wet) else 0.0


def h_ok(hm: np.ndarray, ho: np.ndarray) -> np.ndarray:
    """Nodes whose h_max agree within 1 cm or 1 %."""
    return np.abs(hm - ho) <= np.maximum(0.01, 0.01 * np.maximum(hm, ho))


def crop(box_src, m: np.ndarray, box_dst) -> np.ndarray:
    """Map m over node box box_src = [i0, i1, j0, j1] re-indexed to box_dst
    (zero where box_src does not reach)."""
    out = np.zeros((box_dst[1] - box_dst[0] + 1, box_dst[3] - box_dst[2] + 1))
    a0, a1 = max(box_src[0], box_dst[0]), min(box_src[1], box_dst[1])
    b0, b1 = max(box_src[2], box_dst[2]), min(box_src[3], box_dst[3])
    if a1 >= a0 and b1 >= b0:
        out[a0 - box_dst[0]:a1 - box_dst[0] + 1, b0 - box_dst[2]:b1 - box_dst[2] + 1] = \
            m[a0 - box_src[0]:a1 - box_src[0] + 1, b0 - box_src[2]:b1 - box_src[2] + 1]
    return out


def wet_box(m: np.ndarray):
    """Smallest node box holding every node with m > 0 (full-map indices)."""
    ii = np.nonzero((m > 0).any(axis=1))[0]
    jj = np.nonzero((m > 0).any(axis=0))[0]
    if not len(ii):
        return [0, -1, 0, -1]
    return [int(ii[0]), int(ii[-1]), int(jj[0]), int(jj[-1])]


def compare_max_heights(box_a, ha: np.ndarray, box_b, hb: np.ndarray, dx: float) -> dict:
    """h_max of run a (over box_a) against run b (over box_b): fraction of wet
    nodes within 1 cm / 1 %, largest difference, runout difference."""
    if box_a[1] < box_a[0]:
        box_a = box_b
        ha = np.zeros((box_b[1] - box_b[0] + 1, box_b[3] - box_b[2] + 1))
    u = [min(box_a[0], box_b[0]), max(box_a[1], box_b[1]), min(box_a[2], box_b[2]), max(box_a[3], box_b[3])]
    A, B = crop(box_a, ha, u), crop(box_b, hb, u)
    wet = (A > 0) | (B > 0)
    ok = h_ok(A, B)
    return {"wet_nodes": int(wet.sum()), "within_1cm_1pct": float(ok[wet].mean()) if wet.any() else 1.0,
            "max_abs_m": float(np.abs(A - B).max()) if A.size else 0.0,
            "runout_diff_m": float(abs(runout(A, dx, i0=u[0]) - runout(B, dx, i0=u[0])))}
