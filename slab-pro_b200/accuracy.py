"""Accuracy measures of a run against an FP64 run of the same scenario:
max-flow-height and max-speed maps node by node (within 1 cm or 1 %, within
0.1 m/s or 1 %), runout, the centre-of-mass trajectory frame by frame, total
mass.

Short runs (the GPU tests' cases, the reference's Brienz example) hold the
FP32 split path to h_max within 1 cm or 1 % on at least 99.5 % of the wet
nodes and runout within one grid cell. Whole runs on rough terrain are
chaotic: there the same measures of FP64 against FP64 started from positions
moved by 1e-7 cell (the FP64 envelope, bench.py) set the scale the FP32
error is compared with."""
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


def v_ok(va: np.ndarray, vb: np.ndarray) -> np.ndarray:
    """Nodes whose max speeds agree within 0.1 m/s or 1 %."""
    return np.abs(va - vb) <= np.maximum(0.1, 0.01 * np.maximum(va, vb))


def compare_runs(a: dict, b: dict, dx: float) -> dict:
    """Run a against run b, both {"box", "h_max", "v_max" (speeds, over box),
    "com" [frames, 2], "mass"}: the max-flow-height map (fraction of wet
    nodes within 1 cm / 1 %, largest difference), the max-velocity map
    (fraction within 0.1 m/s / 1 %, largest difference), the runout
    difference in cells, the largest centre-of-mass distance over the output
    frames, and the relative difference of the total masses."""
    u = [min(a["box"][0], b["box"][0]), max(a["box"][1], b["box"][1]), min(a["box"][2], b["box"][2]),
         max(a["box"][3], b["box"][3])]
    ha, hb = crop(a["box"], a["h_max"], u), crop(b["box"], b["h_max"], u)
    va, vb = crop(a["box"], a["v_max"], u), crop(b["box"], b["v_max"], u)
    wet = (ha > 0) | (hb > 0)
    n = min(len(a["com"]), len(b["com"]))
    dcom = np.linalg.norm(np.asarray(a["com"])[:n] - np.asarray(b["com"])[:n], axis=1) if n else np.zeros(1)
    return {"wet_nodes": int(wet.sum()),
            "h_within_1cm_1pct": float(h_ok(ha, hb)[wet].mean()) if wet.any() else 1.0,
            "h_max_abs_m": float(np.abs(ha - hb).max()) if ha.size else 0.0,
            "v_within_01ms_1pct": float(v_ok(va, vb)[wet].mean()) if wet.any() else 1.0,
            "v_max_abs_ms": float(np.abs(va - vb).max()) if va.size else 0.0,
            "runout_diff_cells": float(abs(runout(ha, dx, i0=u[0]) - runout(hb, dx, i0=u[0])) / dx),
            "com_max_m": float(dcom.max()), "com_final_m": float(dcom[-1]) if n else 0.0, "frames": int(n),
            "mass_rel": float(abs(a["mass"] - b["mass"]) / b["mass"]) if b["mass"] else 0.0}


def summarize(rows: list) -> dict:
    """Worst case over scenarios of compare_runs results."""
    if not rows:
        return {}
    worst = {"h_within_1cm_1pct": min, "h_max_abs_m": max, "v_within_01ms_1pct": min, "v_max_abs_ms": max,
             "runout_diff_cells": max, "com_max_m": max, "mass_rel": max}
    out = {k: f(r[k] for r in rows) for k, f in worst.items()}
    out["scenarios"] = len(rows)
    out["median_h_within_1cm_1pct"] = float(np.median([r["h_within_1cm_1pct"] for r in rows]))
    return out
