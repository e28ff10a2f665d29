"""Parity cases shared by the golden-fixture generator (make_golden.py) and the
tests. Each case is a small synthetic workload: terrain, release, parameters.
Every input is generated from code here (no reference data files), so the
same inputs can be rebuilt on any machine.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "slab-pro_b200"))
import workloads as W  # noqa: E402


def case_slope35():
    """The 35-degree slope with circular-arc runout, 1600 particles, Coulomb mu=0.4, 60 s."""
    c = W.config1()
    c["frames"] = [1, 10, 60]
    c["json_release"] = {"type": "RECTANGLE", "h0": 2.0,
                         "rectangle": {"center": [150.0, 250.0], "Lx": 100.0, "Ly": 100.0, "rotation_deg": 0.0}}
    c["json_friction"] = {"type": "COULOMB", "coulomb": {"mu": 0.4}}
    return c


def case_plane_voellmy():
    """The reference's hard-coded ANALYTICAL 5-degree bi-plane, rotated ellipse, Voellmy, 20 s."""
    dx = 4.0
    z = W.analytical_plane(400.0, 300.0, dx)
    cfg = dict(gravity=9.81, rho=1000.0, C_cfl=0.5, dt_max=0.05, flip_ratio=0.9, output_dt=2.0, total_time=20.0,
               friction="VOELLMY", voellmy_mu=0.15, voellmy_xi=800.0)
    rel = {"type": "ELLIPSE", "center": (80.0, 90.0), "rx": 30.0, "ry": 20.0, "rotation_deg": 25.0, "h0": 3.0}
    P = W.release_particles(z, dx, rel, cfg["rho"])
    return {"name": "plane5_ellipse_voellmy", "z": z, "dx": dx, "cfg": cfg, "release": rel, "particles": P,
            "frames": [1, 5, 10], "analytical": {"Lx": 400.0, "Ly": 300.0, "dx": dx},
            "json_release": {"type": "ELLIPSE", "h0": 3.0, "ellipse": {"center": [80.0, 90.0], "rx": 30.0, "ry": 20.0, "rotation_deg": 25.0}},
            "json_friction": {"type": "VOELLMY", "voellmy": {"mu": 0.15, "xi": 800.0}}}


def case_fractal_mui():
    """Small seeded fractal slope, star-polygon RASTER release with lognormal heights, mu(I), 15 s."""
    dx = 2.0
    z = W.fractal_slope_dem(160, dx, seed=7, rms=2.0, lowpass_m=12.0, x_plane_end=180.0, ease_m=80.0)[:, :96]
    poly = W.star_polygon(11, center=(60.0, 96.0), ax=24.0, ay=16.0)
    rel = W.lognormal_release_raster(12, poly, cellsize=2.0, median=1.5, sigma_log=0.4, corr_m=4.0)
    rel["h_min"] = 0.2
    cfg = dict(gravity=9.81, rho=1500.0, C_cfl=0.5, dt_max=0.02, flip_ratio=0.95, output_dt=1.5, total_time=15.0,
               friction="MU_I", mui_mu1=0.38, mui_mu2=0.64, mui_I0=0.279, mui_d=5e-4, mui_phi=0.6)
    P = W.release_particles(z, dx, rel, cfg["rho"])
    return {"name": "fractal_raster_mui", "z": z, "dx": dx, "cfg": cfg, "release": rel, "particles": P,
            "frames": [1, 4, 10],
            "json_release": {"type": "RASTER", "h0": 0.0, "raster": {"filepath": "release.asc", "h_min": 0.2}},
            "json_friction": {"type": "MU_I", "mu_I": {"mu_1": 0.38, "mu_2": 0.64, "I0": 0.279, "d": 5e-4, "phi": 0.6}}}


CASES = {"slope35": case_slope35, "plane_voellmy": case_plane_voellmy, "fractal_mui": case_fractal_mui}


def particle_digest(P: dict) -> str:
    import hashlib
    h = hashlib.sha256()
    for k in ("x", "z", "v", "vz", "h", "A", "mass", "theta"):
        h.update(np.ascontiguousarray(P[k], dtype=np.float64).tobytes())
    return h.hexdigest()


def case_c2_window():
    """A small window of the config-2 construction for GPU parity over whole
    runs: a 512 x 512 DEM at 1 m (30-degree slope easing to 5 degrees over
    100 m from x = 300 m, fBm roughness of 4 m RMS, a 40 m containing rim), a
    seeded star-polygon raster release (~70 x 45 m, lognormal heights,
    h_min 0.2 m), POISSON sampling at 0.5 m with the numpy sampler (~17 k
    particles), Voellmy mu 0.2, xi 1500, 40 s. Not a golden case: the tests
    run the oracle on it."""
    dx = 1.0
    z = W.fractal_slope_dem(512, dx, seed=2026, rms=4.0, x_plane_end=300.0, ease_m=100.0, rim_m=40.0)
    poly = W.star_polygon(2027, center=(110.0, 256.0), ax=70.0, ay=45.0)
    rel = W.lognormal_release_raster(2028, poly, cellsize=dx)
    rel["h_min"] = 0.2
    cfg = dict(gravity=9.81, rho=300.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0, total_time=40.0,
               friction="VOELLMY", voellmy_mu=0.2, voellmy_xi=1500.0)
    h = rel["h"]
    samples = W.poisson_disk_np((h.shape[0] - 1) * dx, (h.shape[1] - 1) * dx, 0.5, 2029)
    P = W.release_particles(z, dx, rel, cfg["rho"], sampling="GIVEN", samples=samples)
    return {"name": "c2_window512_dx1_star_voellmy", "z": z, "dx": dx, "cfg": cfg, "release": rel, "particles": P}
