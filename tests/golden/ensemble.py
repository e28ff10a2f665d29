"""A small ensemble on one shared terrain for batch / server tests: releases of
different size, position, friction law and duration on the 35-degree slope."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "slab-pro_b200"))
import workloads as W  # noqa: E402

BASE = dict(gravity=9.81, rho=300.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0)


def ensemble():
    z = W.slope_arc_dem()
    specs = [
        (dict(BASE, total_time=12.0, friction="COULOMB", coulomb_mu=0.4),
         {"type": "RECTANGLE", "center": (150.0, 250.0), "Lx": 100.0, "Ly": 100.0, "rotation_deg": 0.0, "h0": 2.0}),
        (dict(BASE, total_time=8.0, friction="VOELLMY", voellmy_mu=0.2, voellmy_xi=1500.0),
         {"type": "ELLIPSE", "center": (200.0, 120.0), "rx": 40.0, "ry": 25.0, "rotation_deg": 30.0, "h0": 1.5}),
        (dict(BASE, total_time=10.0, friction="MU_I", mui_mu1=0.38, mui_mu2=0.64, mui_I0=0.279, mui_d=5e-4, mui_phi=0.6),
         {"type": "ELLIPSE", "center": (300.0, 380.0), "rx": 60.0, "ry": 35.0, "rotation_deg": -15.0, "h0": 3.0}),
        (dict(BASE, total_time=6.0, dt_max=0.02, friction="VOELLMY", voellmy_mu=0.35, voellmy_xi=600.0),
         {"type": "RECTANGLE", "center": (120.0, 420.0), "Lx": 30.0, "Ly": 50.0, "rotation_deg": 10.0, "h0": 1.0}),
    ]
    out = []
    for cfg, rel in specs:
        out.append((cfg, W.release_particles(z, 5.0, rel, cfg["rho"])))
    return z, 5.0, out
