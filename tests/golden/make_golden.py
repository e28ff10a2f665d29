"""Generate the golden fixtures tests/golden/<case>.npz by running the
reference's own step-loop sources (oracle/_ref/slab_ref, built by
`make -C oracle ref` from the reference tree) on the cases in cases.py.

    python tests/golden/make_golden.py [case ...]
    python tests/golden/make_golden.py setup_poisson
    SLAB_REF_ROOT=<reference checkout> python tests/golden/make_golden.py brienz5m

Each fixture holds, from the reference run:
  frame0_digest   sha256 of the initial particle arrays (setup parity)
  f<k>_<field>    particle arrays at output frame k (x, z, v, vz, h, A, mass,
                  theta), plus f<k>_time / f<k>_dt
  s<k>_<field>    state after step k of the phase driver (steps 1, 2, 50, 51)
  max_idx, max_h, max_v2   nonzero entries of the final h_max / v_max2
  nsteps          steps taken to total_time
The reference binary writes raw FP64 dumps (oracle/ref_hooks.cpp), so the
fixtures are the reference's exact doubles.
"""
from __future__ import annotations

import glob
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import cases  # noqa: E402
import oracle as O  # noqa: E402

sys.path.insert(0, os.path.join(ROOT, "slab-pro_b200"))
import workloads as W  # noqa: E402

PHASE_STEPS = (1, 2, 50, 51)


def write_inputs(c: dict, d: str) -> str:
    cfg = c["cfg"]
    if "analytical" in c:
        terrain = {"type": "ANALYTICAL", "analytical": c["analytical"]}
    else:
        W.write_asc(os.path.join(d, "dem.asc"), c["z"], c["dx"])
        terrain = {"type": "DEM", "dem": {"filepath": os.path.join(d, "dem.asc")}}
    rel = dict(c["json_release"])
    if rel["type"] == "RASTER":
        r = c["release"]
        W.write_asc(os.path.join(d, "release.asc"), r["h"], r["cellsize"], xll=r["x0"], yll=r["y0"])
        rel["raster"] = dict(rel["raster"], filepath=os.path.join(d, "release.asc"))
    j = {"project_dir": os.path.join(d, "out"), "sim_name": c["name"],
         "physical_params": {"gravity": cfg["gravity"], "rho": cfg["rho"]},
         "time_params": {"output_dt": cfg["output_dt"], "total_time": cfg["total_time"]},
         "numerical_params": {"C_cfl": cfg["C_cfl"], "dt_max": cfg["dt_max"], "flip_ratio": cfg["flip_ratio"],
                              "sampling_method": "UNIFORM"},
         "friction": c["json_friction"], "terrain": terrain, "release": rel}
    path = os.path.join(d, "config.json")
    with open(path, "w") as f:
        json.dump(j, f, indent=1)
    return path


def run_ref(cfg_path: str, *args):
    out = subprocess.run([O.REF_BIN, cfg_path, *args], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"slab_ref failed: {out.stderr}")
    return out.stdout


def make(name: str):
    c = cases.CASES[name]()
    out = {}
    with tempfile.TemporaryDirectory() as d:
        cfg_path = write_inputs(c, d)
        sim_dir = os.path.join(d, "out", c["name"])
        run_ref(cfg_path, "--init-only")
        f0 = O.read_particles_bin(sorted(glob.glob(os.path.join(sim_dir, "particles", "particles_frame_*.bin")))[0])
        out["frame0_digest"] = np.array(cases.particle_digest(f0))
        if cases.particle_digest(c["particles"]) != str(out["frame0_digest"]):
            raise RuntimeError(f"{name}: numpy setup differs from the reference's initializeParticles")
        log = run_ref(cfg_path)
        nsteps = int([ln for ln in log.splitlines() if ln.startswith("Time step:")][-1].split()[2])
        out["nsteps"] = np.array(nsteps)
        for k in c["frames"]:
            P = O.read_particles_bin(_frame_file(sim_dir, k))
            for fld in O.PARTICLE_FIELDS:
                out[f"f{k}_{fld}"] = P[fld]
            out[f"f{k}_time"] = np.array(P["time"])
            out[f"f{k}_dt"] = np.array(P["dt"])
        hm, vm = O.read_max_bin(os.path.join(sim_dir, "max_values.bin"))
        idx = np.nonzero((hm != 0) | (vm != 0))
        out["max_idx"] = np.stack(idx, axis=1).astype(np.int32)
        out["max_h"] = hm[idx]
        out["max_v2"] = vm[idx]
        out["max_shape"] = np.array(hm.shape)
        run_ref(cfg_path, "--steps", str(max(PHASE_STEPS)))
        recs = O.read_steps_bin(os.path.join(sim_dir, "steps.bin"))
        for k in PHASE_STEPS:
            r = recs[k]
            out[f"s{k}_time"] = np.array(r["time"])
            out[f"s{k}_dt"] = np.array(r["dt"])
            for fld in ("x", "v", "h", "z", "vz"):
                out[f"s{k}_{fld}"] = r["particles"][fld]
            g = r["grid"]
            out[f"s{k}_grid_box"] = np.array([g["Nx"], g["Ny"], g["i_off"], g["j_off"]])
            for fld in ("mass", "h", "v", "flip", "vz"):
                out[f"s{k}_grid_{fld}"] = g[fld]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: Np={len(c['particles']['h'])} steps={nsteps} -> {name}.npz")


def _frame_file(sim_dir: str, k: int) -> str:
    for p in glob.glob(os.path.join(sim_dir, "particles", "particles_frame_*.bin")):
        if int(os.path.basename(p)[len("particles_frame_"):-4]) == k:
            return p
    raise FileNotFoundError(f"frame {k} in {sim_dir}")


def make_setup_poisson():
    """setup_poisson.json: sha256 of the reference's initial particles for
    every case with POISSON sampling (the reference's own sampler and
    std::rand), written by the reference binary's --init-only run."""
    out = {}
    for name in cases.CASES:
        c = cases.CASES[name]()
        with tempfile.TemporaryDirectory() as d:
            cfg_path = write_inputs(c, d)
            with open(cfg_path) as f:
                j = json.load(f)
            j["numerical_params"]["sampling_method"] = "POISSON"
            with open(cfg_path, "w") as f:
                json.dump(j, f, indent=1)
            run_ref(cfg_path, "--init-only")
            sim_dir = os.path.join(d, "out", c["name"])
            P = O.read_particles_bin(sorted(glob.glob(os.path.join(sim_dir, "particles", "particles_frame_*.bin")))[0])
            out[name] = {"Np": int(len(P["h"])), "digest": cases.particle_digest(P)}
    with open(os.path.join(HERE, "setup_poisson.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("setup_poisson.json:", {k: v["Np"] for k, v in out.items()})


BRIENZ_FRAMES = (1, 6)  # output frames (10 s apart) kept in the fixture


def make_brienz5m():
    """brienz5m.npz: the reference's own example (examples/brienz_raster.json)
    on its 5 m DEM and release raster, run to its 60 s end by the reference
    binary. Holds the DEM, the parameters, the reference's initial particles
    (POISSON sampling with std::rand seeded 1), its particle positions and
    heights at 10 s and 60 s, its final h_max / v_max2 and step count. The DEM keeps the
    file's nodata cells (-9999), which the reference does not mask."""
    root = os.environ.get("SLAB_REF_ROOT")
    if not root:
        sys.exit("set SLAB_REF_ROOT to the reference checkout")
    ex = os.path.join(root, "examples")
    with open(os.path.join(ex, "brienz_raster.json")) as f:
        j = json.load(f)
    out = {}
    with tempfile.TemporaryDirectory() as d:
        j["project_dir"] = os.path.join(d, "out")
        j["sim_name"] = "brienz5m"
        j["terrain"]["dem"]["filepath"] = os.path.join(ex, "brienz_terrain_5m.asc")
        j["release"]["raster"]["filepath"] = os.path.join(ex, "brienz_release_raster_5m.asc")
        cfg_path = os.path.join(d, "brienz5m.json")
        with open(cfg_path, "w") as f:
            json.dump(j, f)
        sim_dir = os.path.join(d, "out", "brienz5m")
        run_ref(cfg_path, "--init-only")
        P0 = O.read_particles_bin(sorted(glob.glob(os.path.join(sim_dir, "particles", "particles_frame_*.bin")))[0])
        for fld in O.PARTICLE_FIELDS:
            out[f"p0_{fld}"] = P0[fld]
        log = run_ref(cfg_path)
        out["nsteps"] = np.array(int([ln for ln in log.splitlines() if ln.startswith("Time step:")][-1].split()[2]))
        for k in BRIENZ_FRAMES:
            P = O.read_particles_bin(_frame_file(sim_dir, k))
            for fld in ("x", "h"):
                out[f"f{k}_{fld}"] = P[fld]
            out[f"f{k}_time"] = np.array(P["time"])
        hm, vm = O.read_max_bin(os.path.join(sim_dir, "max_values.bin"))
    z, hdr = W.read_asc(os.path.join(ex, "brienz_terrain_5m.asc"))
    out["z"] = z
    out["dx"] = np.array(hdr["cellsize"])
    idx = np.nonzero((hm != 0) | (vm != 0))
    out["max_idx"] = np.stack(idx, axis=1).astype(np.int32)
    out["max_h"] = hm[idx]
    out["max_v2"] = vm[idx]
    fr = j["friction"]["mu_I"]
    out["params"] = np.array([j["physical_params"]["gravity"], j["physical_params"]["rho"], j["numerical_params"]["C_cfl"],
                              j["numerical_params"]["dt_max"], j["numerical_params"]["flip_ratio"], j["time_params"]["output_dt"],
                              j["time_params"]["total_time"], fr["mu_1"], fr["mu_2"], fr["I0"], fr["d"], fr["phi"]])
    np.savez_compressed(os.path.join(HERE, "brienz5m.npz"), **out)
    print(f"brienz5m: Np={len(P0['h'])} steps={int(out['nsteps'])} DEM {z.shape} -> brienz5m.npz")


if __name__ == "__main__":
    if not os.path.exists(O.REF_BIN):
        sys.exit("oracle/_ref/slab_ref is not built (make -C oracle ref)")
    args = sys.argv[1:]
    if args == ["setup_poisson"]:
        make_setup_poisson()
    elif args == ["brienz5m"]:
        make_brienz5m()
    else:
        for n in (args or list(cases.CASES)):
            make(n)
