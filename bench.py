"""Benchmark of the depth-averaged MPM step loop on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c1|c3]

Default workload (c2): 4096^2 fractal-slope DEM at 1 m, star-polygon RASTER
release with lognormal heights, POISSON sampling at 0.5 m (665 653
particles), Voellmy friction -- all generated from fixed seeds (data:
synthetic). A "step" is one MPM time step (dt, P2G, grid update with
friction, G2P) of the whole scenario; the metric is particle-steps/s.

Our arm (--impl ours): the FP32 split-precision path through the C ABI
(libslab_gpu.so). The scenario is first advanced 2 s of simulated time
(untimed) so the flow is developed; then W warm-up steps and K timed steps,
each step bracketed by CUDA events on the library's stream, with a 256 MiB
write between steps to flush L2 (126 MB). Reported beside it: the plain
FP64 GPU path on the same state, per-kernel device times and the HBM
roofline of the dominant kernel, the reference CPU code on the same state
(cpu_baseline), and the end-to-end rate through the public API with host
buffers (e2e).

The reference arm (--impl reference) runs the reference's own step-loop
sources (oracle/_ref/slab_ref) on the box's host cores: one process per core
(up to 8), each on the same workload, timed by the reference's own per-phase
timers.

Multi-GPU: the single-scenario path does not shard; N ranks run N replicas
(scaling "weak"), value = all ranks' particle-steps / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "slab-pro_b200"))

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
METRIC = "particle-steps/s"
# algorithmic bytes of the FP32 split path (per particle-step, per active node-step)
BYTES_P, BYTES_N = 76, 124
KERNEL_BYTES = {  # per kernel: (bytes per particle-step, bytes per active node-step)
    "prep": (0, 0),  # tile descriptors: bookkeeping, no algorithmic bytes
    "p2g": (28, 28),
    "grid": (0, 76),
    "g2p": (48, 20),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_workload(name: str):
    """The named workload, generated with numpy only (no library of this
    repository is loaded, so the reference arm maps none)."""
    import workloads as W
    if name == "c1":
        return W.config1()
    if name == "c2":
        return W.config2()
    if name == "c3":
        return W.config3()
    if name == "c3s":
        return W.config3_small()
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                                          "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 3 + k and s[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def measured_peak():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def write_ref_inputs(c, P, d):
    """Binary DEM + particle files and a JSON for oracle/_ref/slab_ref."""
    import struct
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    dem = os.path.join(d, "dem.bin")
    with open(dem, "wb") as f:
        f.write(struct.pack("<qqd", c["z"].shape[0], c["z"].shape[1], c["dx"]))
        f.write(np.ascontiguousarray(c["z"], dtype=np.float64).tobytes())
    parts = os.path.join(d, "particles.bin")
    O.write_particles_bin(parts, P)
    return dem, parts


def ref_json(c, d, nsteps_time, output_dt=None):
    cfg = c["cfg"]
    fr = cfg["friction"]
    fj = {"type": fr}
    if fr == "COULOMB":
        fj["coulomb"] = {"mu": cfg["coulomb_mu"]}
    elif fr == "VOELLMY":
        fj["voellmy"] = {"mu": cfg["voellmy_mu"], "xi": cfg["voellmy_xi"]}
    else:
        fj["mu_I"] = {"mu_1": cfg["mui_mu1"], "mu_2": cfg["mui_mu2"], "I0": cfg["mui_I0"], "d": cfg["mui_d"], "phi": cfg["mui_phi"]}
    j = {"project_dir": os.path.join(d, "out"), "sim_name": "bench",
         "physical_params": {"gravity": cfg["gravity"], "rho": cfg["rho"]},
         "time_params": {"output_dt": output_dt or nsteps_time, "total_time": nsteps_time},
         "numerical_params": {"C_cfl": cfg["C_cfl"], "dt_max": cfg["dt_max"], "flip_ratio": cfg["flip_ratio"], "sampling_method": "UNIFORM"},
         "friction": fj,
         "terrain": {"type": "ANALYTICAL", "analytical": {"Lx": 8.0, "Ly": 8.0, "dx": c["dx"]}},
         "release": {"type": "RECTANGLE", "h0": 1.0, "rectangle": {"center": [4.0, 4.0], "Lx": 1.0, "Ly": 1.0, "rotation_deg": 0.0}}}
    path = os.path.join(d, f"cfg_{os.getpid()}_{len(os.listdir(d))}.json")
    with open(path, "w") as f:
        json.dump(j, f)
    return path


def run_reference(c, P, nsteps, replicas, warmup=0):
    """Run the reference binary `replicas` times concurrently from state P:
    `warmup` untimed steps, then about `nsteps` timed ones. Output frames are
    placed every `warmup` steps (or once, at the end); at each frame the
    binary prints the sum of the reference's own per-phase timers so far
    (SLAB_REF_FRAME_TIMERS, oracle/ref_hooks.cpp) and the step count, and the
    timed part is what lies between the first frame after the warm-up (t=0
    without one) and the last frame. Returns (particle-steps/s aggregate,
    timed steps of one replica, seconds of the slowest replica)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not os.path.exists(O.REF_BIN):
        raise RuntimeError("oracle/_ref/slab_ref not built")
    dt_max = c["cfg"]["dt_max"]
    if warmup > 0:
        nsteps = -(-nsteps // warmup) * warmup  # whole frames after the warm-up
    T = (warmup + nsteps) * dt_max
    with tempfile.TemporaryDirectory() as d:
        dem, parts = write_ref_inputs(c, P, d)
        procs = []
        for r in range(replicas):
            cfg = ref_json(c, d, T, output_dt=warmup * dt_max if warmup > 0 else None)
            env = dict(os.environ, SLAB_REF_NO_DUMP="1", SLAB_REF_FRAME_TIMERS="1")
            procs.append(subprocess.Popen([O.REF_BIN, cfg, "--dem-bin", dem, "--particles", parts], stdout=subprocess.PIPE,
                                          stderr=subprocess.PIPE, text=True, env=env))
        secs, steps = [], []
        for p in procs:
            out, err = p.communicate()
            if p.returncode != 0:
                raise RuntimeError(f"slab_ref failed: {err.strip()[-300:]}")
            marks, pending = [], None  # (step count, phase seconds so far) per output frame
            for ln in out.splitlines():
                if ln.startswith("Phase seconds so far:"):
                    pending = float(ln.split()[-1])
                elif ln.startswith("Time step:") and pending is not None:
                    marks.append((int(ln.split()[2]), pending))
                    pending = None
            first = 1 if warmup > 0 else 0
            if len(marks) < first + 2:
                raise RuntimeError(f"slab_ref printed {len(marks)} frames")
            (n0, s0), (n1, s1) = marks[first], marks[-1]
            steps.append(n1 - n0)
            secs.append(s1 - s0)
    Np = len(P["h"])
    tmax = max(secs)
    if min(steps) <= 0 or tmax <= 0:
        raise RuntimeError("no timed reference steps")
    return sum(steps) * Np / tmax, steps[0], tmax


def record_run(z, dx, cfg, P, prec, stream, perturb=0.0, seed=0):
    """One scenario from t=0 to total_time through a context, frame by frame:
    the FP64 centre of mass at t=0 and at every output frame (slab_moments),
    the h_max and max-speed maps over the wet box, the total particle mass at
    the start and the end, steps and wall seconds. perturb > 0 moves every
    starting position by a seeded uniform offset of up to perturb * dx in
    each coordinate (the FP64 sensitivity envelope)."""
    import slab
    import accuracy as Acc
    if perturb > 0.0:
        rng = np.random.default_rng(seed)
        P = dict(P, x=P["x"] + dx * perturb * rng.uniform(-1.0, 1.0, P["x"].shape))
    s = slab.Slab(z, dx)
    s.set_stream(stream.cuda_stream)
    s.set_params(cfg, prec)
    w0 = time.perf_counter()
    s.upload(P)
    s.initial_pass()
    m0 = s.moments()
    com, steps = [m0["com"]], 0
    while True:
        t, _, k = s.advance_to_frame()
        steps += k
        mo = s.moments()
        com.append(mo["com"])
        if t >= cfg["total_time"] or k == 0:
            break
    hm, vm = s.max_maps()
    wall = time.perf_counter() - w0
    s.close()
    box = Acc.wet_box(hm)
    crop = (lambda m: m[box[0]:box[1] + 1, box[2]:box[3] + 1].copy()) if box[1] >= box[0] else (lambda m: np.zeros((0, 0)))
    return {"box": box, "h_max": crop(hm), "v_max": np.sqrt(crop(vm)), "com": np.array(com), "mass": m0["mass"],
            "mass_end": mo["mass"], "steps": steps, "wall_s": wall}


def accuracy_block(z, dx, cfg, P, stream, envelope=True):
    """FP32_SPLIT against FP64_PLAIN over a whole run of one scenario, and
    beside it the FP64 envelope: FP64_PLAIN against FP64_PLAIN started from
    positions moved by up to 1e-7 dx (the resolution of the FP32 split
    position)."""
    import slab
    import accuracy as Acc
    r64 = record_run(z, dx, cfg, P, slab.FP64_PLAIN, stream)
    r32 = record_run(z, dx, cfg, P, slab.FP32_SPLIT, stream)
    out = {"fp32_vs_fp64": Acc.compare_runs(r32, r64, dx),
           "steps": {"fp64": r64["steps"], "fp32": r32["steps"]},
           "mass_drift_rel": {"fp64": abs(r64["mass_end"] - r64["mass"]) / r64["mass"],
                              "fp32": abs(r32["mass_end"] - r32["mass"]) / r32["mass"]},
           "wall_s": {"fp64": round(r64["wall_s"], 2), "fp32": round(r32["wall_s"], 2)}}
    if envelope:
        rp = record_run(z, dx, cfg, P, slab.FP64_PLAIN, stream, perturb=1e-7, seed=11)
        out["fp64_envelope"] = Acc.compare_runs(rp, r64, dx)
    return out


def ours(args, rank, world):
    import torch
    import slab

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    if args.only in ("ensemble", "serving", "e2e_cli"):
        if rank != 0:
            return None
        sec = {"ensemble": lambda: ensemble(args, stream, dev), "serving": lambda: serving(args, stream, dev),
               "e2e_cli": lambda: e2e_cli(args)}[args.only]()
        return {"section": args.only, args.only: sec}
    c = load_workload(args.workload)
    P0 = c["particles"]
    Np = len(P0["h"])
    cfg = dict(c["cfg"], output_dt=c["cfg"]["total_time"])  # no frame stops inside the timed region
    log(f"[rank {rank}] workload {c['name']}: Np={Np} DEM {c['z'].shape} dx={c['dx']}")

    def make(prec):
        s = slab.Slab(c["z"], c["dx"])
        s.set_stream(stream.cuda_stream)
        s.set_params(cfg, prec)
        s.upload(P0)
        s.initial_pass()
        return s

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(s, K, profile=False):
        if profile:
            s.set_profiling(True)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        w0 = s.work_counters()
        l0 = s.kernel_launches()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            for k in range(K):
                flush.zero_()
                ev[k][0].record(stream)
                s.advance_steps_async(1)
                ev[k][1].record(stream)
        s.synchronize()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        if world > 1:
            torch.distributed.barrier()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        w1 = s.work_counters()
        phases = None
        if profile:
            phases = s.phase_times()
            s.set_profiling(False)
        return ms, wall, (w1[0] - w0[0], w1[1] - w0[1]), s.kernel_launches() - l0, phases

    def spin_to(s, t_target):
        """advance until the simulated time reaches t_target (developed flow)"""
        while s.state()[0] < t_target - 1e-9:
            if s.advance_steps(max(1, int(round((t_target - s.state()[0]) / cfg["dt_max"])))) == 0:
                break

    def e2e_block():
        """The same metric through the public API from pinned FP64 host
        arrays: upload, t=0 pass, K steps, particle and max-map download."""
        K_e2e = args.e2e_steps

        def pinned(n):  # page-locked host memory, allocated before the timed region
            return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()

        hb = {}
        for k in ("x", "v", "vz", "h", "A", "mass", "z"):
            a = np.ascontiguousarray(P0[k], dtype=np.float64)
            hb[k] = pinned(a.size).reshape(a.shape)
            hb[k][...] = a
        ob = {k: pinned(hb[k].size) for k in hb}
        mb = (pinned(c["z"].size), pinned(c["z"].size))
        e = slab.Slab(c["z"], c["dx"])
        e.set_stream(stream.cuda_stream)
        e.set_params(cfg, slab.FP32_SPLIT)
        e2e_runs = []
        for it in range(2):
            torch.cuda.synchronize()
            tt = [time.perf_counter()]
            e.upload(hb)
            tt.append(time.perf_counter())
            e.initial_pass()
            tt.append(time.perf_counter())
            e.advance_steps(K_e2e)
            tt.append(time.perf_counter())
            out = e.particles(out=ob)
            tt.append(time.perf_counter())
            hmx, _ = e.max_maps(out=mb)
            tt.append(time.perf_counter())
            e2e_runs.append(tt)
        best = min(e2e_runs, key=lambda tt: tt[-1] - tt[0])
        h2d = sum(hb[k].nbytes for k in hb)
        d2h = sum(out[k].nbytes for k in out) + 2 * hmx.nbytes
        e2e = {"value": round(Np * K_e2e / (best[-1] - best[0]), 1), "unit": METRIC,
               "h2d_bytes_per_step": int(h2d / K_e2e), "d2h_bytes_per_step": int(d2h / K_e2e),
               "phases_s": {name: round(best[q + 1] - best[q], 4)
                            for q, name in enumerate(("upload", "t0_pass", "steps", "particles_download", "max_maps_download"))},
               "window": f"upload + t=0 pass + {K_e2e} steps + particle and max-map download, host FP64 arrays in pinned memory "
                         f"allocated before the timed region, best of 2; d2h counts the host arrays returned (the library copies "
                         f"only the node box the flow touched of the max maps)"}
        e.close()
        del hmx, out, ob, mb, hb
        return e2e

    # ---- FP32 split path (the product): W warm-up steps from the workload's
    # initial state, then K timed steps -- the state the reference arm times
    # the end-to-end run comes first: its first steps tune the launch shapes,
    # which the library keeps for later contexts of the same size, so the
    # timed steps below run on tuned shapes (the tuner's trial shapes would
    # otherwise fall inside the timed window)
    e2e = e2e_block()
    s32 = make(slab.FP32_SPLIT)
    s32.advance_steps(args.warmup)
    with ClockSampler(dev) as clk:
        ms, wall, work, launches, _ = timed(s32, args.steps)
    assert work[0] == Np * args.steps, work
    ms_prof, _, work_prof, _, phases = timed(s32, args.steps, profile=True)
    shapes, tunes = s32.launch_shapes()
    # the same after the flow has developed (spin-up to args.spinup simulated seconds)
    spin_to(s32, args.spinup)
    ms_dev, _, work_dev, _, phases_dev = timed(s32, args.steps, profile=True)
    t32 = s32.state()[0]
    s32.close()
    if args.only == "fp32":
        if rank == 0:
            return {"metric": METRIC, "value": round(Np * args.steps / (ms * 1e-3), 1), "unit": METRIC, "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5),
                    "config": {"workload": c["name"], "particles": Np, "only": "fp32"},
                    "phases_ms": [round(p / args.steps, 5) for p in phases],
                    "developed": {"sim_time_s": round(t32, 3), "ms_per_step": round(ms_dev / args.steps, 5),
                                  "phases_ms": [round(p / args.steps, 5) for p in phases_dev],
                                  "active_nodes_per_step": work_dev[1] / args.steps},
                    "active_nodes_per_step": work_prof[1] / args.steps, "gpu_launches": int(launches),
                    "e2e": e2e}
        return None

    # ---- plain FP64 path on the same schedule
    s64 = make(slab.FP64_PLAIN)
    s64.advance_steps(args.warmup)
    ms64, _, work64, _, _ = timed(s64, args.steps)
    spin_to(s64, args.spinup)
    ms64_dev, _, _, _, _ = timed(s64, args.steps)
    s64.close()

    # ---- max over ranks
    step_ms = ms / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_all = float(t.item())
    else:
        ms_all = ms
    value = Np * args.steps * world / (ms_all * 1e-3)
    sharded = None
    if world > 1 and not args.no_ensemble:  # every rank takes part (the same collective steps on all ranks)
        sharded = ensemble_sharded(args, stream, dev, rank, world)
    if rank != 0:
        return None

    # ---- roofline of the dominant kernel (profiled pass, same state)
    peak, peak_kind = measured_peak()
    names = {1: "prep", 2: "p2g", 3: "grid", 4: "g2p"}

    def per_kernel_of(ph, wk):
        nodes = wk[1] / args.steps
        out = {}
        for idx, nm in names.items():
            t_ms = ph[idx] / args.steps
            bp, bn = KERNEL_BYTES[nm]
            bytes_launch = bp * Np + bn * nodes
            out[nm] = {"ms": round(t_ms, 5), "algorithmic_bytes": int(bytes_launch),
                       "gbs": round(bytes_launch / (t_ms * 1e-3) / 1e9, 1) if t_ms > 0 else None,
                       "share": round(ph[idx] / max(sum(ph), 1e-12), 3)}
        return out, nodes

    per_kernel, nodes_per_step = per_kernel_of(phases, work_prof)
    dom = max(("p2g", "grid", "g2p"), key=lambda k: per_kernel[k]["ms"])
    ach = per_kernel[dom]["gbs"]
    traffic = None
    tp = os.path.join(ROOT, "profiles", f"traffic_{args.workload}.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4) if ach else None, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s", "traffic": traffic,
                "whole_step": {"algorithmic_bytes": int(BYTES_P * Np + BYTES_N * nodes_per_step),
                               "gbs": round((BYTES_P * Np + BYTES_N * nodes_per_step) / (step_ms * 1e-3) / 1e9, 1)},
                "per_kernel": per_kernel, "active_nodes_per_step": round(nodes_per_step, 1)}
    pk_dev, nodes_dev = per_kernel_of(phases_dev, work_dev)

    # ---- CPU baseline: the reference's own step loop, 1 core, same state
    cpu = None
    if not args.no_cpu:
        try:
            Pref = dict(P0)
            k_cpu = max(3, int(args.cpu_seconds * 8e6 / Np))
            v_cpu, st_cpu, sec_cpu = run_reference(c, Pref, k_cpu, 1, warmup=args.warmup)
            cpu = {"value": round(v_cpu, 1), "unit": METRIC, "cores": 1, "kind": "reference",
                   "sample": f"{st_cpu} steps after {args.warmup} warm-up steps from the workload's initial state, "
                             f"{Np} particles, reference step-loop sources (oracle/_ref/slab_ref), per-phase timers, {sec_cpu:.1f} s"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": METRIC, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}


    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_all / args.steps, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (f64 dt, time, metric terms, sums)", "data": "synthetic",
        "config": {"workload": c["name"], "particles": Np, "dem": list(c["z"].shape), "dx": c["dx"],
                   "friction": c["cfg"]["friction"], "state": f"{args.warmup} warm-up steps from the initial state",
                   "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "fp64_plain": {"value": round(Np * args.steps / (ms64 * 1e-3), 1), "ms_per_step": round(ms64 / args.steps, 5),
                       "fp32_speedup": round(ms64 / ms, 2)},
        "developed": {"sim_time_s": round(t32, 3), "value": round(Np * args.steps / (ms_dev * 1e-3), 1),
                      "ms_per_step": round(ms_dev / args.steps, 5), "fp64_plain_ms_per_step": round(ms64_dev / args.steps, 5),
                      "fp32_speedup": round(ms64_dev / ms_dev, 2), "active_nodes_per_step": round(nodes_dev, 1),
                      "per_kernel": pk_dev},
        "gpu_launches": int(launches),
        "launch_shapes": {"ctas": dict(zip(("prep", "p2g_dense", "p2g_sparse", "grid", "g2p"), shapes)), "tuning_passes": tunes,
                          "source": "picked on the e2e run's first steps of the same workload size, kept by the library for the process"},
        "clocks": clocks,
        "wall_s_timed": round(wall, 4),
    }
    if world == 1 and not args.no_accuracy:
        try:
            acc = accuracy_block(c["z"], c["dx"], c["cfg"], P0, stream, envelope=not args.no_envelope)
            line["accuracy"] = dict(acc, workload=c["name"])
        except Exception as ex:
            line["accuracy"] = {"error": f"{type(ex).__name__}: {ex}"}
        if args.workload != "c2" and not args.no_c2_accuracy:
            try:
                c2 = load_workload("c2")
                line["accuracy_c2"] = dict(accuracy_block(c2["z"], c2["dx"], c2["cfg"], c2["particles"], stream), workload=c2["name"],
                                           particles=len(c2["particles"]["h"]))
            except Exception as ex:
                line["accuracy_c2"] = {"error": f"{type(ex).__name__}: {ex}"}
    if world == 1 and not args.no_e2e_cli:
        try:
            line["e2e_cli"] = e2e_cli(args)
        except Exception as ex:
            line["e2e_cli"] = {"error": f"{type(ex).__name__}: {ex}"}
    if world == 1 and not args.no_ensemble and args.only != "serving":
        try:
            line["ensemble"] = ensemble(args, stream, dev)
        except Exception as e:  # reported in the line, the headline stands
            line["ensemble"] = {"error": f"{type(e).__name__}: {e}"}
    if world > 1 and not args.no_ensemble:
        line["ensemble_sharded"] = sharded
    if world == 1 and not args.no_serving and args.only != "ensemble":
        try:
            line["serving"] = serving(args, stream, dev)
        except Exception as e:
            line["serving"] = {"error": f"{type(e).__name__}: {e}"}
    return line


def _stratified(keys, k):
    """k indices spread evenly over the order of keys (the middle of each of k strata)."""
    order = np.argsort(np.asarray(keys), kind="stable")
    n = len(order)
    k = max(1, min(k, n))
    return [int(order[(2 * q + 1) * n // (2 * k)]) for q in range(k)]


def _solo_run(s, cfg, P, prec, stream):
    """One scenario alone through a context: (device seconds of the t=0 pass
    and the step loop, wall seconds from upload to max maps on the host, steps,
    h_max, v_max2). P is the particles or a release built on the device."""
    import torch
    import slab
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    s.set_params(cfg, prec)
    if "type" in P:  # a release, built on the device
        s.upload_release(P)
    else:
        s.upload(P)
    e0.record(stream)
    s.initial_pass()
    n = s.advance_steps(1 << 40)
    e1.record(stream)
    hm, vm = s.max_maps()
    wall = time.perf_counter() - w0
    return e0.elapsed_time(e1) * 1e-3, wall, n, hm, vm


def release_host_particles(z, dx, cfg, rel, stream):
    """The particles of a release as FP64 host arrays: built on the device
    (the reference's setup, bit for bit) and read back through the FP64 path,
    which keeps the uploaded doubles."""
    import slab
    s = slab.Slab(z, dx)
    s.set_stream(stream.cuda_stream)
    s.set_params(cfg, slab.FP64_PLAIN)
    s.upload_release(rel)
    P = s.particles()
    s.close()
    return P


def ensemble(args, stream, dev):
    """Batched ensemble: config-4 scenarios on a shared 2048^2 DEM, all in one
    Batch (FP32 split), against the same scenarios one after another through
    the plain FP64 path (a stratified sample of them, timed in full)."""
    import torch
    import slab
    import workloads as W
    import accuracy as Acc
    g0 = time.perf_counter()
    c = W.config4(args.c4_scenarios, particles=False)  # releases: the particles are built on the device
    gen_s = time.perf_counter() - g0
    z, dx, scen = c["z"], c["dx"], c["scenarios"]
    n = len(scen)
    b = slab.Batch(z, dx, n)
    b.set_stream(stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for cfg, rel in scen:
        b.add_release(cfg, rel)
    w_add = time.perf_counter()
    Nps = np.array(b.Np)
    out = {"workload": c["name"], "scenarios": n, "particles": int(Nps.sum()), "particles_min_max": [int(Nps.min()), int(Nps.max())],
           "generate_s": round(gen_s, 1), "setup": "RELEASE ellipses built on the device (slab_batch_add_release), UNIFORM 2x2"}
    l0 = b.kernel_launches()
    run_err = None
    with ClockSampler(dev) as clk:
        e0.record(stream)
        try:
            b.run()
        except slab.SlabError as e:  # failed scenarios stop; the others run to the end
            run_err = str(e)
        e1.record(stream)
        e1.synchronize()
    w_run = time.perf_counter()
    status = [b.scenario_status(i) for i in range(n)]
    ok = [i for i in range(n) if status[i] == 0]
    boxes = {i: b.max_box(i) for i in ok}
    w_dl = time.perf_counter()
    run_s = e0.elapsed_time(e1) * 1e-3
    ps, ns = b.work_counters()
    steps = np.array([b.state(i)[2] for i in ok] or [0])
    out["fp32_batched"] = {
        "completed": len(ok), "failed": n - len(ok), "first_error": run_err,
        "scenarios_per_s": round(len(ok) / run_s, 3), "particle_steps_per_s": round(ps / run_s, 1), "device_s": round(run_s, 3),
        "e2e_scenarios_per_s": round(len(ok) / (w_dl - w0), 3), "e2e_s": round(w_dl - w0, 3), "add_s": round(w_add - w0, 3),
        "download_s": round(w_dl - w_run, 3), "particle_steps": int(ps), "active_node_steps": int(ns),
        "steps_min_max": [int(steps.min()), int(steps.max())], "gpu_launches": int(b.kernel_launches() - l0),
        "clocks": clk.summary()}
    b_results = boxes
    b.close()
    # the same scenarios one after another (a sample of the completed ones, stratified by particle count)
    pick = [ok[q] for q in _stratified(Nps[ok], args.c4_sample)] if ok else []
    full = [0, z.shape[0] - 1, 0, z.shape[1] - 1]
    seq = {}
    for prec, name in ((slab.FP64_PLAIN, "fp64_sequential"), (slab.FP32_SPLIT, "fp32_sequential")):
        s = slab.Slab(z, dx)
        s.set_stream(stream.cuda_stream)
        dev_s, wall_s, acc, same, nrun = 0.0, 0.0, [], True, 0
        for i in pick:
            cfg, P = scen[i]
            try:
                d, w, k, hm, _ = _solo_run(s, cfg, P, prec, stream)
            except slab.SlabError:
                continue
            nrun += 1
            dev_s += d
            wall_s += w
            box, hb, _ = b_results[i]
            wb = Acc.wet_box(hm)
            if prec == slab.FP64_PLAIN:
                acc.append(Acc.compare_max_heights(box, hb, wb, Acc.crop(full, hm, wb), dx))
            else:
                same &= bool(np.array_equal(Acc.crop(full, hm, box), hb)) if box[1] >= box[0] else not (hm > 0).any()
        s.close()
        seq[name] = {"scenarios_per_s": round(nrun / max(dev_s, 1e-9), 3), "e2e_scenarios_per_s": round(nrun / max(wall_s, 1e-9), 3),
                     "sample": len(pick), "completed": nrun, "device_s": round(dev_s, 3), "wall_s": round(wall_s, 3)}
        if acc:
            seq[name]["accuracy_of_batched_fp32"] = {
                "min_within_1cm_1pct": round(min(a["within_1cm_1pct"] for a in acc), 5),
                "max_abs_m": round(max(a["max_abs_m"] for a in acc), 4),
                "max_runout_diff_m": max(a["runout_diff_m"] for a in acc), "dx": dx}
        else:
            seq[name]["batched_equals_alone_bitwise"] = same
    out.update(seq)
    # whole-run accuracy with the FP64 envelope on a stratified sample (the batch gives each
    # scenario the bits of its solo FP32 run, checked above)
    if args.c4_acc_sample > 0 and ok:
        import accuracy as Acc2
        rows32, rows_env = [], []
        for i in [ok[q] for q in _stratified(Nps[ok], args.c4_acc_sample)]:
            cfg, rel = scen[i]
            try:
                a = accuracy_block(z, dx, cfg, release_host_particles(z, dx, cfg, rel, stream), stream)
            except slab.SlabError:
                continue
            rows32.append(a["fp32_vs_fp64"])
            rows_env.append(a["fp64_envelope"])
        out["accuracy"] = {"scenarios": len(rows32), "fp32_vs_fp64": Acc2.summarize(rows32), "fp64_envelope": Acc2.summarize(rows_env),
                           "note": "worst case over the sample; fp64_envelope: FP64 against FP64 started from positions moved by "
                                   "up to 1e-7 dx"}
    f64 = seq["fp64_sequential"]
    out["speedup_vs_fp64_sequential"] = {"device": round(out["fp32_batched"]["scenarios_per_s"] / f64["scenarios_per_s"], 2),
                                         "e2e": round(out["fp32_batched"]["e2e_scenarios_per_s"] / f64["e2e_scenarios_per_s"], 2)}
    out["note"] = ("scenarios/s: completed scenarios / device time of one batched run; sequential rates are the mean over a "
                   "sample of the completed scenarios stratified by particle count, each run in full (t=0 pass to total_time); "
                   "e2e includes the device setup of every release, binning and max-map downloads; a scenario whose flow leaves the "
                   "terrain fails")
    return out


def ensemble_sharded(args, stream, dev, rank, world):
    """The config-4 ensemble sharded by scenario over the ranks (one GPU
    each): every rank runs its share (shard.assign, balanced by particles x
    simulated time) as one batch; no collective touches the data path. The
    host gathers the per-rank counts and device times; scenarios/s = all
    completed scenarios / the slowest rank's device time."""
    import torch
    import torch.distributed as dist
    import slab
    import shard
    import workloads as W
    c = W.config4(args.c4_scenarios, particles=False)
    scen = c["scenarios"]
    est = [W.release_particle_estimate(rel, c["dx"]) for _, rel in scen]
    shards = shard.assign([est[i] * cfg["total_time"] for i, (cfg, _) in enumerate(scen)], world,
                          [shard.footprint_bytes(e) for e in est])
    mine = shards[rank]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ok, ps, err, dev_s = 0, 0, None, 0.0
    try:  # a failure here still takes part in the collectives below
        b = slab.Batch(c["z"], c["dx"], max(1, len(mine)))
        b.set_stream(stream.cuda_stream)
        for i in mine:
            b.add_release(*scen[i])
    except Exception as ex:
        b, err = None, f"{type(ex).__name__}: {ex}"
    dist.barrier()
    if b is not None:
        e0.record(stream)
        try:
            b.run()
        except slab.SlabError:
            pass
        e1.record(stream)
        e1.synchronize()
        dev_s = e0.elapsed_time(e1) * 1e-3
        ok = sum(1 for k in range(len(mine)) if b.scenario_status(k) == 0)
        ps, _ = b.work_counters()
        b.close()
    t = torch.tensor([dev_s, float(ok), float(ps), float(len(mine)), 1.0 if err else 0.0], device="cuda", dtype=torch.float64)
    tmax = t[0:1].clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    if rank != 0:
        return None
    return {"workload": c["name"], "ranks": world, "scenarios": len(scen), "completed": int(t[1].item()),
            "scenarios_per_s": round(t[1].item() / tmax.item(), 3), "particle_steps_per_s": round(t[2].item() / tmax.item(), 1),
            "slowest_rank_device_s": round(tmax.item(), 3), "scenarios_per_rank": [len(x) for x in shards],
            "ranks_failed": int(t[4].item()), "rank0_error": err,
            "scaling": "strong (the same 256 scenarios split over the ranks)"}


def e2e_cli(args):
    """End to end through the drop-in program, as a reference user runs it:
    `bin/slab_b200 <config.json>` (loadFromJSON, initialize, DEM read,
    POISSON setup on the host, simulate with the step loop on the GPU and
    every output frame written as .ply / .tif by the writer thread while the
    GPU runs on, max_values.tif) on a window of the config-2 construction
    (512 x 512 DEM at 1 m, raster release, Voellmy, 40 s, a frame every
    second), beside the reference's own step loop on the same JSON
    (oracle/_ref/slab_ref, its output writers stubbed, one host core).
    Rates are particle-steps per second of wall time, setup included."""
    import workloads as W
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cli = os.path.join(ROOT, "slab-pro_b200", "bin", "slab_b200")
    dx = 1.0
    z = W.fractal_slope_dem(512, dx, seed=2026, rms=4.0, x_plane_end=300.0, ease_m=100.0, rim_m=40.0)
    poly = W.star_polygon(2027, center=(110.0, 256.0), ax=70.0, ay=45.0)
    rel = W.lognormal_release_raster(2028, poly, cellsize=dx)
    out = {"workload": "c2_window512_dx1_star_raster_poisson_voellmy_40s"}
    with tempfile.TemporaryDirectory() as d:
        W.write_asc(os.path.join(d, "dem.asc"), z, dx)
        W.write_asc(os.path.join(d, "release.asc"), rel["h"], rel["cellsize"], xll=rel["x0"], yll=rel["y0"])
        j = {"project_dir": os.path.join(d, "out"), "sim_name": "e2e",
             "physical_params": {"gravity": 9.81, "rho": 300.0}, "time_params": {"output_dt": 1.0, "total_time": 40.0},
             "numerical_params": {"C_cfl": 0.5, "dt_max": 0.01, "flip_ratio": 0.95, "sampling_method": "POISSON"},
             "friction": {"type": "VOELLMY", "voellmy": {"mu": 0.2, "xi": 1500.0}},
             "terrain": {"type": "DEM", "dem": {"filepath": os.path.join(d, "dem.asc")}},
             "release": {"type": "RASTER", "h0": 0.0, "raster": {"filepath": os.path.join(d, "release.asc"), "h_min": 0.2}}}
        cfg = os.path.join(d, "e2e.json")
        with open(cfg, "w") as f:
            json.dump(j, f)

        def timed_run(cmd, env=None):
            t0 = time.perf_counter()
            r = subprocess.run(cmd, capture_output=True, text=True, env=env)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError(f"{os.path.basename(cmd[0])} failed: {r.stderr.strip()[-300:]}")
            return r.stdout, wall

        subprocess.run([cli, cfg, "--no-output"], capture_output=True)  # DEM cache and first-use costs outside the timings
        for label, extra in (("fp32_outputs", []), ("fp32_no_output", ["--no-output"]), ("fp64_outputs", ["--fp64"])):
            txt, wall = timed_run([cli, cfg] + extra)
            np_ = int([ln for ln in txt.splitlines() if ln.startswith("Number of particles:")][-1].split()[-1])
            steps = int([ln for ln in txt.splitlines() if ln.startswith("Simulation finished:")][-1].split()[2])
            out[label] = {"wall_s": round(wall, 3), "particles": np_, "steps": steps, "particle_steps_per_s": round(np_ * steps / wall, 1)}
        nfiles = len(os.listdir(os.path.join(d, "out", "e2e", "particles"))) if os.path.isdir(os.path.join(d, "out", "e2e", "particles")) else 0
        out["fp32_outputs"]["frames_written"] = nfiles
        if os.path.exists(O.REF_BIN) and not args.no_cpu:
            txt, wall = timed_run([O.REF_BIN, cfg], env=dict(os.environ, SLAB_REF_NO_DUMP="1"))
            steps = int([ln for ln in txt.splitlines() if ln.startswith("Time step:")][-1].split()[2])
            np_ = int([ln for ln in txt.splitlines() if ln.startswith("Number of particles:")][-1].split()[-1])
            out["reference_cpu"] = {"wall_s": round(wall, 3), "particles": np_, "steps": steps, "cores": 1,
                                    "particle_steps_per_s": round(np_ * steps / wall, 1),
                                    "note": "the reference's step loop with its output writers stubbed (no files)"}
            out["speedup_fp32_outputs_vs_reference"] = round(out["fp32_outputs"]["particle_steps_per_s"] /
                                                             out["reference_cpu"]["particle_steps_per_s"], 2)
    return out


def _serve(srv, reqs, arrivals, dev):
    """Submit every request (a release, built on the device when admitted) at
    its arrival time, replayed in real time; drain; per-request time to
    result and steps, and the server's figures."""
    import slab
    ids, late = [], 0.0
    with ClockSampler(dev) as clk:
        t_start = time.perf_counter()
        for ta, (_, cfg, rel) in zip(arrivals, reqs):
            now = time.perf_counter() - t_start
            if ta > now:
                time.sleep(ta - now)
            late = max(late, time.perf_counter() - t_start - ta)
            ids.append(srv.submit_release(cfg, rel))
        srv.drain(timeout=1800.0)
        t_end = time.perf_counter()
    st, tm = srv.stats(), srv.timing()
    ttr, ok = [], 0
    for rid in ids:
        state, secs = srv.poll(rid)
        if state == slab.REQ_DONE:
            ttr.append(secs)
            ok += 1
    ttr = np.array(ttr) if ttr else np.array([np.nan])
    span = t_end - t_start
    return {"completed": ok, "failed": len(ids) - ok, "p50_s": round(float(np.percentile(ttr, 50)), 3),
            "p99_s": round(float(np.percentile(ttr, 99)), 3), "scenarios_per_s": round(ok / span, 3),
            "particle_steps_per_s": round(st["particle_steps"] / span, 1), "makespan_s": round(span, 3),
            "busy_s": round(st["busy_s"], 3), "saturation_scenarios_per_s": round(ok / max(st["busy_s"], 1e-9), 3),
            "max_submit_lateness_s": round(late, 4), "worker": {k: round(v, 3) for k, v in tm.items()}, "clocks": clk.summary()}


def _fifo(arrivals, service):
    """Times to result of a FIFO queue of one server with these service times."""
    t, fin = 0.0, np.empty(len(arrivals))
    for q in range(len(arrivals)):
        t = max(t, arrivals[q]) + service[q]
        fin[q] = t
    lat = fin - np.asarray(arrivals)
    return {"p50_s": round(float(np.percentile(lat, 50)), 3), "p99_s": round(float(np.percentile(lat, 99)), 3),
            "scenarios_per_s": round(len(arrivals) / (fin[-1] - arrivals[0]), 3), "busy_s": round(float(np.sum(service)), 3)}


def serving(args, stream, dev):
    """Served request stream (config 5): Poisson arrivals at 20/s on the
    config-3 DEM into the continuous-batching server; each request is an
    ELLIPSE release whose particles are built on the device when it is
    admitted. Against it, every request of the same window runs alone
    through the plain FP64 path (each one's device time measured, release
    built on the device as well), and those service times are replayed as a
    FIFO queue on the same arrival times. The stream is replayed twice: at
    its own rate (20/s, more than either path sustains), and at 70 % of the
    rate the FP32 server sustains, where times to result are not queueing."""
    import torch
    import slab
    import workloads as W
    g0 = time.perf_counter()
    dx = 0.5
    z = W.config3_dem()
    reqs = W.config5_stream(z, dx, args.c5_window, particles=False)
    gen_s = time.perf_counter() - g0
    n = len(reqs)
    arr = np.array([t for t, _, _ in reqs])
    out = {"workload": f"poisson20/s_window{args.c5_window:g}s_fractal8192_dx0.5", "requests": n, "window_s": args.c5_window,
           "window_note": f"the first {args.c5_window:g} s of the 300 s stream", "generate_s": round(gen_s, 1)}
    srv = slab.Server(z, dx, max_scenarios=args.c5_slots, chunk_steps=32)
    out["fp32_served"] = _serve(srv, reqs, arr, dev)
    srv.close()
    # plain FP64, every request alone
    s = slab.Slab(z, dx)
    s.set_stream(stream.cuda_stream)
    svc, nps, fails = np.zeros(n), np.zeros(n), 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    for q, (_, cfg, rel) in enumerate(reqs):
        s.set_params(cfg, slab.FP64_PLAIN)
        try:
            e0.record(stream)
            nps[q] = s.upload_release(rel)
            s.initial_pass()
            s.advance_steps(1 << 40)
            e1.record(stream)
            e1.synchronize()
            svc[q] = e0.elapsed_time(e1) * 1e-3
        except slab.SlabError:
            fails += 1
            torch.cuda.synchronize()
    s.close()
    f64 = {"requests_run": n, "failed": fails, "particles": int(nps.sum()), "device_s": round(float(svc.sum()), 3),
           "wall_s": round(time.perf_counter() - w0, 1), "saturation_scenarios_per_s": round((n - fails) / max(svc.sum(), 1e-9), 3)}
    f64.update(_fifo(arr, svc))
    out["fp64_sequential"] = f64
    fs = out["fp32_served"]
    out["speedup_vs_fp64_sequential"] = {"scenarios_per_s": round(fs["scenarios_per_s"] / f64["scenarios_per_s"], 2),
                                         "saturation": round(fs["saturation_scenarios_per_s"] / max(f64["saturation_scenarios_per_s"], 1e-9), 2),
                                         "p50": round(f64["p50_s"] / fs["p50_s"], 2), "p99": round(f64["p99_s"] / fs["p99_s"], 2)}
    # the same requests at 70 % of the rate the FP32 server sustains
    rate = 0.7 * fs["saturation_scenarios_per_s"]
    if args.c5_sustained and rate > 0:
        arr2 = (arr - arr[0]) * (20.0 / rate)
        srv = slab.Server(z, dx, max_scenarios=args.c5_slots, chunk_steps=32)
        sus = _serve(srv, reqs, arr2, dev)
        srv.close()
        f2 = _fifo(arr2, svc)
        out["sustained"] = {"arrivals_per_s": round(rate, 3), "fp32_served": sus, "fp64_sequential": f2,
                            "speedup_vs_fp64_sequential": {"p50": round(f2["p50_s"] / sus["p50_s"], 2),
                                                           "p99": round(f2["p99_s"] / sus["p99_s"], 2)}}
    out["note"] = ("time to result from submission to the result on the host; arrivals replayed in real time; FP64 "
                   "sequential: every request of the window run alone, its device time (release setup, t=0 pass, steps) "
                   "replayed as a FIFO queue on the same arrival times")
    return out


def ref_process_bytes(c) -> int:
    """Host memory one reference process needs: its terrain Grid holds 17
    doubles per DEM node (src/data_arrays.hpp:49-93), its particles 84 B each,
    its remeshed grid about 4 nodes per particle at 136 B, plus input copies."""
    nodes = c["z"].size
    Np = len(c["particles"]["h"])
    return int(1.2 * (144 * nodes + 84 * Np + 4 * 136 * Np + 8 * nodes + 100 * Np))


def host_available_bytes() -> int:
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    return int(ln.split()[1]) * 1024
    except OSError:
        pass
    return 0


def repo_libraries_loaded() -> list:
    """Shared libraries of this repository mapped into this process."""
    try:
        with open("/proc/self/maps") as f:
            paths = {ln.split()[-1] for ln in f if ln.rstrip().endswith(".so")}
    except OSError:
        return []
    return sorted(os.path.relpath(p, ROOT) for p in paths if p.startswith(ROOT + os.sep))


def reference_arm(args, rank, world):
    if rank != 0:
        return None
    c = load_workload(args.workload)
    P = dict(c["particles"])
    Np = len(P["h"])
    avail = host_available_bytes()
    by_mem = max(1, int(0.7 * avail // ref_process_bytes(c))) if avail else 1
    replicas = max(1, min(os.cpu_count() or 1, args.ref_procs, by_mem))
    k = max(2, min(args.steps, int(args.cpu_seconds * 8e6 / Np)))
    w = max(0, args.warmup)
    t0 = time.perf_counter()
    v, st, sec = run_reference(c, P, k, replicas, warmup=w)
    wall = time.perf_counter() - t0
    return {"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": METRIC, "n_gpus": world, "steps": st,
            "warmup": w, "ms_per_step": round(sec / max(st, 1) * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": c["name"], "particles": Np, "dem": list(c["z"].shape), "dx": c["dx"],
                       "friction": c["cfg"]["friction"], "state": f"{w} warm-up steps from the initial state",
                       "parallelism": f"{replicas} concurrent single-threaded processes"},
            "cpu_baseline": {"value": round(v, 1), "unit": METRIC, "cores": replicas, "kind": "reference",
                             "sample": f"{w} untimed and {st} timed steps from the workload's initial state per process, "
                                       f"{replicas} processes (host cores {os.cpu_count()}, memory bound {by_mem}), "
                                       f"the reference's per-phase timers (slowest {sec:.1f} s, wall {wall:.1f} s)"},
            "e2e": {"value": round(v, 1), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "repo_libraries_loaded": repo_libraries_loaded()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3", "c3s"],
                    help="c3s: a smaller config-3 case for kernel captures")
    ap.add_argument("--spinup", type=float, default=2.0, help="simulated seconds of the developed-flow measurement")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP32-vs-FP64 whole-run accuracy blocks")
    ap.add_argument("--no-envelope", action="store_true", help="skip the FP64 envelope run of the headline accuracy block")
    ap.add_argument("--no-c2-accuracy", action="store_true", help="skip the config-2 accuracy block")
    ap.add_argument("--no-e2e-cli", action="store_true", help="skip the end-to-end run of the drop-in program")
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-procs", type=int, default=8)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--only", default="", choices=["", "fp32", "ensemble", "serving", "e2e_cli"],
                    help="fp32: only the FP32 path (profiling runs); ensemble / serving: only that section")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble section (config 4)")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-stream section (config 5)")
    ap.add_argument("--c4-scenarios", type=int, default=256)
    ap.add_argument("--c4-sample", type=int, default=16, help="scenarios run one after another for the sequential rates")
    ap.add_argument("--c4-acc-sample", type=int, default=8, help="scenarios of the whole-run accuracy block (with the FP64 envelope)")
    ap.add_argument("--c5-window", type=float, default=6.0, help="seconds of Poisson arrivals (the full stream is 300 s)")
    ap.add_argument("--c5-sustained", type=int, default=1, help="also replay the stream at 70 %% of the FP32 saturation rate")
    ap.add_argument("--c5-slots", type=int, default=512)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        log("warmup raised to 3")
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    try:
        line = ours(args, rank, world) if args.impl == "ours" else reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
