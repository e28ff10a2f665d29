"""Python binding of libslab_gpu.so (include/slab_gpu.h) over ctypes.

The library is the product; this module only marshals numpy arrays. It loads
the in-tree build (slab-pro_b200/lib/libslab_gpu.so) and fails loudly when it
is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# SLAB_GPU_LIB selects another build of the library (e.g. an instrumented one)
LIB_PATH = os.environ.get("SLAB_GPU_LIB") or os.path.join(HERE, "lib", "libslab_gpu.so")

COULOMB, VOELLMY, MU_I = 0, 1, 2
FRICTION_NAMES = {"COULOMB": COULOMB, "VOELLMY": VOELLMY, "MU_I": MU_I}
FP64_PLAIN, FP32_SPLIT = 0, 1

STATUS = {0: "SLAB_OK", 1: "SLAB_E_ARG", 2: "SLAB_E_CUDA", 3: "SLAB_E_OOM", 4: "SLAB_E_DOMAIN",
          5: "SLAB_E_NONFINITE", 6: "SLAB_E_TIMEOUT", 7: "SLAB_E_STATE", 8: "SLAB_E_NOTFOUND"}


class SlabError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Friction(C.Structure):
    _fields_ = [("type", C.c_int32), ("pad_", C.c_int32), ("coulomb_mu", C.c_double),
                ("voellmy_mu", C.c_double), ("voellmy_xi", C.c_double),
                ("mu_1", C.c_double), ("mu_2", C.c_double), ("I0", C.c_double), ("d", C.c_double), ("phi", C.c_double)]


class Params(C.Structure):
    _fields_ = [("gravity", C.c_double), ("rho", C.c_double), ("C_cfl", C.c_double), ("dt_max", C.c_double),
                ("flip_ratio", C.c_double), ("output_dt", C.c_double), ("total_time", C.c_double),
                ("friction", Friction), ("precision", C.c_int32), ("pad_", C.c_int32)]


class TerrainDesc(C.Structure):
    _fields_ = [("Nx", C.c_int32), ("Ny", C.c_int32), ("dx", C.c_double), ("xllcorner", C.c_double), ("yllcorner", C.c_double)]


class GridView(C.Structure):
    _fields_ = [("Nx", C.c_int32), ("Ny", C.c_int32), ("i_off", C.c_int32), ("j_off", C.c_int32), ("cap_nodes", C.c_int64),
                ("h", C.POINTER(C.c_double)), ("mass", C.POINTER(C.c_double)), ("v", C.POINTER(C.c_double)),
                ("vz", C.POINTER(C.c_double)), ("flip", C.POINTER(C.c_double)), ("F", C.POINTER(C.c_double)),
                ("a", C.POINTER(C.c_double))]


class Release(C.Structure):
    _fields_ = [("type", C.c_int32), ("pad_", C.c_int32), ("cx", C.c_double), ("cy", C.c_double), ("a", C.c_double),
                ("b", C.c_double), ("rotation_deg", C.c_double), ("h0", C.c_double)]


RELEASE_RECTANGLE, RELEASE_ELLIPSE = 0, 1


def make_release(rel: dict) -> Release:
    """A RECTANGLE / ELLIPSE release in the form of workloads.release_particles."""
    if rel["type"] == "RECTANGLE":
        return Release(RELEASE_RECTANGLE, 0, rel["center"][0], rel["center"][1], rel["Lx"], rel["Ly"], rel["rotation_deg"], rel["h0"])
    if rel["type"] == "ELLIPSE":
        return Release(RELEASE_ELLIPSE, 0, rel["center"][0], rel["center"][1], rel["rx"], rel["ry"], rel["rotation_deg"], rel["h0"])
    raise ValueError(f"release type {rel['type']} is built on the host only")


class Frame(C.Structure):
    _fields_ = [("frame", C.c_int32), ("Np", C.c_int32), ("time", C.c_double), ("particles", C.POINTER(C.c_float)),
                ("Nx", C.c_int32), ("Ny", C.c_int32), ("i_off", C.c_int32), ("j_off", C.c_int32), ("grid", C.POINTER(C.c_float))]


_lib = None


def lib():
    """Load the in-tree CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C slab-pro_b200` or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        vp = C.c_void_p
        L.slab_create.argtypes = [C.POINTER(TerrainDesc), dp, C.POINTER(vp)]
        L.slab_set_params.argtypes = [vp, C.POINTER(Params)]
        L.slab_set_stream.argtypes = [vp, vp]
        L.slab_upload_particles.argtypes = [vp, C.c_int32] + [dp] * 7
        L.slab_initial_pass.argtypes = [vp]
        L.slab_advance_to_frame.argtypes = [vp, dp, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
        L.slab_advance_steps.argtypes = [vp, C.c_int64, C.POINTER(C.c_int64)]
        L.slab_advance_steps_async.argtypes = [vp, C.c_int64]
        L.slab_synchronize.argtypes = [vp]
        L.slab_download_particles.argtypes = [vp] + [dp] * 7
        L.slab_download_grid.argtypes = [vp, C.POINTER(GridView)]
        L.slab_download_max.argtypes = [vp, dp, dp]
        L.slab_conservation.argtypes = [vp, dp]
        L.slab_moments.argtypes = [vp, dp]
        L.slab_frame_capture.argtypes = [vp, C.c_int32]
        L.slab_upload_release.argtypes = [vp, C.POINTER(Release), C.POINTER(C.c_int32)]
        L.slab_frame_wait.argtypes = [vp, C.c_int32, C.POINTER(Frame)]
        L.slab_batch_moments.argtypes = [vp, C.c_int32, dp]
        L.slab_get_state.argtypes = [vp, dp, dp, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
        L.slab_set_profiling.argtypes = [vp, C.c_int32]
        L.slab_get_phase_times.argtypes = [vp, dp]
        L.slab_work_counters.argtypes = [vp, C.POINTER(C.c_int64)]
        L.slab_poisson_disk.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int32, C.c_uint64, dp, C.c_int64,
                                        C.POINTER(C.c_int64)]
        L.slab_kernel_launches.argtypes = [vp]
        L.slab_launch_shapes.argtypes = [vp, C.POINTER(C.c_int32)]
        L.slab_kernel_launches.restype = C.c_int64
        L.slab_last_error.argtypes = [vp]
        L.slab_last_error.restype = C.c_char_p
        L.slab_destroy.argtypes = [vp]
        L.slab_version.restype = C.c_char_p
        L.slab_status_name.restype = C.c_char_p
        L.slab_status_name.argtypes = [C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _out_array(a, n: int) -> np.ndarray:
    """A caller's output array as a flat float64 view of at least n values."""
    a = np.asarray(a)
    if a.dtype != np.float64 or not a.flags.c_contiguous or a.size < n:
        raise ValueError(f"output array must be contiguous float64 of at least {n} values")
    return a.reshape(-1)[:n]


def poisson_disk(Lx: float, Ly: float, r: float, seed: int, k: int = 30) -> np.ndarray:
    """Poisson-disk samples (n, 2) in [0,Lx]x[0,Ly] relative to the corner
    (seed 0 reproduces the reference's rand()-driven sampler)."""
    L = lib()
    n = C.c_int64()
    code = L.slab_poisson_disk(Lx, Ly, r, k, seed, None, 0, C.byref(n))
    if code:
        raise SlabError(code, "slab_poisson_disk")
    out = np.zeros(2 * n.value)
    code = L.slab_poisson_disk(Lx, Ly, r, k, seed, _dp(out), n.value, C.byref(n))
    if code:
        raise SlabError(code, "slab_poisson_disk")
    return out.reshape(-1, 2)


def make_params(cfg: dict, precision: int = FP64_PLAIN) -> Params:
    """cfg: flat dict with gravity, rho, C_cfl, dt_max, flip_ratio, output_dt,
    total_time, friction ('COULOMB'|'VOELLMY'|'MU_I') and its coefficients
    (coulomb_mu | voellmy_mu, voellmy_xi | mui_mu1, mui_mu2, mui_I0, mui_d, mui_phi)."""
    p = Params()
    p.gravity, p.rho = cfg["gravity"], cfg["rho"]
    p.C_cfl, p.dt_max, p.flip_ratio = cfg["C_cfl"], cfg["dt_max"], cfg["flip_ratio"]
    p.output_dt, p.total_time = cfg["output_dt"], cfg["total_time"]
    f = p.friction
    f.type = FRICTION_NAMES[cfg["friction"]]
    f.coulomb_mu = cfg.get("coulomb_mu", 0.0)
    f.voellmy_mu, f.voellmy_xi = cfg.get("voellmy_mu", 0.0), cfg.get("voellmy_xi", 1.0)
    f.mu_1, f.mu_2 = cfg.get("mui_mu1", 0.0), cfg.get("mui_mu2", 0.0)
    f.I0, f.d, f.phi = cfg.get("mui_I0", 1.0), cfg.get("mui_d", 0.0), cfg.get("mui_phi", 1.0)
    p.precision = precision
    return p


class Slab:
    """One simulation context on the current CUDA device."""

    def __init__(self, z: np.ndarray, dx: float, xll: float = 0.0, yll: float = 0.0):
        self.L = lib()
        self.Nx, self.Ny = z.shape
        zz = np.ascontiguousarray(z, dtype=np.float64)
        td = TerrainDesc(self.Nx, self.Ny, float(dx), float(xll), float(yll))
        h = C.c_void_p()
        self._check(self.L.slab_create(C.byref(td), _dp(zz), C.byref(h)), None)
        self.h = h
        self.Np = 0

    def _check(self, code, h="self"):
        if code != 0:
            msg = self.L.slab_last_error(self.h if h == "self" else None)
            raise SlabError(code, (msg or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.slab_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_params(self, cfg: dict, precision: int = FP64_PLAIN):
        self._params = make_params(cfg, precision)
        self._check(self.L.slab_set_params(self.h, C.byref(self._params)))

    def set_stream(self, stream_handle: int):
        self._check(self.L.slab_set_stream(self.h, C.c_void_p(stream_handle)))

    def set_persistent(self, on: bool = True, limit_cycles: int = 0):
        """FP32_SPLIT: run each chunk of steps as one persistent cooperative
        launch (bitwise the same results); barrier waits give up after
        limit_cycles SM clocks (0: the current limit)."""
        self.L.slab_set_persistent.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
        self._check(self.L.slab_set_persistent(self.h, int(bool(on)), int(limit_cycles)))

    def upload(self, P: dict):
        n = len(P["h"])
        arrs = [np.ascontiguousarray(P[k], dtype=np.float64) for k in ("x", "v", "vz", "h", "A", "mass", "z")]
        self._check(self.L.slab_upload_particles(self.h, n, *[_dp(a) for a in arrs]))
        self.Np = n

    def upload_release(self, rel: dict) -> int:
        """Particles of a RECTANGLE / ELLIPSE release (UNIFORM sampling) built
        on the device; returns their count."""
        r = make_release(rel)
        n = C.c_int32()
        self._check(self.L.slab_upload_release(self.h, C.byref(r), C.byref(n)))
        self.Np = n.value
        return n.value

    def initial_pass(self):
        self._check(self.L.slab_initial_pass(self.h))

    def advance_to_frame(self):
        t, f, s = C.c_double(), C.c_int32(), C.c_int64()
        self._check(self.L.slab_advance_to_frame(self.h, C.byref(t), C.byref(f), C.byref(s)))
        return t.value, f.value, s.value

    def advance_steps(self, n: int) -> int:
        s = C.c_int64()
        self._check(self.L.slab_advance_steps(self.h, int(n), C.byref(s)))
        return s.value

    def advance_steps_async(self, n: int):
        """Enqueue n steps on the context's stream without waiting."""
        self._check(self.L.slab_advance_steps_async(self.h, int(n)))

    def synchronize(self):
        self._check(self.L.slab_synchronize(self.h))

    def particles(self, out: dict = None) -> dict:
        """The particles in the reference layout (FP64, upload order). `out`
        may hold caller-owned contiguous float64 arrays (pinned host memory
        makes the copy run at full link speed): x and v of 2 n values, the
        others of n."""
        n = self.Np
        keys = ("x", "v", "vz", "h", "A", "mass", "z")
        if out is None:
            out = {k: np.zeros(2 * n if k in ("x", "v") else n) for k in keys}
        else:
            out = {k: _out_array(out[k], 2 * n if k in ("x", "v") else n) for k in keys}
        self._check(self.L.slab_download_particles(self.h, *[_dp(out[k]) for k in keys]))
        out["x"] = out["x"].reshape(n, 2)
        out["v"] = out["v"].reshape(n, 2)
        return out

    def grid(self) -> dict:
        """The last step's grid over the remeshed box: the members of the
        reference's Grid (h, mass, vz; v, flip, F, a as [Nx, Ny, 2])."""
        box = GridView()
        self._check(self.L.slab_download_grid(self.h, C.byref(box)))
        cap = max(1, box.Nx * box.Ny)
        vec = ("v", "flip", "F", "a")
        bufs = {k: np.zeros(2 * cap if k in vec else cap) for k in ("h", "mass", "v", "vz", "flip", "F", "a")}
        gv = GridView(0, 0, 0, 0, cap, *[_dp(bufs[k]) for k in ("h", "mass", "v", "vz", "flip", "F", "a")])
        self._check(self.L.slab_download_grid(self.h, C.byref(gv)))
        n = gv.Nx * gv.Ny
        g = {k: bufs[k][:n].reshape(gv.Nx, gv.Ny) for k in ("h", "mass", "vz")}
        for k in vec:
            g[k] = bufs[k][:2 * n].reshape(gv.Nx, gv.Ny, 2)
        g.update(Nx=gv.Nx, Ny=gv.Ny, i_off=gv.i_off, j_off=gv.j_off)
        return g

    def max_maps(self, out=None):
        """(h_max, v_max) over the whole terrain; `out` may be a caller-owned
        pair of contiguous float64 arrays of Nx * Ny values."""
        n = self.Nx * self.Ny
        hm, vm = (np.zeros(n), np.zeros(n)) if out is None else (_out_array(out[0], n), _out_array(out[1], n))
        self._check(self.L.slab_download_max(self.h, _dp(hm), _dp(vm)))
        return hm.reshape(self.Nx, self.Ny), vm.reshape(self.Nx, self.Ny)

    def conservation(self):
        out = np.zeros(4)
        self._check(self.L.slab_conservation(self.h, _dp(out)))
        return out

    def frame_capture(self, slot: int):
        """Pack the current frame on the device and start its copy to the host."""
        self._check(self.L.slab_frame_capture(self.h, int(slot)))

    def frame_wait(self, slot: int) -> dict:
        """The captured frame: particles [Np, 8] float32 (x y vx vy vz z h A)
        and grid [6, Ny, Nx] float32 bands in GeoTIFF order (copies)."""
        f = Frame()
        code = self.L.slab_frame_wait(self.h, int(slot), C.byref(f))
        if code != 0:
            raise SlabError(code, (self.L.slab_last_error(None) or b"").decode())
        parts = np.ctypeslib.as_array(f.particles, shape=(f.Np * 8,)).reshape(f.Np, 8).copy() if f.Np else np.zeros((0, 8), np.float32)
        n = f.Nx * f.Ny
        grid = np.ctypeslib.as_array(f.grid, shape=(6 * n,)).reshape(6, f.Ny, f.Nx).copy() if n else np.zeros((6, 0, 0), np.float32)
        return {"frame": f.frame, "time": f.time, "particles": parts, "grid": grid, "Nx": f.Nx, "Ny": f.Ny, "i_off": f.i_off,
                "j_off": f.j_off}

    def moments(self) -> dict:
        """FP64 particle moments summed on the device: mass, centre of mass,
        momentum, kinetic energy."""
        out = np.zeros(6)
        self._check(self.L.slab_moments(self.h, _dp(out)))
        return {"mass": out[0], "com": out[1:3].copy(), "momentum": out[3:5].copy(), "kinetic": out[5]}

    def state(self):
        t, dt, f, s = C.c_double(), C.c_double(), C.c_int32(), C.c_int64()
        self._check(self.L.slab_get_state(self.h, C.byref(t), C.byref(dt), C.byref(f), C.byref(s)))
        return t.value, dt.value, f.value, s.value

    def work_counters(self):
        """(particle-steps, active node-steps) done so far."""
        out = (C.c_int64 * 2)()
        self._check(self.L.slab_work_counters(self.h, out))
        return int(out[0]), int(out[1])

    def kernel_launches(self) -> int:
        return self.L.slab_kernel_launches(self.h)

    def set_profiling(self, on: bool):
        self._check(self.L.slab_set_profiling(self.h, 1 if on else 0))

    def phase_times(self):
        out = np.zeros(5)
        self._check(self.L.slab_get_phase_times(self.h, _dp(out)))
        return out

    def launch_shapes(self):
        """FP32: (CTA counts of k_prep, dense P2G, sparse P2G, grid update, G2P; tuning passes done)."""
        out = (C.c_int32 * 6)()
        self._check(self.L.slab_launch_shapes(self.h, out))
        return [int(v) for v in out[:5]], int(out[5])


class Batch:
    """Many scenarios on one shared terrain, advanced together (FP32 split)."""

    def __init__(self, z: np.ndarray, dx: float, max_scenarios: int, capacity_hint: int = 0):
        self.L = L = lib()
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.slab_batch_create.argtypes = [C.POINTER(TerrainDesc), dp, C.c_int32, C.c_int64, C.POINTER(vp)]
        L.slab_batch_set_stream.argtypes = [vp, vp]
        L.slab_batch_add.argtypes = [vp, C.POINTER(Params), C.c_int32] + [dp] * 7 + [C.POINTER(C.c_int32)]
        L.slab_batch_add_release.argtypes = [vp, C.POINTER(Params), C.POINTER(Release), C.POINTER(C.c_int32)]
        L.slab_batch_scenario_particles.argtypes = [vp, C.c_int32]
        L.slab_batch_scenario_particles.restype = C.c_int32
        L.slab_batch_run.argtypes = [vp, C.c_int64, C.POINTER(C.c_int64)]
        L.slab_batch_state.argtypes = [vp, C.c_int32, dp, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
        L.slab_batch_scenario_status.argtypes = [vp, C.c_int32]
        L.slab_batch_download_particles.argtypes = [vp, C.c_int32] + [dp] * 7
        L.slab_batch_download_max.argtypes = [vp, C.c_int32, dp, dp]
        L.slab_batch_download_max_box.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32), dp, dp, C.c_int64]
        L.slab_batch_work_counters.argtypes = [vp, C.POINTER(C.c_int64)]
        L.slab_batch_kernel_launches.argtypes = [vp]
        L.slab_batch_set_profiling.argtypes = [vp, C.c_int32]
        L.slab_batch_phase_times.argtypes = [vp, dp]
        L.slab_batch_launch_shapes.argtypes = [vp, C.POINTER(C.c_int32)]
        L.slab_batch_set_launch_shapes.argtypes = [vp, C.POINTER(C.c_int32), C.c_int32]
        L.slab_batch_kernel_launches.restype = C.c_int64
        L.slab_batch_last_error.argtypes = [vp]
        L.slab_batch_last_error.restype = C.c_char_p
        L.slab_batch_destroy.argtypes = [vp]
        self.Nx, self.Ny = z.shape
        zz = np.ascontiguousarray(z, dtype=np.float64)
        td = TerrainDesc(self.Nx, self.Ny, float(dx), 0.0, 0.0)
        h = C.c_void_p()
        code = L.slab_batch_create(C.byref(td), _dp(zz), int(max_scenarios), int(capacity_hint), C.byref(h))
        if code:
            raise SlabError(code, (L.slab_last_error(None) or b"").decode())
        self.h = h
        self.Np = []
        self._params = []

    def _check(self, code):
        if code:
            raise SlabError(code, (self.L.slab_batch_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.slab_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_stream(self, stream_handle: int):
        self._check(self.L.slab_batch_set_stream(self.h, C.c_void_p(stream_handle)))

    def add(self, cfg: dict, P: dict) -> int:
        prm = make_params(cfg, FP32_SPLIT)
        self._params.append(prm)
        n = len(P["h"])
        arrs = [np.ascontiguousarray(P[k], dtype=np.float64) for k in ("x", "v", "vz", "h", "A", "mass", "z")]
        sid = C.c_int32()
        self._check(self.L.slab_batch_add(self.h, C.byref(prm), n, *[_dp(a) for a in arrs], C.byref(sid)))
        self.Np.append(n)
        return sid.value

    def set_persistent(self, on: bool = True, limit_cycles: int = 0):
        """Run each chunk of steps as one persistent cooperative launch
        (bitwise the same results as separate kernels); barrier waits give up
        after limit_cycles SM clocks (0: the current limit)."""
        self.L.slab_batch_set_persistent.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
        self._check(self.L.slab_batch_set_persistent(self.h, int(bool(on)), int(limit_cycles)))

    def add_release(self, cfg: dict, rel: dict) -> int:
        """A scenario whose particles are built on the device from a release."""
        prm = make_params(cfg, FP32_SPLIT)
        self._params.append(prm)
        r = make_release(rel)
        sid = C.c_int32()
        self._check(self.L.slab_batch_add_release(self.h, C.byref(prm), C.byref(r), C.byref(sid)))
        self.Np.append(self.L.slab_batch_scenario_particles(self.h, sid.value))
        return sid.value

    def run(self, max_steps: int = 1 << 40) -> int:
        s = C.c_int64()
        self._check(self.L.slab_batch_run(self.h, int(max_steps), C.byref(s)))
        return s.value

    def state(self, sid: int):
        t, f, s = C.c_double(), C.c_int32(), C.c_int64()
        self._check(self.L.slab_batch_state(self.h, sid, C.byref(t), C.byref(f), C.byref(s)))
        return t.value, f.value, s.value

    def scenario_status(self, sid: int) -> int:
        """0 (OK) or the status code of the error that stopped the scenario."""
        return int(self.L.slab_batch_scenario_status(self.h, sid))

    def particles(self, sid: int) -> dict:
        n = self.Np[sid]
        out = {k: np.zeros(2 * n if k in ("x", "v") else n) for k in ("x", "v", "vz", "h", "A", "mass", "z")}
        self._check(self.L.slab_batch_download_particles(self.h, sid, *[_dp(out[k]) for k in ("x", "v", "vz", "h", "A", "mass", "z")]))
        out["x"] = out["x"].reshape(n, 2)
        out["v"] = out["v"].reshape(n, 2)
        return out

    def moments(self, sid: int) -> dict:
        out = np.zeros(6)
        self._check(self.L.slab_batch_moments(self.h, sid, _dp(out)))
        return {"mass": out[0], "com": out[1:3].copy(), "momentum": out[3:5].copy(), "kinetic": out[5]}

    def max_maps(self, sid: int):
        hm = np.zeros(self.Nx * self.Ny)
        vm = np.zeros(self.Nx * self.Ny)
        self._check(self.L.slab_batch_download_max(self.h, sid, _dp(hm), _dp(vm)))
        return hm.reshape(self.Nx, self.Ny), vm.reshape(self.Nx, self.Ny)

    def max_box(self, sid: int):
        """(box {i0, i1, j0, j1}, h_max, v_max2) over the nodes the flow touched."""
        box = (C.c_int32 * 4)()
        self._check(self.L.slab_batch_download_max_box(self.h, sid, box, None, None, 0))
        nI, nJ = max(box[1] - box[0] + 1, 0), max(box[3] - box[2] + 1, 0)
        hm, vm = np.zeros(max(nI * nJ, 1)), np.zeros(max(nI * nJ, 1))
        self._check(self.L.slab_batch_download_max_box(self.h, sid, box, _dp(hm), _dp(vm), nI * nJ))
        return list(box), hm[:nI * nJ].reshape(nI, nJ), vm[:nI * nJ].reshape(nI, nJ)

    def work_counters(self):
        out = (C.c_int64 * 2)()
        self._check(self.L.slab_batch_work_counters(self.h, out))
        return int(out[0]), int(out[1])

    def kernel_launches(self) -> int:
        return self.L.slab_batch_kernel_launches(self.h)

    def set_profiling(self, on: bool):
        self._check(self.L.slab_batch_set_profiling(self.h, int(on)))

    def phase_times(self):
        """ms per kernel family since profiling was switched on: control, binning, P2G, grid, G2P."""
        out = np.zeros(5)
        self._check(self.L.slab_batch_phase_times(self.h, _dp(out)))
        return out.tolist()

    def launch_shapes(self):
        """(CTA counts of k_prep, dense P2G, sparse P2G, grid update, G2P; tuning passes done)."""
        out = (C.c_int32 * 6)()
        self._check(self.L.slab_batch_launch_shapes(self.h, out))
        return [int(v) for v in out[:5]], int(out[5])

    def set_launch_shapes(self, grids=None, tune: bool = True):
        """Fix CTA counts (grids[k] > 0; 0 or None: tuned); tune=False stops the tuner."""
        g = None if grids is None else (C.c_int32 * 5)(*[int(v) for v in grids])
        self._check(self.L.slab_batch_set_launch_shapes(self.h, g, 1 if tune else 0))


class ServerConfig(C.Structure):
    _fields_ = [("max_scenarios", C.c_int32), ("chunk_steps", C.c_int32), ("hbm_budget_bytes", C.c_int64)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_CANCELLED, REQ_FAILED = range(5)


class Server:
    """Continuous-batching request loop on one GPU (a worker thread in the library)."""

    def __init__(self, z: np.ndarray, dx: float, max_scenarios: int = 64, chunk_steps: int = 32, hbm_budget_bytes: int = 0):
        self.L = L = lib()
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.slab_server_create.argtypes = [C.POINTER(TerrainDesc), dp, C.POINTER(ServerConfig), C.POINTER(vp)]
        L.slab_server_submit.argtypes = [vp, C.POINTER(Params), C.c_int32] + [dp] * 7 + [C.POINTER(C.c_int64)]
        L.slab_server_submit_release.argtypes = [vp, C.POINTER(Params), C.POINTER(Release), C.POINTER(C.c_int64)]
        L.slab_server_particles.argtypes = [vp, C.c_int64, C.POINTER(C.c_int32)]
        L.slab_server_poll.argtypes = [vp, C.c_int64, C.POINTER(C.c_int32), dp]
        L.slab_server_wait.argtypes = [vp, C.c_int64, C.c_double]
        L.slab_server_result.argtypes = [vp, C.c_int64, C.POINTER(C.c_int32), dp, dp, C.c_int64, dp, dp, dp, dp, dp]
        L.slab_server_cancel.argtypes = [vp, C.c_int64]
        L.slab_server_drain.argtypes = [vp, C.c_double]
        L.slab_server_stats.argtypes = [vp, dp]
        L.slab_server_timing.argtypes = [vp, dp]
        L.slab_server_last_error.argtypes = [vp]
        L.slab_server_last_error.restype = C.c_char_p
        L.slab_server_destroy.argtypes = [vp]
        self.Nx, self.Ny = z.shape
        zz = np.ascontiguousarray(z, dtype=np.float64)
        td = TerrainDesc(self.Nx, self.Ny, float(dx), 0.0, 0.0)
        cfg = ServerConfig(int(max_scenarios), int(chunk_steps), int(hbm_budget_bytes))
        h = C.c_void_p()
        code = L.slab_server_create(C.byref(td), _dp(zz), C.byref(cfg), C.byref(h))
        if code:
            raise SlabError(code, (L.slab_last_error(None) or b"").decode())
        self.h = h
        self.Np = {}

    def _check(self, code):
        if code:
            raise SlabError(code, (self.L.slab_server_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.slab_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def submit(self, cfg: dict, P: dict) -> int:
        prm = make_params(cfg, FP32_SPLIT)
        n = len(P["h"])
        arrs = [np.ascontiguousarray(P[k], dtype=np.float64) for k in ("x", "v", "vz", "h", "A", "mass", "z")]
        rid = C.c_int64()
        self._check(self.L.slab_server_submit(self.h, C.byref(prm), n, *[_dp(a) for a in arrs], C.byref(rid)))
        self.Np[rid.value] = n
        return rid.value

    def submit_release(self, cfg: dict, rel: dict) -> int:
        """Queue a scenario given as a release; its particles are built on the
        device at admission."""
        prm = make_params(cfg, FP32_SPLIT)
        r = make_release(rel)
        rid = C.c_int64()
        self._check(self.L.slab_server_submit_release(self.h, C.byref(prm), C.byref(r), C.byref(rid)))
        self.Np[rid.value] = None  # known once admitted
        return rid.value

    def poll(self, rid: int):
        st, t = C.c_int32(), C.c_double()
        self._check(self.L.slab_server_poll(self.h, rid, C.byref(st), C.byref(t)))
        return st.value, t.value

    def wait(self, rid: int, timeout: float = 600.0):
        self._check(self.L.slab_server_wait(self.h, rid, timeout))

    def result(self, rid: int) -> dict:
        box = (C.c_int32 * 4)()
        info = np.zeros(4)
        self._check(self.L.slab_server_result(self.h, rid, box, None, None, 0, None, None, None, None, _dp(info)))
        nI, nJ = box[1] - box[0] + 1, box[3] - box[2] + 1
        cap = max(nI, 0) * max(nJ, 0)
        n = self.Np[rid]
        if n is None:
            k = C.c_int32()
            self._check(self.L.slab_server_particles(self.h, rid, C.byref(k)))
            n = self.Np[rid] = k.value
        hm, vm = np.zeros(max(cap, 1)), np.zeros(max(cap, 1))
        x, v, h, m = np.zeros(2 * n), np.zeros(2 * n), np.zeros(n), np.zeros(n)
        self._check(self.L.slab_server_result(self.h, rid, box, _dp(hm), _dp(vm), cap, _dp(x), _dp(v), _dp(h), _dp(m), _dp(info)))
        return {"box": list(box), "h_max": hm[:cap].reshape(max(nI, 0), max(nJ, 0)), "v_max2": vm[:cap].reshape(max(nI, 0), max(nJ, 0)),
                "x": x.reshape(n, 2), "v": v.reshape(n, 2), "h": h, "mass": m, "steps": int(info[0]), "time": info[1],
                "seconds_to_result": info[2], "seconds_queued": info[3]}

    def cancel(self, rid: int):
        self._check(self.L.slab_server_cancel(self.h, rid))

    def drain(self, timeout: float = 600.0):
        self._check(self.L.slab_server_drain(self.h, timeout))

    def stats(self) -> dict:
        out = np.zeros(8)
        self._check(self.L.slab_server_stats(self.h, _dp(out)))
        keys = ("completed", "p50_s", "p99_s", "scenarios_per_s", "particle_steps", "batched_steps", "busy_s", "bytes_admitted")
        return dict(zip(keys, out.tolist()))

    def timing(self) -> dict:
        out = np.zeros(8)
        self._check(self.L.slab_server_timing(self.h, _dp(out)))
        keys = ("admit_s", "chunk_s", "retire_s", "chunks", "mean_running", "max_running", "capacity_growths", "kernel_launches")
        return dict(zip(keys, out.tolist()))
