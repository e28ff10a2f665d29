"""ctypes binding of the C oracle (liboracle.so) plus readers for the dumps
written by the reference oracle binary (oracle/_ref/slab_ref).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "slab_ref")

FRICTION = {"COULOMB": 0, "VOELLMY": 1, "MU_I": 2}


class OracleParams(C.Structure):
    _fields_ = [
        ("gravity", C.c_double), ("rho", C.c_double),
        ("C_cfl", C.c_double), ("dt_max", C.c_double), ("flip_ratio", C.c_double),
        ("output_dt", C.c_double), ("total_time", C.c_double),
        ("friction_type", C.c_int32), ("sort_period", C.c_int32),
        ("coulomb_mu", C.c_double),
        ("voellmy_mu", C.c_double), ("voellmy_xi", C.c_double),
        ("mui_mu1", C.c_double), ("mui_mu2", C.c_double), ("mui_I0", C.c_double),
        ("mui_d", C.c_double), ("mui_phi", C.c_double),
    ]


def params_from_dict(d: dict) -> OracleParams:
    """d uses the keys of the reference JSON flattened (see workloads.Config)."""
    p = OracleParams()
    p.gravity, p.rho = d["gravity"], d["rho"]
    p.C_cfl, p.dt_max, p.flip_ratio = d["C_cfl"], d["dt_max"], d["flip_ratio"]
    p.output_dt, p.total_time = d["output_dt"], d["total_time"]
    p.friction_type = FRICTION[d["friction"]]
    p.sort_period = d.get("sort_period", 50)
    p.coulomb_mu = d.get("coulomb_mu", 0.0)
    p.voellmy_mu, p.voellmy_xi = d.get("voellmy_mu", 0.0), d.get("voellmy_xi", 1.0)
    p.mui_mu1, p.mui_mu2 = d.get("mui_mu1", 0.0), d.get("mui_mu2", 0.0)
    p.mui_I0, p.mui_d, p.mui_phi = d.get("mui_I0", 1.0), d.get("mui_d", 0.0), d.get("mui_phi", 1.0)
    return p


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.POINTER(OracleParams), C.c_int32, C.c_int32, C.c_double, dp]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_set_particles.argtypes = [C.c_void_p, C.c_int32] + [dp] * 8
        L.oracle_t0.argtypes = [C.c_void_p]
        L.oracle_step.argtypes = [C.c_void_p]
        L.oracle_run.argtypes = [C.c_void_p, C.c_int64]
        L.oracle_run.restype = C.c_int64
        L.oracle_get_state.argtypes = [C.c_void_p, dp, dp, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
        L.oracle_get_particles.argtypes = [C.c_void_p] + [dp] * 8
        L.oracle_get_grid_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        L.oracle_get_grid.argtypes = [C.c_void_p] + [dp] * 5
        L.oracle_get_grid_force.argtypes = [C.c_void_p, dp, dp]
        L.oracle_get_max.argtypes = [C.c_void_p, dp, dp]
        L.oracle_get_terrain_metrics.argtypes = [C.c_void_p, dp, dp]
        L.oracle_get_ids.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """FP64 CPU restatement of Simulation::simulate()'s step loop."""

    def __init__(self, params: dict, z: np.ndarray, dx: float):
        self.L = lib()
        self.Nx, self.Ny = z.shape
        self._z = np.ascontiguousarray(z, dtype=np.float64)
        self._p = params_from_dict(params)
        self.h = self.L.oracle_create(C.byref(self._p), self.Nx, self.Ny, float(dx), _dp(self._z))
        if not self.h:
            raise MemoryError("oracle_create failed")
        self.Np = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def set_particles(self, P: dict):
        self.Np = len(P["h"])
        a = {k: np.ascontiguousarray(P[k], dtype=np.float64) for k in ("x", "z", "v", "vz", "h", "A", "mass", "theta")}
        self._keep = a
        r = self.L.oracle_set_particles(self.h, self.Np, *[_dp(a[k]) for k in ("x", "z", "v", "vz", "h", "A", "mass", "theta")])
        if r:
            raise ValueError(f"oracle_set_particles: {r}")

    def t0(self):
        if self.L.oracle_t0(self.h):
            raise RuntimeError("oracle: particle stencil outside the terrain")

    def step(self) -> int:
        r = self.L.oracle_step(self.h)
        if r < 0:
            raise RuntimeError("oracle: particle stencil outside the terrain")
        return r

    def run(self, max_steps: int = 1 << 62) -> int:
        r = self.L.oracle_run(self.h, max_steps)
        if r < 0:
            raise RuntimeError("oracle: particle stencil outside the terrain")
        return r

    def state(self):
        t, dt = C.c_double(), C.c_double()
        fr, st = C.c_int32(), C.c_int64()
        self.L.oracle_get_state(self.h, C.byref(t), C.byref(dt), C.byref(fr), C.byref(st))
        return t.value, dt.value, fr.value, st.value

    def particles(self) -> dict:
        n = self.Np
        out = {k: np.zeros(2 * n if k in ("x", "v") else n) for k in ("x", "z", "v", "vz", "h", "A", "mass", "theta")}
        self.L.oracle_get_particles(self.h, *[_dp(out[k]) for k in ("x", "z", "v", "vz", "h", "A", "mass", "theta")])
        out["x"] = out["x"].reshape(n, 2)
        out["v"] = out["v"].reshape(n, 2)
        return out

    def ids(self) -> np.ndarray:
        """Upload index of each particle in the oracle's current order."""
        out = np.zeros(self.Np, dtype=np.int32)
        self.L.oracle_get_ids(self.h, out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out

    def particles_by_id(self) -> dict:
        """Particle arrays in upload order (undoing the every-50-steps sort)."""
        P = self.particles()
        ids = self.ids()
        out = {}
        for k, a in P.items():
            b = np.empty_like(a)
            b[ids] = a
            out[k] = b
        return out

    def grid(self) -> dict:
        d = (C.c_int32 * 4)()
        self.L.oracle_get_grid_dims(self.h, d)
        gNx, gNy, i0, j0 = list(d)
        n = gNx * gNy
        out = {"h": np.zeros(n), "mass": np.zeros(n), "v": np.zeros(2 * n), "vz": np.zeros(n), "flip": np.zeros(2 * n),
               "F": np.zeros(2 * n), "a": np.zeros(2 * n)}
        self.L.oracle_get_grid(self.h, *[_dp(out[k]) for k in ("h", "mass", "v", "vz", "flip")])
        self.L.oracle_get_grid_force(self.h, _dp(out["F"]), _dp(out["a"]))
        vec = ("v", "flip", "F", "a")
        g = {k: out[k].reshape(gNx, gNy, -1).squeeze(-1) if k not in vec else out[k].reshape(gNx, gNy, 2) for k in out}
        g.update(Nx=gNx, Ny=gNy, i_off=i0, j_off=j0)
        return g

    def max_maps(self):
        hm = np.zeros(self.Nx * self.Ny)
        vm = np.zeros(self.Nx * self.Ny)
        self.L.oracle_get_max(self.h, _dp(hm), _dp(vm))
        return hm.reshape(self.Nx, self.Ny), vm.reshape(self.Nx, self.Ny)

    def terrain_metrics(self):
        g = np.zeros(2 * self.Nx * self.Ny)
        th = np.zeros(self.Nx * self.Ny)
        self.L.oracle_get_terrain_metrics(self.h, _dp(g), _dp(th))
        return g.reshape(self.Nx, self.Ny, 2), th.reshape(self.Nx, self.Ny)


# ---------------------------------------------------------------------------
# readers for the reference binary's dumps (layouts in oracle/ref_hooks.cpp)

PARTICLE_FIELDS = ("x", "z", "v", "vz", "h", "A", "mass", "theta")


def _read_particle_block(buf, off, n):
    out = {}
    for k in PARTICLE_FIELDS:
        cnt = 2 * n if k in ("x", "v") else n
        a = np.frombuffer(buf, dtype=np.float64, count=cnt, offset=off).copy()
        off += 8 * cnt
        out[k] = a.reshape(n, 2) if k in ("x", "v") else a
    return out, off


def read_particles_bin(path: str) -> dict:
    buf = open(path, "rb").read()
    n, frame = struct.unpack_from("<qq", buf, 0)
    time, dt = struct.unpack_from("<dd", buf, 16)
    out, _ = _read_particle_block(buf, 32, n)
    out.update(Np=n, frame=frame, time=time, dt=dt)
    return out


def write_particles_bin(path: str, P: dict, frame: int = 0, time: float = 0.0, dt: float = 0.0):
    n = len(P["h"])
    with open(path, "wb") as f:
        f.write(struct.pack("<qqdd", n, frame, time, dt))
        for k in PARTICLE_FIELDS:
            f.write(np.ascontiguousarray(P[k], dtype=np.float64).tobytes())


def _read_grid_block(buf, off, Nx, Ny):
    n = Nx * Ny
    g = {}
    for k, c in (("h", 1), ("mass", 1), ("v", 2), ("vz", 1), ("flip", 2)):
        a = np.frombuffer(buf, dtype=np.float64, count=c * n, offset=off).copy()
        off += 8 * c * n
        g[k] = a.reshape(Nx, Ny, 2) if c == 2 else a.reshape(Nx, Ny)
    return g, off


def read_grid_bin(path: str) -> dict:
    buf = open(path, "rb").read()
    Nx, Ny, i0, j0, frame = struct.unpack_from("<5q", buf, 0)
    time, dt = struct.unpack_from("<dd", buf, 40)
    g, _ = _read_grid_block(buf, 56, Nx, Ny)
    g.update(Nx=Nx, Ny=Ny, i_off=i0, j_off=j0, frame=frame, time=time, dt=dt)
    return g


def read_max_bin(path: str):
    buf = open(path, "rb").read()
    Nx, Ny = struct.unpack_from("<qq", buf, 0)
    n = Nx * Ny
    hm = np.frombuffer(buf, dtype=np.float64, count=n, offset=16).reshape(Nx, Ny).copy()
    vm = np.frombuffer(buf, dtype=np.float64, count=n, offset=16 + 8 * n).reshape(Nx, Ny).copy()
    return hm, vm


def read_steps_bin(path: str):
    """Records of the phase driver (ref_hooks.cpp saveTerrain)."""
    buf = open(path, "rb").read()
    Np, TNx, TNy, nsteps = struct.unpack_from("<4q", buf, 0)
    off = 32
    recs = []
    for _ in range(nsteps + 1):
        (k,) = struct.unpack_from("<q", buf, off)
        time, dt = struct.unpack_from("<dd", buf, off + 8)
        off += 24
        P, off = _read_particle_block(buf, off, Np)
        gNx, gNy, i0, j0 = struct.unpack_from("<4q", buf, off)
        off += 32
        g, off = _read_grid_block(buf, off, gNx, gNy)
        g.update(Nx=gNx, Ny=gNy, i_off=i0, j_off=j0)
        nt = TNx * TNy
        hm = np.frombuffer(buf, dtype=np.float64, count=nt, offset=off).reshape(TNx, TNy).copy()
        off += 8 * nt
        vm = np.frombuffer(buf, dtype=np.float64, count=nt, offset=off).reshape(TNx, TNy).copy()
        off += 8 * nt
        recs.append(dict(step=k, time=time, dt=dt, particles=P, grid=g, h_max=hm, v_max2=vm))
    return recs
