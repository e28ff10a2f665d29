"""slab_initial_grid_static: the frame-0 grid for callers that cannot allocate
device memory (a host framework that owns the whole GPU heap, or a real-time
loop that may not allocate after start-up). The test owns the device buffers
(allocated here with torch, as such a framework would own them), calls the
entry point through the C ABI twice in a row, and checks both results against
the regular path (upload + initial pass + grid download, FP32 split) with the
tolerance of the FP32 t=0 grid tests, and against the oracle's grid. The
device's free memory must not change across the second call. It also checks
the error paths: an empty particle set, a box one node short of the
particles' stencils, an oversized box. This file sorts last so that a run
that stops at the first failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest

import cases
import oracle as O
import slab

pytestmark = pytest.mark.gpu


def _regular_grid(c):
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], slab.FP32_SPLIT)
    s.upload(c["particles"])
    s.initial_pass()
    g = s.grid()
    s.close()
    return g


def _oracle_grid(c):
    o = O.Oracle(c["cfg"], c["z"], c["dx"])
    o.set_particles(c["particles"])
    o.t0()
    return o.grid()


class StaticCall:
    """Device buffers of one case, owned by the caller, and the C-ABI call."""

    def __init__(self, c, box, torch, Np=None):
        self.L = slab.lib()
        dev = torch.device("cuda:0")
        P = c["particles"]
        self.Np = len(P["h"]) if Np is None else Np
        self.t = {k: torch.as_tensor(np.ascontiguousarray(P[k], dtype=np.float64), device=dev) for k in ("x", "v", "vz", "h", "mass")}
        self.z = torch.as_tensor(np.ascontiguousarray(c["z"], dtype=np.float64), device=dev)
        self.nI, self.nJ = box[1] - box[0] + 1, box[3] - box[2] + 1
        n = max(1, self.nI * self.nJ)
        self.out = {k: torch.zeros(n * (2 if k == "v" else 1), dtype=torch.float64, device=dev) for k in ("h", "mass", "v", "vz")}
        self.td = slab.TerrainDesc(c["z"].shape[0], c["z"].shape[1], float(c["dx"]), 0.0, 0.0)
        self.prm = slab.make_params(c["cfg"], slab.FP32_SPLIT)
        self.bx = (C.c_int32 * 4)(*box)
        vp = C.c_void_p
        self.L.slab_initial_grid_static.argtypes = [C.POINTER(slab.TerrainDesc), vp, C.POINTER(slab.Params), C.c_int32] + [vp] * 5 + \
            [C.POINTER(C.c_int32)] + [vp] * 4 + [vp]

    def __call__(self):
        vp = C.c_void_p
        t, out = self.t, self.out
        return self.L.slab_initial_grid_static(C.byref(self.td), vp(self.z.data_ptr()), C.byref(self.prm), self.Np,
                                               vp(t["x"].data_ptr()), vp(t["v"].data_ptr()), vp(t["vz"].data_ptr()),
                                               vp(t["h"].data_ptr()), vp(t["mass"].data_ptr()), self.bx, vp(out["h"].data_ptr()),
                                               vp(out["mass"].data_ptr()), vp(out["v"].data_ptr()), vp(out["vz"].data_ptr()), vp(None))

    def result(self):
        nI, nJ = self.nI, self.nJ
        return {k: self.out[k].cpu().numpy()[:nI * nJ * (2 if k == "v" else 1)].reshape((nI, nJ, 2) if k == "v" else (nI, nJ))
                for k in self.out}


def _box(g):
    return [g["i_off"], g["i_off"] + g["Nx"] - 1, g["j_off"], g["j_off"] + g["Ny"] - 1]


@pytest.mark.parametrize("name", ["slope35", "plane_voellmy", "fractal_mui"])
def test_static_grid_matches_regular_path_twice(name):
    torch = pytest.importorskip("torch")
    c = cases.CASES[name]()
    g = _regular_grid(c)
    go = _oracle_grid(c)
    call = StaticCall(c, _box(g), torch)
    for k in range(2):  # the second call must not see the first call's sums
        for t in call.out.values():
            t.fill_(-1.0)  # stale output values must be overwritten
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        code = call()
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert code == 0, slab.lib().slab_last_error(None)
        if k == 1:  # the first call may load the library's code on the device; the second allocates nothing
            assert free1 == free0, (free0, free1)
        s = call.result()
        sc = np.abs(g["mass"]).max()
        np.testing.assert_allclose(s["mass"], g["mass"], rtol=1e-5, atol=1e-6 * sc)
        np.testing.assert_allclose(s["h"], g["h"], rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(s["v"], g["v"], rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(s["vz"], g["vz"], rtol=1e-5, atol=1e-5)
        # and directly against the oracle's FP64 grid (tolerance of the FP32 t=0 grid tests)
        np.testing.assert_allclose(s["mass"], go["mass"], rtol=1e-5, atol=1e-6 * np.abs(go["mass"]).max())
        np.testing.assert_allclose(s["h"], go["h"], rtol=1e-5, atol=1e-5)


def test_static_grid_empty_particle_set():
    torch = pytest.importorskip("torch")
    c = cases.case_plane_voellmy()
    g = _regular_grid(c)
    call = StaticCall(c, _box(g), torch, Np=0)
    for t in call.out.values():
        t.fill_(-1.0)
    assert call() == 0, slab.lib().slab_last_error(None)
    s = call.result()
    for k in s:
        assert np.all(s[k] == 0.0), k


def test_static_grid_box_one_node_short_is_a_domain_error():
    torch = pytest.importorskip("torch")
    c = cases.case_plane_voellmy()
    g = _regular_grid(c)
    box = _box(g)
    # the remesh box has a margin of one node below and two above the
    # particles; the stencils need one node less on each side
    x = c["particles"]["x"] / c["dx"]
    i_hi = int(np.floor(x[:, 0] - 0.5).max()) + 2  # last stencil node in x
    box[1] = i_hi - 1
    call = StaticCall(c, box, torch)
    assert call() == 4  # SLAB_E_DOMAIN
    assert b"outside the box" in slab.lib().slab_last_error(None)


def test_static_grid_rejects_oversized_box():
    torch = pytest.importorskip("torch")
    c = dict(cases.case_slope35(), z=np.zeros((300, 300)))  # 90 000 nodes > the maximum of 65 536
    call = StaticCall(c, [0, 299, 0, 299], torch)
    assert call() == 1
    assert b"maximum" in slab.lib().slab_last_error(None)


def test_static_grid_rejects_reversed_box():
    torch = pytest.importorskip("torch")
    c = cases.case_slope35()
    call = StaticCall(c, [40, 2, 0, 50], torch)
    assert call() == 1
    assert b"box" in slab.lib().slab_last_error(None)
