"""slab_initial_grid_static: the frame-0 grid for callers that cannot allocate
device memory (a host framework that owns the whole GPU heap, or a real-time
loop that may not allocate after start-up). The test owns the device buffers
(allocated here with torch, as such a framework would own them), calls the
entry point through the C ABI twice in a row, and checks both results against
the regular path (upload + initial pass + grid download, FP32 split) with the
tolerance of the FP32 t=0 grid tests. This file sorts last so that a run that
stops at the first failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest

import cases
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


def _static_grid(c, box, torch, stream=None):
    L = slab.lib()
    dev = torch.device("cuda:0")
    P = c["particles"]
    t = {k: torch.as_tensor(np.ascontiguousarray(P[k], dtype=np.float64), device=dev) for k in ("x", "v", "vz", "h", "mass")}
    z = torch.as_tensor(np.ascontiguousarray(c["z"], dtype=np.float64), device=dev)
    nI, nJ = box[1] - box[0] + 1, box[3] - box[2] + 1
    out = {k: torch.zeros(nI * nJ * (2 if k == "v" else 1), dtype=torch.float64, device=dev) for k in ("h", "mass", "v", "vz")}
    td = slab.TerrainDesc(c["z"].shape[0], c["z"].shape[1], float(c["dx"]), 0.0, 0.0)
    prm = slab.make_params(c["cfg"], slab.FP32_SPLIT)
    bx = (C.c_int32 * 4)(*box)
    vp = C.c_void_p
    L.slab_initial_grid_static.argtypes = [C.POINTER(slab.TerrainDesc), vp, C.POINTER(slab.Params), C.c_int32] + [vp] * 5 + \
        [C.POINTER(C.c_int32)] + [vp] * 4 + [vp]
    code = L.slab_initial_grid_static(C.byref(td), vp(z.data_ptr()), C.byref(prm), len(P["h"]), vp(t["x"].data_ptr()),
                                      vp(t["v"].data_ptr()), vp(t["vz"].data_ptr()), vp(t["h"].data_ptr()),
                                      vp(t["mass"].data_ptr()), bx, vp(out["h"].data_ptr()), vp(out["mass"].data_ptr()),
                                      vp(out["v"].data_ptr()), vp(out["vz"].data_ptr()), vp(stream))
    return code, {k: out[k].cpu().numpy().reshape((nI, nJ, 2) if k == "v" else (nI, nJ)) for k in out}


@pytest.mark.parametrize("name", ["slope35", "plane_voellmy", "fractal_mui"])
def test_static_grid_matches_regular_path_twice(name):
    torch = pytest.importorskip("torch")
    c = cases.CASES[name]()
    g = _regular_grid(c)
    box = [g["i_off"], g["i_off"] + g["Nx"] - 1, g["j_off"], g["j_off"] + g["Ny"] - 1]
    for _ in range(2):  # the second call must not see the first call's sums
        code, s = _static_grid(c, box, torch)
        assert code == 0, slab.lib().slab_last_error(None)
        sc = np.abs(g["mass"]).max()
        np.testing.assert_allclose(s["mass"], g["mass"], rtol=1e-5, atol=1e-6 * sc)
        np.testing.assert_allclose(s["h"], g["h"], rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(s["v"], g["v"], rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(s["vz"], g["vz"], rtol=1e-5, atol=1e-5)


def test_static_grid_rejects_oversized_box():
    torch = pytest.importorskip("torch")
    c = dict(cases.case_slope35(), z=np.zeros((300, 300)))  # 90 000 nodes > the maximum of 65 536
    box = [0, 299, 0, 299]
    code, _ = _static_grid(c, box, torch)
    assert code == 1
    assert b"maximum" in slab.lib().slab_last_error(None)
