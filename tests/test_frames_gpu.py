"""Output frames packed on the device (slab_frame_capture / slab_frame_wait)
against the synchronous downloads of the same state, for both arithmetics:
the particle vertices are the float32 values of the downloaded particles
(x y vx vy vz z h A, upload order, the PLY vertex layout), the grid bands the
float32 values of the downloaded grid in GeoTIFF order (row 0 = north edge,
-9999 where h == 0). Frames are captured into both slots while the steps of
the next frame run; the values must be identical, bit for bit."""
import numpy as np
import pytest

import cases
import slab

pytestmark = pytest.mark.gpu


def _expected(s):
    P = s.particles()
    G = s.grid()
    V = np.stack([P["x"][:, 0], P["x"][:, 1], P["v"][:, 0], P["v"][:, 1], P["vz"], P["z"], P["h"], P["A"]], axis=1).astype(np.float32)
    h = G["h"].astype(np.float32)
    vn = np.sqrt(G["v"][..., 0] ** 2 + G["v"][..., 1] ** 2).astype(np.float32)
    bands = np.stack([h, vn, G["mass"].astype(np.float32), G["v"][..., 0].astype(np.float32), G["v"][..., 1].astype(np.float32),
                      G["vz"].astype(np.float32)])
    bands[:, h == 0] = -9999.0
    return V, bands[:, :, ::-1].transpose(0, 2, 1), G  # [band, i, j] -> [band, row (north first), i]


@pytest.mark.parametrize("prec", [slab.FP64_PLAIN, slab.FP32_SPLIT])
@pytest.mark.parametrize("name", list(cases.CASES))
def test_packed_frames_equal_downloads(name, prec):
    c = cases.CASES[name]()
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], prec)
    s.upload(c["particles"])
    s.initial_pass()
    for k in range(4):  # frames 0..3, slots 0, 1, 0, 1
        slot = k % 2
        s.frame_capture(slot)
        F = s.frame_wait(slot)
        V, B, G = _expected(s)
        assert F["frame"] == k
        assert (F["Nx"], F["Ny"], F["i_off"], F["j_off"]) == (G["Nx"], G["Ny"], G["i_off"], G["j_off"])
        assert np.array_equal(F["particles"], V)
        assert np.array_equal(F["grid"], B)
        s.advance_to_frame()
    s.close()


def test_capture_overlaps_the_next_frame():
    """A frame captured before the next advance call still holds its own
    state after that call, and the other slot holds the next frame."""
    c = cases.case_slope35()
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], slab.FP32_SPLIT)
    s.upload(c["particles"])
    s.initial_pass()
    s.advance_to_frame()
    V1, _, _ = _expected(s)
    s.frame_capture(1)
    s.advance_to_frame()  # the copy of frame 1 runs beside these steps
    s.frame_capture(0)
    F1, F2 = s.frame_wait(1), s.frame_wait(0)
    V2, _, _ = _expected(s)
    assert F1["frame"] == 1 and F2["frame"] == 2
    assert np.array_equal(F1["particles"], V1) and np.array_equal(F2["particles"], V2)
    assert not np.array_equal(V1, V2)
    s.close()
