"""Plain FP64 GPU step loop against the oracle (pinned bit-exact to the
reference by test_oracle.py), through the C ABI.

Tolerances: the GPU path differs from the reference only in the order of
the P2G atomic sums and the last bit of CUDA's cos/atan, so single steps
agree to ~1e-13 relative; over whole runs the difference stays below
1e-6 m in positions and flow heights."""
import numpy as np
import pytest

import cases
import oracle as O
import slab

pytestmark = pytest.mark.gpu

CASES = list(cases.CASES)


def _gpu(c, precision=slab.FP64_PLAIN):
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], precision)
    s.upload(c["particles"])
    return s


def _oracle(c):
    o = O.Oracle(c["cfg"], c["z"], c["dx"])
    o.set_particles(c["particles"])
    o.t0()
    return o


@pytest.mark.parametrize("name", CASES)
def test_initial_pass_grid(name):
    c = cases.CASES[name]()
    s = _gpu(c)
    s.initial_pass()
    o = _oracle(c)
    G, Go = s.grid(), o.grid()
    assert (G["Nx"], G["Ny"], G["i_off"], G["j_off"]) == (Go["Nx"], Go["Ny"], Go["i_off"], Go["j_off"])
    for k in ("mass", "h", "vz"):
        np.testing.assert_allclose(G[k], Go[k], rtol=1e-13, atol=1e-12 * max(1.0, np.abs(Go[k]).max()))
    np.testing.assert_allclose(G["v"], Go["v"], rtol=1e-12, atol=1e-12)
    hm, _ = s.max_maps()
    ho, _ = o.max_maps()
    np.testing.assert_allclose(hm, ho, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("name", CASES)
def test_first_steps_match_reference_fixture(name, golden):
    """Steps 1 and 2 (before the reference's first sort) against the
    reference's own dumps."""
    c = cases.CASES[name]()
    g = golden(name)
    s = _gpu(c)
    s.initial_pass()
    for k in (1, 2):
        assert s.advance_steps(1) == 1
        t, dt, _, steps = s.state()
        assert steps == k
        assert t == pytest.approx(float(g[f"s{k}_time"]), rel=1e-15, abs=0)
        P = s.particles()
        np.testing.assert_allclose(P["x"], g[f"s{k}_x"], rtol=1e-14, atol=1e-12)
        np.testing.assert_allclose(P["v"], g[f"s{k}_v"], rtol=1e-11, atol=1e-11)
        np.testing.assert_allclose(P["h"], g[f"s{k}_h"], rtol=1e-12)
        np.testing.assert_allclose(P["z"], g[f"s{k}_z"], rtol=1e-13, atol=1e-10)


@pytest.mark.parametrize("name", CASES)
def test_frames_and_max_maps_vs_oracle(name):
    c = cases.CASES[name]()
    s = _gpu(c)
    s.initial_pass()
    o = _oracle(c)
    last = max(c["frames"])
    for f in range(1, last + 1):
        t, frame, _ = s.advance_to_frame()
        while True:
            if o.step() == 1:
                break
        assert frame == f
        to, _, fo, _ = o.state()
        assert fo == f and abs(t - to) < 1e-9
        if f in c["frames"]:
            P, Po = s.particles(), o.particles_by_id()
            dx_err = np.abs(P["x"] - Po["x"]).max()
            dh_err = np.abs(P["h"] - Po["h"]).max()
            assert dx_err < 1e-6, (f, dx_err)
            assert dh_err < 1e-6, (f, dh_err)
    hm, vm = s.max_maps()
    ho, vo = o.max_maps()
    assert np.abs(hm - ho).max() < 1e-6
    assert np.abs(np.sqrt(vm) - np.sqrt(vo)).max() < 1e-5


def test_run_to_total_time_and_conservation():
    c = cases.case_slope35()
    s = _gpu(c)
    s.initial_pass()
    M0 = c["particles"]["mass"].sum()
    n = 0
    while True:
        t, f, k = s.advance_to_frame()
        n += k
        if t >= c["cfg"]["total_time"]:
            break
    o = _oracle(c)
    no = o.run()
    assert n == no
    cons = s.conservation()
    assert abs(cons[0] - M0) <= 1e-12 * M0
    assert s.kernel_launches() > 4 * n
