"""The Grid members a, F and flip (src/data_arrays.hpp:76,78,84) through the
C ABI's grid download, against the oracle's grid, for both arithmetics: after
simulate()'s t=0 pass and at the first output frame.

Tolerances: FP64 as the other FP64 grid tests (the P2G atomic sums may add
in another order); FP32 within 1e-5 of the field's largest magnitude at t=0
and 1e-2 at the first frame, where the FP32 state has run ~100 steps."""
import numpy as np
import pytest

import cases
import oracle as O
import slab

pytestmark = pytest.mark.gpu

CASES = list(cases.CASES)


def _pair(c, prec):
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], prec)
    s.upload(c["particles"])
    s.initial_pass()
    o = O.Oracle(c["cfg"], c["z"], c["dx"])
    o.set_particles(c["particles"])
    o.t0()
    return s, o


def _close(G, Go, keys, rel):
    assert (G["Nx"], G["Ny"], G["i_off"], G["j_off"]) == (Go["Nx"], Go["Ny"], Go["i_off"], Go["j_off"])
    for k in keys:
        sc = max(np.abs(Go[k]).max(), 1e-30)
        np.testing.assert_allclose(G[k], Go[k], rtol=0, atol=rel * sc, err_msg=k)


@pytest.mark.parametrize("name", CASES)
def test_fp64_force_acceleration_flip(name):
    c = cases.CASES[name]()
    s, o = _pair(c, slab.FP64_PLAIN)
    _close(s.grid(), o.grid(), ("F", "a", "flip"), 1e-12)
    s.advance_to_frame()
    while o.step() != 1:
        pass
    G, Go = s.grid(), o.grid()
    _close(G, Go, ("F", "a", "flip"), 1e-8)
    # a = F / mass where the node has mass, zero elsewhere
    moving = G["mass"] > 1e-6
    assert np.all(G["a"][~moving] == 0.0)
    np.testing.assert_allclose(G["a"][moving], G["F"][moving] / G["mass"][moving][:, None], rtol=1e-15)
    s.close()


@pytest.mark.parametrize("name", CASES)
def test_fp32_force_acceleration_flip(name):
    c = cases.CASES[name]()
    s, o = _pair(c, slab.FP32_SPLIT)
    _close(s.grid(), o.grid(), ("F", "a"), 1e-5)
    s.advance_to_frame()
    while o.step() != 1:
        pass
    _close(s.grid(), o.grid(), ("F", "a", "flip"), 1e-2)
    s.close()
