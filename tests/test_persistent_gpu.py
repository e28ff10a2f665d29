"""Persistent steps (slab_batch_set_persistent / slab_set_persistent): a chunk
of steps as one cooperative launch whose phases are separated by grid-wide
barriers. The results must be bitwise those of the default path (separate
kernels in CUDA graphs), with about one launch per chunk, and a barrier whose
wait runs out must end the launch with SLAB_E_TIMEOUT and leave the device
usable. The timeout is made by a limit far below the time one phase takes:
the first CTAs to reach a barrier give up before the last ones arrive (a
bounded wait, no fault)."""
import numpy as np
import pytest

import cases
import ensemble
import slab

pytestmark = pytest.mark.gpu


def _run_batch(persistent):
    z, dx, items = ensemble.ensemble()
    b = slab.Batch(z, dx, max_scenarios=8)
    if persistent:
        b.set_persistent(True)
    ids = [b.add(cfg, P) for cfg, P in items]
    l0 = b.kernel_launches()
    steps = b.run()
    launches = b.kernel_launches() - l0
    out = []
    for sid in ids:
        out.append((b.state(sid), b.particles(sid), b.max_maps(sid)))
    b.close()
    return out, steps, launches


def test_persistent_batch_equals_graph_path_bitwise():
    ref, steps_r, launches_r = _run_batch(False)
    per, steps_p, launches_p = _run_batch(True)
    assert steps_p == steps_r
    for (st_a, Pa, (ha, va)), (st_b, Pb, (hb, vb)) in zip(ref, per):
        assert st_a[2] == st_b[2]
        for k in ("x", "v", "vz", "h", "mass"):
            assert np.array_equal(Pa[k], Pb[k]), k
        assert np.array_equal(ha, hb) and np.array_equal(va, vb)
    # one cooperative launch per chunk of up to 32 steps, plus the per-call
    # start and the t=0 pass, against six kernels per step
    assert launches_p < launches_r / 20, (launches_p, launches_r)


@pytest.mark.parametrize("name", ["slope35", "fractal_mui"])
def test_persistent_single_scenario_frames_equal(name):
    c = cases.CASES[name]()
    res = []
    for persistent in (False, True):
        s = slab.Slab(c["z"], c["dx"])
        s.set_params(c["cfg"], slab.FP32_SPLIT)
        if persistent:
            s.set_persistent(True)
        s.upload(c["particles"])
        s.initial_pass()
        frames = []
        for _ in range(3):
            t, f, n = s.advance_to_frame()
            frames.append((t, f, n, s.particles()))
        res.append((frames, s.max_maps()))
        s.close()
    (fa, (ha, va)), (fb, (hb, vb)) = res
    for (ta, ka, na, Pa), (tb, kb, nb, Pb) in zip(fa, fb):
        assert (ta, ka, na) == (tb, kb, nb)
        for k in ("x", "v", "h"):
            assert np.array_equal(Pa[k], Pb[k]), k
    assert np.array_equal(ha, hb) and np.array_equal(va, vb)


def test_persistent_barrier_wait_gives_up_with_timeout():
    z, dx, items = ensemble.ensemble()
    b = slab.Batch(z, dx, max_scenarios=8)
    b.set_persistent(True, limit_cycles=64)  # far below one phase: the early CTAs give up
    for cfg, P in items:
        b.add(cfg, P)
    with pytest.raises(slab.SlabError) as ex:
        b.run(max_steps=64)
    assert ex.value.code == 6  # SLAB_E_TIMEOUT
    b.close()
    # the device is still usable: a new context runs normally
    c = cases.CASES["slope35"]()
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], slab.FP32_SPLIT)
    s.upload(c["particles"])
    s.initial_pass()
    assert s.advance_steps(10) == 10
    s.close()


def test_persistent_rejects_fp64():
    c = cases.CASES["slope35"]()
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], slab.FP64_PLAIN)
    with pytest.raises(slab.SlabError):
        s.set_persistent(True)
    s.close()
