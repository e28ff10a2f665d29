"""Batched ensemble: every scenario of a batch gives bitwise the same result as
running it alone through slab_ctx (FP32 split), although all scenarios share
every kernel launch and have their own dt, friction law and duration."""
import numpy as np
import pytest

import ensemble
import slab

pytestmark = pytest.mark.gpu


def test_batch_equals_alone_bitwise():
    z, dx, items = ensemble.ensemble()
    b = slab.Batch(z, dx, max_scenarios=8)
    ids = [b.add(cfg, P) for cfg, P in items]
    b.run()
    for sid, (cfg, P) in zip(ids, items):
        t, _, steps = b.state(sid)
        assert abs(t - cfg["total_time"]) < 1e-9
        s = slab.Slab(z, dx)
        s.set_params(cfg, slab.FP32_SPLIT)
        s.upload(P)
        s.initial_pass()
        n = s.advance_steps(10 ** 9)
        assert n == steps
        Pa, Pb = s.particles(), b.particles(sid)
        for k in ("x", "v", "h", "mass"):
            assert np.array_equal(Pa[k], Pb[k]), (sid, k)
        ha, va = s.max_maps()
        hb, vb = b.max_maps(sid)
        assert np.array_equal(ha, hb) and np.array_equal(va, vb), sid
        s.close()
    pw, nw = b.work_counters()
    assert pw == sum(b.state(i)[2] * len(items[i][1]["h"]) for i in ids)
    assert nw > 0
    b.close()


def test_batch_rejects_fp64_and_overflow():
    z, dx, items = ensemble.ensemble()
    b = slab.Batch(z, dx, max_scenarios=1)
    cfg, P = items[0]
    b.add(cfg, P)
    with pytest.raises(slab.SlabError):
        b.add(cfg, P)  # full
    b.close()


def test_heterogeneous_batch_against_fp64():
    """A batch of scenarios with different friction laws, sizes and durations
    (FP32 split) against each scenario run alone in FP64_PLAIN: max-height
    maps within 1 cm or 1 % on at least 99 % of the wet nodes, runout within
    one cell, the same step count within 1 %, and the particle mass of each
    scenario equal to its FP64 total within float rounding (a mass never
    changes in either path)."""
    import accuracy as Acc
    z, dx, items = ensemble.ensemble()
    b = slab.Batch(z, dx, max_scenarios=8)
    ids = [b.add(cfg, P) for cfg, P in items]
    b.run()
    for sid, (cfg, P) in zip(ids, items):
        hb, _ = b.max_maps(sid)
        s = slab.Slab(z, dx)
        s.set_params(cfg, slab.FP64_PLAIN)
        s.upload(P)
        s.initial_pass()
        n64 = s.advance_steps(10 ** 9)
        h64, _ = s.max_maps()
        s.close()
        wet = (hb > 0) | (h64 > 0)
        assert wet.any()
        assert Acc.h_ok(hb, h64)[wet].mean() >= 0.99, sid
        assert abs(Acc.runout(hb, dx) - Acc.runout(h64, dx)) <= dx, sid
        assert abs(b.state(sid)[2] - n64) <= max(1, 0.01 * n64), sid
        m32 = b.particles(sid)["mass"].sum()
        assert abs(m32 - P["mass"].sum()) <= 1e-7 * P["mass"].sum(), sid
    b.close()
