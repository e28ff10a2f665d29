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
