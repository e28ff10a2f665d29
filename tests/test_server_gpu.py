"""Serving with continuous batching: requests that arrive while others run are
admitted between chunks, share the GPU, and each result is bitwise the same
as a solo run. Failures are injected on the host side (a request whose flow
leaves the terrain, a cancelled request, a tiny memory budget): none of them
faults the GPU, and the other requests still complete."""
import time

import numpy as np
import pytest

import ensemble
import slab

pytestmark = pytest.mark.gpu


def _solo(z, dx, cfg, P):
    s = slab.Slab(z, dx)
    s.set_params(cfg, slab.FP32_SPLIT)
    s.upload(P)
    s.initial_pass()
    s.advance_steps(10 ** 9)
    out = s.particles()
    hm, vm = s.max_maps()
    s.close()
    return out, hm, vm


def test_results_equal_solo_runs_in_the_mix():
    z, dx, items = ensemble.ensemble()
    srv = slab.Server(z, dx, max_scenarios=3, chunk_steps=16)
    ids = [srv.submit(*items[0]), srv.submit(*items[1])]
    time.sleep(0.2)  # the first two are on the GPU when the others arrive
    ids += [srv.submit(*items[2]), srv.submit(*items[3])]
    srv.drain(600)
    for rid, (cfg, P) in zip(ids, items):
        st, ttr = srv.poll(rid)
        assert st == slab.REQ_DONE and ttr > 0
        r = srv.result(rid)
        ref, hm, vm = _solo(z, dx, cfg, P)
        for k in ("x", "v", "h", "mass"):
            assert np.array_equal(r[k], ref[k]), (rid, k)
        i0, i1, j0, j1 = r["box"]
        assert np.array_equal(r["h_max"], hm[i0:i1 + 1, j0:j1 + 1]) and np.array_equal(r["v_max2"], vm[i0:i1 + 1, j0:j1 + 1])
        assert hm.sum() == r["h_max"].sum()  # nothing outside the box
        assert abs(r["time"] - cfg["total_time"]) < 1e-9
    st = srv.stats()
    assert st["completed"] == 4 and st["p99_s"] >= st["p50_s"] > 0
    srv.close()


def test_failure_cancel_and_budget_do_not_disturb_others():
    z, dx, items = ensemble.ensemble()
    # tiny budget: one request at a time
    srv = slab.Server(z, dx, max_scenarios=4, chunk_steps=16, hbm_budget_bytes=1)
    cfg0, P0 = items[0]
    # a request whose flow leaves the terrain (fast particles at the right edge)
    bad = {k: v[:50].copy() for k, v in items[3][1].items()}
    bad["x"][:, 0] = (z.shape[0] - 6) * dx
    bad["v"][:, 0] = 300.0
    rid_bad = srv.submit(dict(items[3][0], total_time=5.0), bad)
    rid_ok = srv.submit(cfg0, P0)
    rid_cancel = srv.submit(*items[2])
    srv.cancel(rid_cancel)
    srv.drain(600)
    assert srv.poll(rid_bad)[0] == slab.REQ_FAILED
    assert srv.poll(rid_cancel)[0] == slab.REQ_CANCELLED
    assert srv.poll(rid_ok)[0] == slab.REQ_DONE
    r = srv.result(rid_ok)
    ref, hm, _ = _solo(z, dx, cfg0, P0)
    assert np.array_equal(r["x"], ref["x"])
    assert r["seconds_queued"] >= 0
    srv.close()
