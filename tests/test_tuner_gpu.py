"""Launch-shape tuner of the FP32 step: the CTA counts of the five work
kernels (k_prep, dense/sparse P2G, grid update, G2P) change which CTA computes
a tile, never a value. A batch run with the tuner on (it times its candidates
on the first steps, so those steps run under all five candidate shapes), with
the occupancy shapes fixed, and with small odd grids that give each CTA many
tiles, ends in bitwise the same particles and maxima."""
import numpy as np
import pytest

import ensemble
import slab

pytestmark = pytest.mark.gpu

STEPS = 400


def _run(z, dx, items, grids, tune):
    b = slab.Batch(z, dx, max_scenarios=len(items))
    if grids is not None or not tune:
        b.set_launch_shapes(grids, tune=tune)
    ids = [b.add(cfg, P) for cfg, P in items]
    b.run(STEPS)
    out = []
    for sid in ids:
        P = b.particles(sid)
        out.append(({k: P[k] for k in ("x", "v", "h", "mass")}, b.max_maps(sid), b.state(sid)))
    shapes, tunes = b.launch_shapes()
    b.close()
    return out, shapes, tunes


def test_launch_shapes_do_not_change_results():
    z, dx, items = ensemble.ensemble()
    ref, occ_shapes, n0 = _run(z, dx, items, None, tune=False)
    assert n0 == 0 and min(occ_shapes) > 0
    odd, odd_shapes, _ = _run(z, dx, items, [1, 3, 2, 5, 7], tune=False)
    assert odd_shapes == [1, 3, 2, 5, 7]
    tuned, tuned_shapes, n1 = _run(z, dx, items, None, tune=True)
    assert n1 >= 1
    for k, f in enumerate(tuned_shapes):  # every pick is one of the candidates: 1/4 to 4 occupancy grids
        assert f in [max(1, occ_shapes[k] * m // 4) for m in (1, 2, 4, 8, 16)], (k, f, occ_shapes[k])
    for other in (odd, tuned):
        for (Pa, (ha, va), sa), (Pb, (hb, vb), sb) in zip(ref, other):
            assert sa == sb
            for k in Pa:
                assert np.array_equal(Pa[k], Pb[k]), k
            assert np.array_equal(ha, hb) and np.array_equal(va, vb)


def test_set_launch_shapes_rejects_negative():
    z, dx, items = ensemble.ensemble()
    b = slab.Batch(z, dx, max_scenarios=1)
    with pytest.raises(slab.SlabError):
        b.set_launch_shapes([1, -1, 1, 1, 1])
    b.close()
