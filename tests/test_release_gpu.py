"""Release setup on the device (slab_upload_release, slab_batch_add_release,
slab_server_submit_release) against the host setup of the reference
(workloads.release_particles, whose particles equal the reference binary's,
tests/test_host.py and the golden frame-0 digests): the particles are the
same doubles, bit for bit, and a scenario built either way runs to the same
bits."""
import numpy as np
import pytest

import cases
import slab
import workloads as W

pytestmark = pytest.mark.gpu

FIELDS = ("x", "v", "vz", "h", "A", "mass", "z")


def _device_particles(c, rel):
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], slab.FP64_PLAIN)  # the FP64 path keeps the uploaded doubles
    n = s.upload_release(rel)
    P = s.particles()
    s.close()
    return n, P


@pytest.mark.parametrize("name", ["slope35", "plane_voellmy"])
def test_release_particles_equal_the_reference_setup(name):
    c = cases.CASES[name]()
    n, P = _device_particles(c, c["release"])
    ref = c["particles"]
    assert n == len(ref["h"])
    for k in FIELDS:
        assert np.array_equal(P[k], ref[k]), k


def test_rotated_ellipse_on_fractal_terrain():
    z = W.fractal_slope_dem(512, 2.0, seed=5, rms=3.0, x_plane_end=600.0, ease_m=200.0)
    cfg = dict(gravity=9.81, rho=300.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0, total_time=5.0,
               friction="VOELLMY", voellmy_mu=0.2, voellmy_xi=1500.0)
    rel = {"type": "ELLIPSE", "center": (301.3, 497.7), "rx": 121.7, "ry": 63.1, "rotation_deg": 37.3, "h0": 1.7}
    ref = W.release_particles(z, 2.0, rel, cfg["rho"])
    n, P = _device_particles({"z": z, "dx": 2.0, "cfg": cfg}, rel)
    assert n == len(ref["h"])
    for k in FIELDS:
        assert np.array_equal(P[k], ref[k]), k


def test_release_at_the_terrain_edge_is_a_domain_error():
    c = cases.case_slope35()
    rel = dict(c["release"], center=(40.0, 250.0))  # the 4x4 z stencil of the first cells leaves the terrain
    s = slab.Slab(c["z"], c["dx"])
    s.set_params(c["cfg"], slab.FP64_PLAIN)
    with pytest.raises(slab.SlabError) as e:
        s.upload_release(rel)
    assert e.value.code == 4
    s.close()


def test_batch_and_server_release_runs_equal_particle_runs():
    c = cases.case_plane_voellmy()
    cfg = dict(c["cfg"], total_time=4.0)
    b = slab.Batch(c["z"], c["dx"], 2)
    a = b.add(cfg, c["particles"])
    r = b.add_release(cfg, c["release"])
    b.run()
    Pa, Pr = b.particles(a), b.particles(r)
    for k in Pa:
        assert np.array_equal(Pa[k], Pr[k]), k
    b.close()
    srv = slab.Server(c["z"], c["dx"], max_scenarios=4)
    i1 = srv.submit(cfg, c["particles"])
    i2 = srv.submit_release(cfg, c["release"])
    srv.drain(timeout=300.0)
    R1, R2 = srv.result(i1), srv.result(i2)
    for k in ("x", "v", "h", "mass", "h_max", "v_max2"):
        assert np.array_equal(R1[k], R2[k]), k
    assert R1["box"] == R2["box"]
    srv.close()
