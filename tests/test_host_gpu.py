"""The C++ drop-in end to end on the GPU: bin/slab_b200 runs a reference
input file (loadFromJSON -> initialize -> initializeTerrain ->
initializeParticles -> simulate) and writes the reference's output set --
particles_frame_N.ply and rasters_frame_N.tif for every frame, and
max_values.tif -- which are read back and checked against the FP64 oracle:
FP64_PLAIN within float32 storage of the values, FP32_SPLIT within the
tolerances of the FP32 parity tests (1 cm / 1 % on >= 99.5 % of wet nodes,
5 cm at most, runout within one cell)."""
import glob
import os
import subprocess
import sys

import numpy as np
import pytest

import cases
import oracle as O
import tiffread

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, os.path.join(ROOT, "slab-pro_b200"))
import accuracy as Acc  # noqa: E402
import make_golden as MG  # noqa: E402

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "slab-pro_b200", "bin", "slab_b200")


def _tif_to_nodes(band):
    """GDAL order (row 0 = north) -> [i, j] node order, nodata -> 0."""
    m = band[::-1, :].T.astype(np.float64)
    m[m == -9999.0] = 0.0
    return m


@pytest.fixture(scope="module")
def slope_oracle():
    c = cases.case_slope35()
    o = O.Oracle(c["cfg"], c["z"], c["dx"])
    o.set_particles(c["particles"])
    o.t0()
    frames = {}
    k = 0
    while True:
        if o.step() == 1:
            k += 1
            if k in (10, 60):
                frames[k] = o.particles_by_id()
            if k == 60:
                break
    return c, frames, o.max_maps()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_cli_run_writes_reference_outputs(prec, slope_oracle, tmp_path):
    c, frames, (ho, vo) = slope_oracle
    cfg = MG.write_inputs(c, str(tmp_path))
    args = [CLI, cfg] + (["--fp64"] if prec == "fp64" else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    sim = os.path.join(str(tmp_path), "out", c["name"])
    plys = sorted(glob.glob(os.path.join(sim, "particles", "particles_frame_*.ply")))
    tifs = sorted(glob.glob(os.path.join(sim, "rasters", "rasters_frame_*.tif")))
    assert len(plys) == 61 and len(tifs) == 61  # frames 0..60, zero-padded to 2 digits
    assert os.path.basename(plys[10]) == "particles_frame_10.ply"
    assert os.path.exists(os.path.join(sim, os.path.basename(cfg)))  # the input copied into the run directory

    # frame 10: particle count and centre of mass against the oracle
    P = tiffread.read_ply(plys[10])
    Po = frames[10]
    assert len(P["x"]) == len(Po["h"])
    m = Po["mass"]
    com = np.array([(P["x"] * m).sum(), (P["y"] * m).sum()]) / m.sum()
    como = (Po["x"] * m[:, None]).sum(0) / m.sum()
    assert np.abs(com - como).max() < (1e-3 if prec == "fp64" else c["dx"])

    # a frame raster: 6 bands, nodata where h == 0, georeferenced at the grid box corner
    T = tiffread.read_tiff(tifs[10])
    assert T["bands"].shape[0] == 6 and T["nodata"] == "-9999" and T["pixel_scale"][0] == c["dx"]
    h10 = T["bands"][0]
    assert ((h10 == -9999.0) == (T["bands"][2] == -9999.0)).all()

    # max_values.tif over the whole terrain
    M = tiffread.read_tiff(os.path.join(sim, "max_values.tif"))
    assert M["nx"] == c["z"].shape[0] and M["ny"] == c["z"].shape[1]
    hm = _tif_to_nodes(M["bands"][0])
    if prec == "fp64":
        assert np.abs(hm - ho).max() < 1e-5
        vm = _tif_to_nodes(M["bands"][1])
        assert np.abs(vm - np.sqrt(vo)).max() < 1e-4
    else:
        ok = Acc.h_ok(hm, ho)
        wet = (hm > 0) | (ho > 0)
        assert ok[wet].mean() >= 0.995
        assert np.abs(hm - ho).max() <= 0.05
        assert abs(Acc.runout(hm, c["dx"]) - Acc.runout(ho, c["dx"])) <= c["dx"]
