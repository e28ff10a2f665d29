"""The C++ host layer (libslab_sim.so, bin/slab_b200) without a GPU:
setup parity of Simulation::initializeParticles with the reference, the JSON
reader's errors, and the PLY / GeoTIFF writers read back byte for byte."""
import ctypes
import json
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
import make_golden as MG  # noqa: E402

CLI = os.path.join(ROOT, "slab-pro_b200", "bin", "slab_b200")
SIMLIB = os.path.join(ROOT, "slab-pro_b200", "lib", "libslab_sim.so")


def _init_only(cfg_path, out):
    r = subprocess.run([CLI, cfg_path, "--init-only", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return O.read_particles_bin(out)


@pytest.mark.parametrize("name", list(cases.CASES))
def test_setup_matches_reference_uniform(name, golden, tmp_path):
    """UNIFORM sampling: the initial particles equal the reference's, bit for bit."""
    c = cases.CASES[name]()
    cfg = MG.write_inputs(c, str(tmp_path))
    P = _init_only(cfg, str(tmp_path / "p.bin"))
    assert cases.particle_digest(P) == str(golden(name)["frame0_digest"])


@pytest.mark.parametrize("name", list(cases.CASES))
def test_setup_matches_reference_poisson(name, tmp_path):
    """POISSON sampling (the reference's sampler driven by std::rand seeded
    with 1): digests written by the reference binary (setup_poisson.json)."""
    ref = json.load(open(os.path.join(HERE, "golden", "setup_poisson.json")))[name]
    c = cases.CASES[name]()
    cfg = MG.write_inputs(c, str(tmp_path))
    j = json.load(open(cfg))
    j["numerical_params"]["sampling_method"] = "POISSON"
    json.dump(j, open(cfg, "w"))
    P = _init_only(cfg, str(tmp_path / "p.bin"))
    assert len(P["h"]) == ref["Np"]
    assert cases.particle_digest(P) == ref["digest"]


def test_missing_key_is_reported(tmp_path):
    c = cases.case_slope35()
    cfg = MG.write_inputs(c, str(tmp_path))
    j = json.load(open(cfg))
    del j["friction"]["coulomb"]
    json.dump(j, open(cfg, "w"))
    r = subprocess.run([CLI, cfg, "--init-only", str(tmp_path / "p.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "coulomb" in r.stderr


def test_malformed_json_and_unknown_names(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text('{"project_dir": "x", "sim_name": ')
    r = subprocess.run([CLI, str(p), "--init-only", str(tmp_path / "p.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "JSON parse error" in r.stderr
    c = cases.case_slope35()
    cfg = MG.write_inputs(c, str(tmp_path))
    j = json.load(open(cfg))
    j["friction"]["type"] = "GRANITE"
    json.dump(j, open(cfg, "w"))
    r = subprocess.run([CLI, cfg, "--init-only", str(tmp_path / "p.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown friction type" in r.stderr


def _write_asc(d, text):
    p = os.path.join(str(d), "bad.asc")
    with open(p, "w") as f:
        f.write(text)
    return p


BAD_INPUTS = {
    "terrain type": (lambda j, d: j["terrain"].__setitem__("type", "MOON"), "Unknown terrain type: MOON"),
    "release type": (lambda j, d: j["release"].__setitem__("type", "TRIANGLE"), "Unknown release shape type: TRIANGLE"),
    "sampling": (lambda j, d: j["numerical_params"].__setitem__("sampling_method", "HEXAGONAL"), "Unknown sampling method"),
    "polygon": (lambda j, d: j["release"].update({"type": "POLYGON", "polygon": {"filepath": os.path.join(str(d), "x.shp")}}),
                "POLYGON releases need a shapefile reader"),
    "missing dem": (lambda j, d: j["terrain"]["dem"].__setitem__("filepath", os.path.join(str(d), "none.asc")), "Failed to open ASC file"),
    "bad header": (lambda j, d: j["terrain"]["dem"].__setitem__("filepath", _write_asc(d, "hello world\n")), "Bad ASC header"),
    "short dem": (lambda j, d: j["terrain"]["dem"].__setitem__(
        "filepath", _write_asc(d, "ncols 4\nnrows 3\nxllcorner 0\nyllcorner 0\ncellsize 5\nNODATA_value -9999\n1 2 3 4\n5 6\n")),
        "ASC file ended early"),
    # releases past each side of the 2000 x 500 m terrain: a clear error, not a read outside it
    "edge low": (lambda j, d: j["release"]["rectangle"].__setitem__("center", [5.0, 5.0]), "release reaches the terrain edge"),
    "edge x": (lambda j, d: j["release"]["rectangle"].__setitem__("center", [1990.0, 250.0]), "release reaches the terrain edge"),
    "edge y": (lambda j, d: j["release"]["rectangle"].__setitem__("center", [150.0, 498.0]), "release reaches the terrain edge"),
}


@pytest.mark.parametrize("case", list(BAD_INPUTS))
def test_bad_inputs_are_reported(case, tmp_path):
    """Each bad input stops initialisation with exit code 1 and a message, as
    the reference's main() reports a std::runtime_error."""
    mutate, msg = BAD_INPUTS[case]
    c = cases.case_slope35()
    cfg = MG.write_inputs(c, str(tmp_path))
    j = json.load(open(cfg))
    mutate(j, tmp_path)
    json.dump(j, open(cfg, "w"))
    r = subprocess.run([CLI, cfg, "--init-only", str(tmp_path / "p.bin")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and msg in r.stderr, (r.returncode, r.stderr[-300:])


def _writers():
    L = ctypes.CDLL(SIMLIB)
    L.slab_write_geotiff.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_char_p,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_float, ctypes.c_int32]
    dp = ctypes.POINTER(ctypes.c_double)
    L.slab_write_ply.argtypes = [ctypes.c_char_p, ctypes.c_int32] + [dp] * 6
    return L


@pytest.mark.parametrize("comp", [1, 8, 50000, -1])
def test_geotiff_roundtrip(comp, tmp_path):
    L = _writers()
    rng = np.random.default_rng(comp & 0xFFFF)
    nx, ny, nb = 53, 701, 6
    b = rng.standard_normal((nb, ny, nx)).astype(np.float32)
    b[:, 10:20, 5:9] = -9999.0
    p = str(tmp_path / "t.tif")
    assert L.slab_write_geotiff(p.encode(), nx, ny, nb, b.ctypes.data, b"h,v_norm,m,v_x,v_y,v_z", 12.5, 3000.0, 2.0, -9999.0, comp) == 0
    t = tiffread.read_tiff(p)
    assert np.array_equal(t["bands"], b)
    assert t["compression"] == (L.slab_tiff_default_compression() if comp < 0 else comp)
    assert t["predictor"] == (1 if t["compression"] == 1 else 3)
    assert t["tiepoint"] == [0.0, 0.0, 0.0, 12.5, 3000.0, 0.0] and t["pixel_scale"] == [2.0, 2.0, 0.0]
    assert t["nodata"] == "-9999"
    assert 'sample="5" role="description">v_z<' in t["metadata"]


def test_geotiff_rejects_bad_arguments(tmp_path):
    L = _writers()
    b = np.zeros((1, 4, 4), np.float32)
    assert L.slab_write_geotiff(str(tmp_path / "a.tif").encode(), 0, 4, 1, b.ctypes.data, None, 0, 0, 1, 0, 1) == 1
    assert L.slab_write_geotiff(str(tmp_path / "a.tif").encode(), 4, 4, 1, b.ctypes.data, None, 0, 0, 1, 0, 7) == 1
    assert L.slab_write_geotiff(str(tmp_path / "no" / "dir" / "a.tif").encode(), 4, 4, 1, b.ctypes.data, None, 0, 0, 1, 0, 1) == 2


def test_ply_roundtrip(tmp_path):
    L = _writers()
    rng = np.random.default_rng(3)
    n = 1001
    x, v = rng.uniform(0, 1000, (n, 2)), rng.standard_normal((n, 2))
    vz, z, h, A = rng.standard_normal(n), rng.uniform(0, 500, n), rng.uniform(0.1, 3, n), np.full(n, 0.25)
    dp = ctypes.POINTER(ctypes.c_double)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, v, vz, z, h, A)]
    p = str(tmp_path / "p.ply")
    assert L.slab_write_ply(p.encode(), n, *[a.ctypes.data_as(dp) for a in arrs]) == 0
    r = tiffread.read_ply(p)
    assert list(r) == ["x", "y", "vx", "vy", "vz", "z", "h", "A"]
    for k, a in (("x", x[:, 0]), ("y", x[:, 1]), ("vx", v[:, 0]), ("vy", v[:, 1]), ("vz", vz), ("z", z), ("h", h), ("A", A)):
        assert np.array_equal(r[k], a.astype(np.float32)), k


def test_reference_style_caller_reads_grid_members(tmp_path):
    """A caller written against the reference's Grid (src/data_arrays.hpp:71-84)
    that reads grid.a, grid.F and grid.flip compiles and links against
    libslab_sim.so; the members resize with the grid."""
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include "simulation.hpp"
#include <cstdio>
int main() {
    slab::Grid g(3, 4);
    g.flip[5](0) = 1.0;
    g.F[5](1) = 2.0;
    g.a[5] = g.F[5];
    slab::Simulation sim;
    const slab::Grid& cur = sim.getGrid();
    std::printf("%zu %zu %zu %zu %g %g %g\n", g.a.size(), g.F.size(), g.flip.size(), cur.flip.size(), g.flip[5](0), g.F[5](1),
                g.a[5](1));
    return 0;
}
''')
    exe = tmp_path / "caller"
    inc = [f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(ROOT, 'slab-pro_b200', 'host')}"]
    libdir = os.path.dirname(SIMLIB)
    r = subprocess.run(["g++", "-std=c++17", *inc, str(src), "-o", str(exe), f"-L{libdir}", "-lslab_sim", "-lslab_gpu",
                        f"-Wl,-rpath,{libdir}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["12", "12", "12", "0", "1", "2", "2"]


def test_dem_binary_cache(golden, tmp_path):
    """readASC keeps a binary copy of a parsed DEM next to it
    (<file>.slabbin); a second run loads it and sets up the same particles, a
    damaged or stale cache is ignored and the text parsed again."""
    c = cases.case_fractal_mui()  # a DEM terrain and a raster release, both .asc
    cfg = MG.write_inputs(c, str(tmp_path))
    dem = os.path.join(str(tmp_path), "dem.asc")
    digest = str(golden("fractal_mui")["frame0_digest"])
    P = _init_only(cfg, str(tmp_path / "p1.bin"))
    assert cases.particle_digest(P) == digest
    cache = dem + ".slabbin"
    assert os.path.exists(cache)
    assert cases.particle_digest(_init_only(cfg, str(tmp_path / "p2.bin"))) == digest  # from the cache
    with open(cache, "r+b") as f:  # damaged: ignored
        f.write(b"XXXXXXXX")
    assert cases.particle_digest(_init_only(cfg, str(tmp_path / "p3.bin"))) == digest
    with open(dem, "a") as f:  # the source changed (size and time): the cache is stale
        f.write("\n")
    assert cases.particle_digest(_init_only(cfg, str(tmp_path / "p4.bin"))) == digest
