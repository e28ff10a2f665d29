"""Synthetic inputs and host-side setup for the Slab-Pro step loop.

* ESRI ASCII grid (.asc) reading and writing with the reference's conventions
  (Simulation::readASC, src/complex_terrain.cpp:31-65: rows are stored top
  to bottom and reversed so that j grows northwards; node (i, j) sits at
  (i*cellsize, j*cellsize) and z is flattened i*Ny + j).
* The reference's particle initialisation for RECTANGLE / ELLIPSE / RASTER
  releases with UNIFORM sampling (Simulation::initializeParticles,
  src/simulation.cpp:259-476), restated with numpy in the same operation
  order so the particle sets are bit-identical.
* Seeded generators for the benchmark workloads: the 35-degree slope with a
  circular-arc runout (1 600 particles), fractal slopes with spectral
  roughness on 4096^2 / 8192^2 / 2048^2 DEMs, star-polygon raster releases
  with lognormal heights, and ensembles of elliptical releases.

No public dataset is involved: every workload is generated here from a seed.
"""
from __future__ import annotations

import math

import numpy as np

# ---------------------------------------------------------------- .asc files


def read_asc(path: str):
    """Return (z[Nx, Ny], header dict) exactly as Simulation::readASC."""
    with open(path) as f:
        hdr = {}
        for _ in range(6):
            k, v = f.readline().split()
            hdr[k.lower()] = float(v)
        nc, nr = int(hdr["ncols"]), int(hdr["nrows"])
        vals = np.array(f.read().split(), dtype=np.float64)
    if vals.size != nc * nr:
        raise ValueError(f"{path}: expected {nc * nr} values, found {vals.size}")
    z = np.empty((nc, nr))
    z[:, ::-1] = vals.reshape(nr, nc).T
    return z, hdr


def write_asc(path: str, z: np.ndarray, cellsize: float, xll: float = 0.0, yll: float = 0.0, nodata: float = -9999.0):
    """Write z[Nx, Ny] so that read_asc (and the reference) read back the same doubles."""
    nc, nr = z.shape
    with open(path, "w") as f:
        f.write(f"ncols {nc}\nnrows {nr}\nxllcorner {xll!r}\nyllcorner {yll!r}\ncellsize {cellsize!r}\nNODATA_value {nodata!r}\n")
        rows = z[:, ::-1].T  # top row first
        for r in rows:
            f.write(" ".join(repr(float(v)) for v in r))
            f.write("\n")


# ------------------------------------------------------- reference particle setup


def _N(u):
    """Quadratic B-spline, src/tools.hpp:119-128 (vectorised)."""
    a = np.abs(u)
    return np.where(a < 0.5, 0.75 - a * a, np.where(a < 1.5, 0.5 * (1.5 - a) * (1.5 - a), 0.0))


def terrain_gradient_norm(z: np.ndarray, dx: float) -> np.ndarray:
    """|grad z| of terrainGradients (src/complex_terrain.cpp:84-100)."""
    ood = 1.0 / dx
    gx = np.zeros_like(z)
    gy = np.zeros_like(z)
    gx[:-1, :-1] = (z[1:, :-1] + z[1:, 1:] - z[:-1, :-1] - z[:-1, 1:]) / 2.0 * ood
    gy[:-1, :-1] = (z[:-1, 1:] + z[1:, 1:] - z[:-1, :-1] - z[1:, :-1]) / 2.0 * ood
    return np.sqrt(gx * gx + gy * gy)


def libm_atan(a: np.ndarray) -> np.ndarray:
    """atan through the C library (as the reference calls it); numpy's own
    vectorised arctan can differ in the last bit."""
    return np.frompyfunc(math.atan, 1, 1)(a).astype(np.float64)


def terrain_theta(z: np.ndarray, dx: float) -> np.ndarray:
    """terrainTheta (src/complex_terrain.cpp:102-111) over the whole terrain."""
    return libm_atan(terrain_gradient_norm(z, dx))


def release_particles(z: np.ndarray, dx: float, release: dict, rho: float, sampling: str = "UNIFORM",
                      samples: np.ndarray | None = None, fast_theta: bool = False, grad_norm: np.ndarray | None = None) -> dict:
    """Simulation::initializeParticles for RECTANGLE/ELLIPSE/RASTER releases.

    release: {"type": "RECTANGLE", "center": (x, y), "Lx", "Ly", "rotation_deg", "h0"}
             {"type": "ELLIPSE", "center": (x, y), "rx", "ry", "rotation_deg", "h0"}
             {"type": "RASTER", "h": h[nc, nr], "x0", "y0", "cellsize", "nodata", "h_min"}
               (x0, y0: raster origin relative to the terrain origin)
    sampling: "UNIFORM" (2x2 per cell) or "GIVEN" (samples: positions relative
    to the bounding box corner, as the Poisson sampler returns them).
    """
    ood = 1.0 / dx
    typ = release["type"]
    if typ == "RECTANGLE":
        cx, cy = release["center"]
        Lx, Ly = release["Lx"], release["Ly"]
        diag = math.sqrt(Lx * Lx + Ly * Ly) / 2.0
        x_min, x_max, y_min, y_max = cx - diag, cx + diag, cy - diag, cy + diag
        area = Lx * Ly
    elif typ == "ELLIPSE":
        cx, cy = release["center"]
        big = max(release["rx"], release["ry"])
        x_min, x_max, y_min, y_max = cx - big, cx + big, cy - big, cy + big
        area = math.pi * release["rx"] * release["ry"]
    elif typ == "RASTER":
        rh = release["h"]
        cs = release["cellsize"]
        x_min, y_min = release["x0"], release["y0"]
        x_max = x_min + cs * (rh.shape[0] - 1)
        y_max = y_min + cs * (rh.shape[1] - 1)
        # loop order j outer, i inner as in the reference (src/simulation.cpp:337-345)
        mask = (rh >= release["h_min"]) & (rh > 0.0)
        vol = 0.0
        cell_area = cs * cs
        for j in range(rh.shape[1]):
            for i in np.nonzero(mask[:, j])[0]:
                vol += rh[i, j] * cell_area
        area = int(mask.sum()) * cell_area
    else:
        raise ValueError(f"release type {typ} not supported here")
    volume = vol if typ == "RASTER" else area * release["h0"]
    x_min = math.floor(x_min * ood) * dx
    x_max = math.ceil(x_max * ood) * dx
    y_min = math.floor(y_min * ood) * dx
    y_max = math.ceil(y_max * ood) * dx
    if sampling == "UNIFORM":
        nxc = int(round((x_max - x_min) * ood))
        nyc = int(round((y_max - y_min) * ood))
        dxp = np.array([0.25, 0.75, 0.25, 0.75])
        dyp = np.array([0.25, 0.25, 0.75, 0.75])
        I, J, D = np.meshgrid(np.arange(nxc, dtype=np.float64), np.arange(nyc, dtype=np.float64), np.arange(4), indexing="ij")
        px = ((I + dxp[D]) * dx).ravel()
        py = ((J + dyp[D]) * dx).ravel()
    else:
        px, py = samples[:, 0].copy(), samples[:, 1].copy()
    sx = px + x_min
    sy = py + y_min
    if typ in ("RECTANGLE", "ELLIPSE"):
        rot = release["rotation_deg"] * math.pi / 180.0
        c, s = math.cos(-rot), math.sin(-rot)
        dx0, dy0 = sx - release["center"][0], sy - release["center"][1]
        lx = c * dx0 - s * dy0
        ly = s * dx0 + c * dy0
        if typ == "RECTANGLE":
            keep = (np.abs(lx) <= release["Lx"] / 2.0) & (np.abs(ly) <= release["Ly"] / 2.0)
        else:
            keep = (lx / release["rx"]) ** 2 + (ly / release["ry"]) ** 2 <= 1.0
        hk = None
    else:
        hk = raster_height(release, sx, sy)
        keep = (hk >= release["h_min"]) & (hk > 0.0)
        hk = hk[keep]
    x = np.stack([sx[keep], sy[keep]], axis=1)
    n = len(x)
    h = np.full(n, float(release.get("h0", 0.0))) if hk is None else hk
    sum_h = float(np.cumsum(h)[-1]) if n else 0.0  # sequential sum, as the reference loop
    A_init = volume / sum_h
    A = np.full(n, A_init)
    mass = rho * h * A
    gn = terrain_gradient_norm(z, dx) if grad_norm is None else grad_norm
    ci = np.floor(x[:, 0] * ood).astype(np.int64)
    cj = np.floor(x[:, 1] * ood).astype(np.int64)
    if fast_theta:  # numpy's arctan (may differ from libm in the last bit); theta is recomputed by the step anyway
        theta = np.arctan(gn[ci, cj])
    else:
        cells, inv = np.unique(ci * z.shape[1] + cj, return_inverse=True)
        theta = libm_atan(gn.ravel()[cells])[inv]  # particleSlopeAngle (src/complex_terrain.cpp:113-120)
    # z by the 4x4 stencil of src/simulation.cpp:455-465
    zp = np.zeros(n)
    ib = (x[:, 0] * ood).astype(np.int64) - 1
    jb = (x[:, 1] * ood).astype(np.int64) - 1
    for a in range(4):
        for b in range(4):
            i = ib + a
            j = jb + b
            w = _N((x[:, 0] - i * dx) * ood) * _N((x[:, 1] - j * dx) * ood)
            zp = zp + z[i, j] * w
    return {"x": x, "z": zp, "v": np.zeros((n, 2)), "vz": np.zeros(n), "h": h, "A": A, "mass": mass, "theta": theta}


def raster_height(release: dict, px: np.ndarray, py: np.ndarray) -> np.ndarray:
    """Simulation::getReleaseHeightFromRaster (src/complex_terrain.cpp:132-183), vectorised."""
    rh = release["h"]
    cs = release["cellsize"]
    nx, ny = rh.shape
    x0, y0 = release["x0"], release["y0"]
    xr = px - x0
    yr = py - y0
    # the reference compares the relative position with the raster's last
    # absolute coordinate x.back(); the index test below is the binding one
    xlast = x0 + (nx - 1) * cs
    ylast = y0 + (ny - 1) * cs
    dxl = (x0 + cs) - x0
    dyl = (y0 + cs) - y0
    out = np.zeros_like(px)
    ok = (xr >= 0) & (yr >= 0) & (xr < xlast) & (yr < ylast)
    i = np.floor(xr / dxl).astype(np.int64)
    j = np.floor(yr / dyl).astype(np.int64)
    ok &= (i >= 0) & (j >= 0) & (i < nx - 1) & (j < ny - 1)
    i = np.where(ok, i, 0)
    j = np.where(ok, j, 0)
    fx = (xr - i * dxl) / dxl
    fy = (yr - j * dyl) / dyl
    z00, z10, z01, z11 = rh[i, j], rh[i + 1, j], rh[i, j + 1], rh[i + 1, j + 1]
    nd = release.get("nodata", -9999.0)
    bad = (np.abs(z00 - nd) < 1e-6) | (np.abs(z10 - nd) < 1e-6) | (np.abs(z01 - nd) < 1e-6) | (np.abs(z11 - nd) < 1e-6)
    z0 = z00 * (1.0 - fx) + z10 * fx
    z1 = z01 * (1.0 - fx) + z11 * fx
    hgt = z0 * (1.0 - fy) + z1 * fy
    hgt = np.where(hgt > 0.0, hgt, 0.0)
    return np.where(ok & ~bad, hgt, 0.0)


# ------------------------------------------------------------ terrains


def slope_arc_dem(Lx=2000.0, Ly=500.0, dx=5.0, angle_deg=35.0, x_break=1200.0, radius=100.0):
    """35-degree plane z = tan(35)(1200 - x) for x < 1200, blended into a flat
    runout by a circular arc of the given radius tangent to both (the arc's
    tangent points lie R tan(a/2) from the break on either side)."""
    a = math.radians(angle_deg)
    t = radius * math.tan(a / 2.0)
    x1 = x_break - t * math.cos(a)
    x2 = x_break + t
    nx = int(round(Lx / dx)) + 1
    ny = int(round(Ly / dx)) + 1
    x = np.arange(nx) * dx
    zx = np.where(x <= x1, math.tan(a) * (x_break - x),
                  np.where(x < x2, radius - np.sqrt(np.maximum(radius * radius - (x - x2) ** 2, 0.0)), 0.0))
    return np.repeat(zx[:, None], ny, axis=1)


def analytical_plane(Lx: float, Ly: float, dx: float):
    """The reference's hard-coded ANALYTICAL terrain (src/simulation.cpp:181-185):
    z = -x tan5 - y tan5 on generateGrid nodes (src/complex_terrain.cpp:67-82)."""
    def gen(L):
        g = [0.0]
        x, idx = 0.0, 0
        while x < L:
            idx += 1
            x = float(idx) * dx
            g.append(x)
        return np.array(g)
    xs, ys = gen(Lx), gen(Ly)
    th = 5.0 * math.pi / 180.0
    return -xs[:, None] * math.tan(th) - ys[None, :] * math.tan(th)


def fractal_slope_dem(n: int, dx: float, seed: int, rms: float = 15.0, hurst: float = 0.8, lowpass_m: float = 20.0,
                      x_plane_end: float = 2500.0, ease_m: float = 500.0, steep_deg: float = 30.0, flat_deg: float = 5.0,
                      rim_m: float = 0.0, rim_deg: float = 25.0):
    """Planar 30-degree slope for x < 2500 m easing (smoothstep in tan) to a
    5-degree runout over 500 m, plus seeded fBm roughness: spectrum
    PSD ~ k^-(2H+2), wavelengths shorter than lowpass_m removed, scaled to rms.

    rim_m > 0 adds a containing rim: the runout turns into a rim_deg
    counter-slope over the last rim_m metres in x, and rim_deg walls rise
    over the rim_m metres next to each y edge, so that no flow released
    away from them leaves the terrain (the reference indexes outside its
    arrays when one does, src/simulation.cpp:603-641)."""
    rng = np.random.default_rng(seed)
    L = n * dx
    x = np.arange(n) * dx
    s0, s1 = math.tan(math.radians(steep_deg)), math.tan(math.radians(flat_deg))
    u = np.clip((x - x_plane_end) / ease_m, 0.0, 1.0)
    slope = s0 + (s1 - s0) * (u * u * (3 - 2 * u))
    zx = -np.concatenate([[0.0], np.cumsum(0.5 * (slope[1:] + slope[:-1]) * dx)])
    zx -= zx.min()
    kx = np.fft.fftfreq(n, d=dx)
    ky = np.fft.rfftfreq(n, d=dx)
    K = np.sqrt(kx[:, None] ** 2 + ky[None, :] ** 2)
    amp = np.zeros_like(K)
    nz = K > 0
    amp[nz] = K[nz] ** (-(2 * hurst + 2) / 2.0)
    amp[K > 1.0 / lowpass_m] = 0.0
    amp[K < 1.0 / L] = 0.0
    ph = rng.standard_normal(K.shape) + 1j * rng.standard_normal(K.shape)
    rough = np.fft.irfft2(amp * ph, s=(n, n))
    rough *= rms / max(rough.std(), 1e-30)
    z = zx[:, None] + rough
    if rim_m > 0.0:
        t = math.tan(math.radians(rim_deg))
        z += (t * np.clip(x - (L - dx - rim_m), 0.0, None))[:, None]
        dist = np.minimum(x, (n - 1) * dx - x)  # y nodes: the same spacing
        z += (t * np.clip(rim_m - dist, 0.0, None))[None, :]
    return z


# ----------------------------------------------------------- releases


def poisson_disk_np(Lx: float, Ly: float, r: float, seed: int, rounds: int = 4) -> np.ndarray:
    """Poisson-disk samples in [0, Lx] x [0, Ly] with minimum distance r, by
    parallel dart throwing (numpy, seeded): a background grid of cells of
    edge r/sqrt(2) holds at most one sample each; the cells are visited in 9
    phase groups (i mod 3, j mod 3), whose cells are more than r apart, so
    one candidate per empty cell of a group can be tested against the
    accepted samples of its 5 x 5 neighbourhood all at once. `rounds` passes
    over the groups. Positions are relative to the lower-left corner, like
    the reference's sampler (src/poisson_disk_sampling.hpp:23-134) returns
    them; the sample set is a different one of the same kind."""
    rng = np.random.default_rng(seed)
    a = r / math.sqrt(2.0)
    nx, ny = int(math.ceil(Lx / a)), int(math.ceil(Ly / a))
    W = ny + 4  # row length of the grid with a 2-cell border of empty cells
    g = np.full(((nx + 4) * W, 2), np.nan)
    ci_all, cj_all = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    ci_all, cj_all = ci_all.ravel(), cj_all.ravel()
    grp = (ci_all % 3) * 3 + (cj_all % 3)
    flat_all = (ci_all + 2) * W + (cj_all + 2)
    groups = [np.nonzero(grp == k)[0] for k in range(9)]
    offs = np.array([di * W + dj for di in range(-2, 3) for dj in range(-2, 3) if (di, dj) != (0, 0)])
    r2 = r * r
    for _ in range(rounds):
        added = 0
        for k in range(9):
            idx = groups[k]
            idx = idx[np.isnan(g[flat_all[idx], 0])]
            groups[k] = idx  # filled cells leave the group for good
            if not len(idx):
                continue
            px = (ci_all[idx] + rng.random(len(idx))) * a
            py = (cj_all[idx] + rng.random(len(idx))) * a
            ok = (px <= Lx) & (py <= Ly)
            f = flat_all[idx]
            for o in offs:
                q = g[f + o]
                d2 = (q[:, 0] - px) ** 2 + (q[:, 1] - py) ** 2
                ok &= ~(d2 < r2)  # NaN (empty cell) compares false
            g[f[ok], 0] = px[ok]
            g[f[ok], 1] = py[ok]
            added += int(ok.sum())
        if added == 0:
            break
    keep = ~np.isnan(g[flat_all, 0])
    return g[flat_all[keep]]


def star_polygon(seed: int, center, ax: float, ay: float, nvert: int = 12):
    rng = np.random.default_rng(seed)
    ang = np.sort(rng.uniform(0, 2 * np.pi, nvert))
    r = rng.uniform(0.6, 1.0, nvert)
    return np.stack([center[0] + ax * r * np.cos(ang), center[1] + ay * r * np.sin(ang)], axis=1)


def point_in_polygon(px, py, poly):
    """Even-odd rule (the algorithm of src/polygon_tools.cpp), vectorised."""
    inside = np.zeros(px.shape, dtype=bool)
    n = len(poly)
    j = n - 1
    for i in range(n):
        xi, yi = poly[i]
        xj, yj = poly[j]
        cond = ((yi > py) != (yj > py)) & (px < (xj - xi) * (py - yi) / (yj - yi + 1e-300) + xi)
        inside ^= cond
        j = i
    return inside


def lognormal_release_raster(seed: int, poly, cellsize: float, median: float = 1.5, sigma_log: float = 0.4, corr_m: float = 10.0):
    """RASTER release covering the polygon: lognormal heights (median, sigma_log)
    from a smooth seeded Gaussian field, zero (below h_min) outside the polygon."""
    rng = np.random.default_rng(seed)
    x0, y0 = np.floor(poly.min(axis=0) / cellsize) * cellsize - 2 * cellsize
    x1, y1 = np.ceil(poly.max(axis=0) / cellsize) * cellsize + 2 * cellsize
    nx = int(round((x1 - x0) / cellsize)) + 1
    ny = int(round((y1 - y0) / cellsize)) + 1
    g = rng.standard_normal((nx, ny))
    kx = np.fft.fftfreq(nx, d=cellsize)
    ky = np.fft.fftfreq(ny, d=cellsize)
    filt = np.exp(-0.5 * (2 * np.pi * corr_m) ** 2 * (kx[:, None] ** 2 + ky[None, :] ** 2))
    g = np.real(np.fft.ifft2(np.fft.fft2(g) * filt))
    g /= max(g.std(), 1e-30)
    h = np.exp(math.log(median) + sigma_log * g)
    X = x0 + np.arange(nx)[:, None] * cellsize + 0 * np.arange(ny)[None, :]
    Y = y0 + 0 * np.arange(nx)[:, None] + np.arange(ny)[None, :] * cellsize
    inside = point_in_polygon(X, Y, poly)
    h = np.where(inside, h, 0.0)
    return {"type": "RASTER", "h": h, "x0": float(x0), "y0": float(y0), "cellsize": cellsize, "nodata": -9999.0}


# ------------------------------------------------------------ configs

# containing rim of the benchmark DEMs (fractal_slope_dem rim_m): metres of
# counter-slope at the far x end and of side wall at each y edge
RIM_M = 300.0


def config1():
    """35-degree slope with circular-arc runout, 1 600 particles, Coulomb."""
    z = slope_arc_dem()
    cfg = dict(gravity=9.81, rho=300.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0, total_time=60.0,
               friction="COULOMB", coulomb_mu=0.4)
    rel = {"type": "RECTANGLE", "center": (150.0, 250.0), "Lx": 100.0, "Ly": 100.0, "rotation_deg": 0.0, "h0": 2.0}
    P = release_particles(z, 5.0, rel, cfg["rho"])
    return {"name": "slope35_arc_401x101_dx5", "z": z, "dx": 5.0, "cfg": cfg, "release": rel, "particles": P}


def config2(seed: int = 2026, sampler=poisson_disk_np):
    """4096^2 DEM at 1 m (30-degree slope easing to 5 degrees + fBm roughness,
    Hurst 0.8, 15 m RMS, wavelengths < 20 m removed), seeded 12-vertex
    star-convex release polygon with ~500 x 300 m semi-axes rasterised with
    lognormal heights (median 1.5 m, sigma_log 0.4, h_min 0.2 m), POISSON
    sampling at r = 0.5 m (~0.55-0.6 M particles), Voellmy mu=0.2 xi=1500,
    total_time 120 s. `sampler(Lx, Ly, r, seed)` returns the Poisson-disk
    samples (default: poisson_disk_np, numpy only)."""
    dx = 1.0
    z = fractal_slope_dem(4096, dx, seed=seed, rim_m=RIM_M)
    poly = star_polygon(seed + 1, center=(700.0, 2048.0), ax=500.0, ay=300.0)
    rel = lognormal_release_raster(seed + 2, poly, cellsize=dx)
    rel["h_min"] = 0.2
    cfg = dict(gravity=9.81, rho=300.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0, total_time=120.0,
               friction="VOELLMY", voellmy_mu=0.2, voellmy_xi=1500.0)
    h = rel["h"]
    Lx = (h.shape[0] - 1) * dx
    Ly = (h.shape[1] - 1) * dx
    samples = sampler(Lx, Ly, 0.5, seed + 3)
    P = release_particles(z, dx, rel, cfg["rho"], sampling="GIVEN", samples=samples)
    return {"name": "fractal4096_dx1_star_poisson_voellmy", "z": z, "dx": dx, "cfg": cfg, "release": rel, "particles": P}


def config3_dem(seed: int = 2027):
    """The 8192^2, 0.5 m DEM of config 3 (and of the served stream, config 5)."""
    return fractal_slope_dem(8192, 0.5, seed=seed, rms=7.5, rim_m=RIM_M)


def config3(seed: int = 2027):
    """8192^2 DEM at 0.5 m (same construction, roughness amplitude scaled to
    7.5 m RMS), 1200 x 800 m ellipse h0 = 3 m, UNIFORM 2x2 sampling
    (~12 M particles), mu(I) (0.38, 0.64, 0.279, d 0.5 mm, phi 0.6), rho 1500,
    total_time 90 s."""
    dx = 0.5
    z = config3_dem(seed)
    cfg = dict(gravity=9.81, rho=1500.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0, total_time=90.0,
               friction="MU_I", mui_mu1=0.38, mui_mu2=0.64, mui_I0=0.279, mui_d=5e-4, mui_phi=0.6)
    rel = {"type": "ELLIPSE", "center": (800.0, 2048.0), "rx": 600.0, "ry": 400.0, "rotation_deg": 0.0, "h0": 3.0}
    P = release_particles(z, dx, rel, cfg["rho"], fast_theta=True)
    return {"name": "fractal8192_dx05_ellipse_uniform_mui", "z": z, "dx": dx, "cfg": cfg, "release": rel, "particles": P}


def config3_small(seed: int = 2027):
    """A smaller case of config 3 for kernel captures: the same construction
    on a 4096^2 DEM at 0.5 m, a 900 x 600 m ellipse (h0 = 3 m, ~6.8 M
    particles, more than the L2 holds), mu(I) as config 3."""
    dx = 0.5
    z = fractal_slope_dem(4096, dx, seed=seed, rms=7.5, rim_m=RIM_M)
    cfg = dict(gravity=9.81, rho=1500.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0, total_time=90.0,
               friction="MU_I", mui_mu1=0.38, mui_mu2=0.64, mui_I0=0.279, mui_d=5e-4, mui_phi=0.6)
    rel = {"type": "ELLIPSE", "center": (700.0, 1024.0), "rx": 450.0, "ry": 300.0, "rotation_deg": 0.0, "h0": 3.0}
    P = release_particles(z, dx, rel, cfg["rho"], fast_theta=True)
    return {"name": "fractal4096_dx05_ellipse_uniform_mui", "z": z, "dx": dx, "cfg": cfg, "release": rel, "particles": P}


def config4(n_scenarios: int = 256, seed: int = 2028, particles: bool = True):
    """Ensemble on a shared 2048^2 DEM at 2 m (fractal-slope construction,
    roughness 7.5 m RMS): elliptical releases with semi-axes U(20, 300) m,
    centres uniform in the upper third, h0 U(0.5, 3) m, UNIFORM 2x2 sampling
    (1.9 k - 265 k particles, 20.7 M in all), Voellmy with mu U(0.1, 0.4),
    xi U(500, 3000), total_time 60 s; the other parameters as the 35-degree
    slope case (rho 300, C_cfl 0.5, dt_max 0.01 s, flip_ratio 0.95).
    Scenarios are (cfg, particles), or (cfg, release) with particles=False
    (the release is then built where it runs, e.g. on the device; the same
    random draws give the same releases either way)."""
    dx = 2.0
    n = 2048
    z = fractal_slope_dem(n, dx, seed=seed, rms=7.5, rim_m=RIM_M)
    gn = terrain_gradient_norm(z, dx) if particles else None
    rng = np.random.default_rng(seed + 1)
    L = n * dx
    out = []
    for k in range(n_scenarios):
        rx, ry = rng.uniform(20.0, 300.0, 2)
        rot = rng.uniform(0.0, 180.0)
        r = max(rx, ry) + 4 * dx
        cx = rng.uniform(r, max(r + 1.0, L / 3.0))
        cy = rng.uniform(r + RIM_M, L - r - RIM_M)  # clear of the side walls
        cfg = dict(gravity=9.81, rho=300.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0, total_time=60.0,
                   friction="VOELLMY", voellmy_mu=float(rng.uniform(0.1, 0.4)), voellmy_xi=float(rng.uniform(500.0, 3000.0)))
        rel = {"type": "ELLIPSE", "center": (float(cx), float(cy)), "rx": float(rx), "ry": float(ry), "rotation_deg": float(rot),
               "h0": float(rng.uniform(0.5, 3.0))}
        out.append((cfg, release_particles(z, dx, rel, cfg["rho"], fast_theta=True, grad_norm=gn) if particles else rel))
    return {"name": f"ensemble{n_scenarios}_fractal2048_dx2_voellmy", "z": z, "dx": dx, "scenarios": out}


def release_particle_estimate(rel: dict, dx: float) -> int:
    """About how many particles UNIFORM 2x2 sampling gives an ELLIPSE or
    RECTANGLE release (4 per covered cell), for balancing work before the
    particles exist."""
    if rel["type"] == "ELLIPSE":
        area = np.pi * rel["rx"] * rel["ry"]
    else:
        area = rel["Lx"] * rel["Ly"]
    return int(round(4.0 * area / (dx * dx)))


def config5_stream(z: np.ndarray, dx: float, window_s: float, seed: int = 2029, rate: float = 20.0, median: float = 20000.0,
                   sigma_log: float = 1.0, cap: int = 2_000_000, t_range=(30.0, 120.0), particles: bool = True):
    """Poisson arrivals at `rate` per second over `window_s` seconds of requests
    on DEM z: particle count lognormal (median, sigma_log) capped at `cap`, an
    ellipse of area N/16 m^2 (UNIFORM at 0.5 m) with random aspect and
    position in the upper third, friction law uniform over COULOMB / VOELLMY /
    MU_I with coefficients from the ranges of the other workloads, total_time
    uniform in t_range. Returns (arrival time, cfg, particles) per request,
    or (arrival time, cfg, release) with particles=False (the release is then
    built where it runs, e.g. on the device)."""
    rng = np.random.default_rng(seed)
    gn = terrain_gradient_norm(z, dx)
    L = z.shape[0] * dx
    t = 0.0
    reqs = []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window_s:
            break
        N = int(min(cap, rng.lognormal(math.log(median), sigma_log)))
        area = N / (4.0 / (dx * dx))
        aspect = rng.uniform(1.0, 2.5)
        rx = math.sqrt(area * aspect / math.pi)
        ry = area / (math.pi * rx)
        r = max(rx, ry) + 4 * dx
        cx = rng.uniform(r, max(r + 1.0, L / 3.0))
        cy = rng.uniform(r + RIM_M, z.shape[1] * dx - r - RIM_M)  # clear of the side walls
        law = ["COULOMB", "VOELLMY", "MU_I"][int(rng.integers(3))]
        cfg = dict(gravity=9.81, rho=1500.0, C_cfl=0.5, dt_max=0.01, flip_ratio=0.95, output_dt=1.0,
                   total_time=float(rng.uniform(*t_range)), friction=law)
        if law == "COULOMB":
            cfg["coulomb_mu"] = float(rng.uniform(0.3, 0.6))
        elif law == "VOELLMY":
            cfg.update(voellmy_mu=float(rng.uniform(0.1, 0.4)), voellmy_xi=float(rng.uniform(500.0, 3000.0)))
        else:
            cfg.update(mui_mu1=float(rng.uniform(0.3, 0.45)), mui_mu2=float(rng.uniform(0.55, 0.7)), mui_I0=0.279, mui_d=5e-4, mui_phi=0.6)
        rel = {"type": "ELLIPSE", "center": (float(cx), float(cy)), "rx": rx, "ry": ry, "rotation_deg": float(rng.uniform(0, 180)),
               "h0": float(rng.uniform(0.5, 3.0))}
        reqs.append((t, cfg, release_particles(z, dx, rel, cfg["rho"], fast_theta=True, grad_norm=gn) if particles else rel))
    return reqs
