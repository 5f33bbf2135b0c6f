"""Seeded synthetic basins for the barotropic step.

No dataset is involved: every basin is generated from a seed with
numpy.random.default_rng.  The generators fill a Basin with the T mask lu,
metrics, Coriolis, rest depth, wind stress on T points, viscosity, drag and
time step; the derived masks (gridcon) and the wind forcing (surface stress
and RHS assembly) are computed afterwards by a backend, on the GPU for the
product and by the CPU oracle in tests, see ``finalize``.

Workloads (sizes are significant points):
  beta_plane_basin   256x256, 10 km, beta plane, bumpy 4000 m basin
  regional_basin     2048x1536, 1 km, fractal coastline (~40 % land),
                     log-normal shallow depth, smooth random wind
  ridge_basin        4096x4096, 2 km, 4000 m with a 200 m-rms ridge
  spherical_basin    lat-lon grid with the reference's spherical metrics
  williamson2_basin  Williamson et al.'s shallow-water test 2 on a
                     zonally periodic lat-lon band (analytic steady state)
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .grid import Basin, Bounds, Consts, METRICS

# Service/basin_parameters.f90:160: the literal 3.1415926535897 has no d0
# suffix, so Fortran stores it in single precision before dividing by 180d0.
DPIP180 = float(np.float32(3.1415926535897)) / 180.0
RAD_EARTH = 6371000.0              # Inc/basinpar.fi:73
EARTH_ANG_VEL = 7.292115974546454e-5  # Inc/basinpar.fi:74


def _set_metric_range(basin: Basin, values: dict) -> None:
    """Metrics are set on nx_start-1..nx_end+1 x ny_start-1..ny_end+1 and
    left zero outside, as basinpar does (Service/basin_parameters.f90:249-296)."""
    b = basin.bounds
    s = b.sl(b.nx_start - 1, b.nx_end + 1, b.ny_start - 1, b.ny_end + 1)
    for k in METRICS:
        arr = b.zeros()
        v = values[k]
        arr[s] = v if np.isscalar(v) else v[s]
        basin.metrics[k] = arr


def uniform_metrics(basin: Basin, spacing: float) -> None:
    _set_metric_range(basin, {k: spacing for k in METRICS})


def _y_of_rows(b: Bounds, spacing: float, offset: float) -> np.ndarray:
    """y of row n (T rows for offset 0, h/v rows for offset 0.5) measured
    from the centre of the significant area."""
    n = np.arange(b.bnd_y1, b.bnd_y2 + 1, dtype=np.float64)
    y = (n - b.nnn + offset) * spacing
    return y - 0.5 * (b.ny - 1) * spacing


def _interior_mask(b: Bounds) -> np.ndarray:
    lu = b.zeros(np.float32)
    lu[b.interior] = 1.0
    return lu


def _gaussian_field(rng, shape, corr_cells: float) -> np.ndarray:
    """Zero-mean, unit-variance Gaussian random field with a Gaussian
    correlation of length corr_cells (FFT filter of white noise)."""
    nx, ny = shape
    w = rng.standard_normal((nx, ny))
    kx = np.fft.fftfreq(nx)[:, None]
    ky = np.fft.fftfreq(ny)[None, :]
    filt = np.exp(-0.5 * (2 * math.pi) ** 2 * (kx ** 2 + ky ** 2) * corr_cells ** 2)
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def _fbm(rng, shape, slope: float = 3.0) -> np.ndarray:
    """Fractal (fBm-like) noise: white noise with a k^(-slope/2) spectrum."""
    nx, ny = shape
    w = rng.standard_normal((nx, ny))
    kx = np.fft.fftfreq(nx)[:, None]
    ky = np.fft.fftfreq(ny)[None, :]
    k = np.sqrt(kx ** 2 + ky ** 2)
    k[0, 0] = 1.0
    amp = k ** (-slope / 2.0)
    amp[0, 0] = 0.0
    return np.real(np.fft.ifft2(np.fft.fft2(w) * amp))


def _largest_ocean(ocean: np.ndarray) -> np.ndarray:
    """Keep the largest 4-connected ocean component (integer labelling)."""
    from scipy import ndimage
    lab, nlab = ndimage.label(ocean, structure=[[0, 1, 0], [1, 1, 1], [0, 1, 0]])
    if nlab == 0:
        return ocean
    sizes = np.bincount(lab.ravel())
    sizes[0] = 0
    return lab == int(np.argmax(sizes))


def beta_plane_basin(n: int = 256, spacing: float = 1.0e4, f0: float = 1.0e-4,
                     beta: float = 2.0e-11, depth: float = 4000.0, nbumps: int = 16,
                     bump_amp: float = 1500.0, bump_sigma: float = 5.0,
                     tau0: float = 0.1, visc: float = 1.0e3, drag: float = 1.0e-6,
                     dt: float = 15.0, seed: int = 0, ny: Optional[int] = None) -> Basin:
    """Closed rectangular C-grid basin on a beta plane: a 1-point land ring
    inside the significant area, depth `depth` minus `nbumps` seeded Gaussian
    bumps (amplitude U(0, bump_amp), sigma `bump_sigma` points), zonal wind
    stress tau0*cos(pi*y/Ly) with y from the basin centre, Laplacian
    viscosity `visc`, linear drag `drag` through the Rayleigh term, rest.

    dt defaults to 15 s: leap-frog on the C grid is stable only for
    2*c*dt*sqrt(1/dx^2+1/dy^2) <= 1 (c = sqrt(g*H)), which 20 s violates at
    4000 m and 10 km (1.12): the checkerboard gravity wave then grows until
    the range guard trips.  ``cfl_number`` evaluates the criterion."""
    rng = np.random.default_rng(seed)
    ny = n if ny is None else ny
    b = Bounds.serial(n, ny)
    basin = Basin(b, Consts())
    lu = b.zeros(np.float32)
    lu[b.sl(b.nx_start + 1, b.nx_end - 1, b.ny_start + 1, b.ny_end - 1)] = 1.0
    basin.masks["lu"] = lu
    uniform_metrics(basin, spacing)
    yh = _y_of_rows(b, spacing, 0.5)
    basin.rlh_s = np.asfortranarray(np.broadcast_to(f0 + beta * yh[None, :], b.shape).copy())
    m = np.arange(b.bnd_x1, b.bnd_x2 + 1, dtype=np.float64)[:, None]
    nn = np.arange(b.bnd_y1, b.bnd_y2 + 1, dtype=np.float64)[None, :]
    h = np.full(b.shape, depth)
    cm = rng.uniform(b.nx_start, b.nx_end, nbumps)
    cn = rng.uniform(b.ny_start, b.ny_end, nbumps)
    amp = rng.uniform(0.0, bump_amp, nbumps)
    for k in range(nbumps):
        h -= amp[k] * np.exp(-((m - cm[k]) ** 2 + (nn - cn[k]) ** 2) / (2.0 * bump_sigma ** 2))
    h = np.maximum(h, 100.0)
    basin.hhq_rest = np.asfortranarray(np.where(lu > 0.5, h, 0.0))
    Ly = b.ny * spacing
    yt = _y_of_rows(b, spacing, 0.0)
    basin.taux = np.asfortranarray(np.broadcast_to(tau0 * np.cos(math.pi * yt / Ly)[None, :], b.shape).copy())
    basin.tauy = b.zeros()
    basin.forcing["mu"] = np.full(b.shape, visc, order="F")
    basin.forcing["rdis"] = np.full(b.shape, drag, order="F")
    basin.dt = dt
    basin.info.update(workload="beta_plane_basin", n=n, ny=ny, spacing=spacing, seed=seed,
                      nbumps=nbumps, f0=f0, beta=beta, visc=visc, drag=drag)
    return basin.fill_defaults()


def regional_basin(nx: int = 2048, ny: int = 1536, spacing: float = 1.0e3,
                   land_frac: float = 0.4, median_depth: float = 60.0,
                   depth_sigma: float = 0.8, wind_corr: float = 5.0e4, wind_rms: float = 0.08,
                   f0: float = 1.0e-4, beta: float = 2.0e-11, visc: float = 1.0e3,
                   drag: float = 1.0e-6, dt: float = 2.0, seed: int = 1) -> Basin:
    """Regional shelf basin: coastline from seeded fractal noise thresholded
    at `land_frac` with only the largest 4-connected ocean kept, log-normal
    depth (median `median_depth`, clipped to 5..300 m, 3-point box smoothing),
    spatially smooth random wind stress (Gaussian correlation `wind_corr`,
    rms `wind_rms` per component).  The wind's 6-hour cycle is applied as a
    per-substep amplitude (``wind_cycle``)."""
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    b = Bounds.serial(nx, ny)
    basin = Basin(b, Consts())
    noise = _fbm(rng, (nx, ny))
    # threshold so that the land fraction after dropping the small ocean
    # components is close to land_frac (a few bisection steps)
    lo, hi = 0.0, land_frac
    for _ in range(8):
        q = 0.5 * (lo + hi)
        ocean = _largest_ocean(noise > np.quantile(noise, q))
        if 1.0 - ocean.mean() > land_frac:
            hi = q
        else:
            lo = q
    ocean = _largest_ocean(noise > np.quantile(noise, lo))
    lu = b.zeros(np.float32)
    lu[b.interior] = ocean.astype(np.float32)
    basin.masks["lu"] = lu
    uniform_metrics(basin, spacing)
    yh = _y_of_rows(b, spacing, 0.5)
    basin.rlh_s = np.asfortranarray(np.broadcast_to(f0 + beta * yh[None, :], b.shape).copy())
    h = np.exp(math.log(median_depth) + depth_sigma * rng.standard_normal((nx, ny)))
    h = np.clip(h, 5.0, 300.0)
    h = np.clip(ndimage.uniform_filter(h, size=3, mode="nearest"), 5.0, 300.0)
    hr = b.zeros()
    hr[b.interior] = np.where(ocean, h, 0.0)
    basin.hhq_rest = hr
    corr = wind_corr / spacing
    taux, tauy = b.zeros(), b.zeros()
    taux[b.interior] = wind_rms * _gaussian_field(rng, (nx, ny), corr)
    tauy[b.interior] = wind_rms * _gaussian_field(rng, (nx, ny), corr)
    basin.taux, basin.tauy = taux, tauy
    basin.forcing["mu"] = np.full(b.shape, visc, order="F")
    basin.forcing["rdis"] = np.full(b.shape, drag, order="F")
    basin.dt = dt
    basin.info.update(workload="regional_basin", nx=nx, ny=ny, spacing=spacing, seed=seed,
                      land_fraction=float(1.0 - ocean.mean()), visc=visc, drag=drag,
                      wind_period_s=6 * 3600.0)
    return basin.fill_defaults()


def wind_cycle(nsub: int, dt: float, t0: float = 0.0, period: float = 6 * 3600.0) -> np.ndarray:
    """Per-substep wind amplitude cos(2*pi*t/period) at t = t0 + k*dt."""
    t = t0 + dt * np.arange(nsub, dtype=np.float64)
    return np.cos(2.0 * math.pi * t / period)


def ridge_basin(n: int = 4096, spacing: float = 2.0e3, depth: float = 4000.0,
                ridge_rms: float = 200.0, tau0: float = 0.1, f0: float = 1.0e-4,
                beta: float = 2.0e-11, visc: float = 1.0e3, drag: float = 1.0e-6,
                dt: float = 3.0, seed: int = 2) -> Basin:
    """Double-gyre basin: flat `depth` with a meandering meridional ridge of
    `ridge_rms` rms height, wind as beta_plane_basin scaled to the basin."""
    rng = np.random.default_rng(seed)
    b = Bounds.serial(n, n)
    basin = Basin(b, Consts())
    lu = b.zeros(np.float32)
    lu[b.sl(b.nx_start + 1, b.nx_end - 1, b.ny_start + 1, b.ny_end - 1)] = 1.0
    basin.masks["lu"] = lu
    uniform_metrics(basin, spacing)
    yh = _y_of_rows(b, spacing, 0.5)
    basin.rlh_s = np.asfortranarray(np.broadcast_to(f0 + beta * yh[None, :], b.shape).copy())
    x = np.arange(n, dtype=np.float64)[:, None]
    axis = 0.5 * n + 0.1 * n * _gaussian_field(rng, (1, n), n / 8.0)[0][None, :]
    crest = 1.0 + 0.3 * _gaussian_field(rng, (1, n), n / 16.0)[0][None, :]
    width = n / 40.0
    r = crest * np.exp(-0.5 * ((x - axis) / width) ** 2)
    r *= ridge_rms / np.sqrt(np.mean(r ** 2))
    hr = b.zeros()
    hr[b.interior] = depth - r
    basin.hhq_rest = np.asfortranarray(np.where(lu > 0.5, hr, 0.0))
    Ly = b.ny * spacing
    yt = _y_of_rows(b, spacing, 0.0)
    basin.taux = np.asfortranarray(np.broadcast_to(tau0 * np.cos(math.pi * yt / Ly)[None, :], b.shape).copy())
    basin.tauy = b.zeros()
    basin.forcing["mu"] = np.full(b.shape, visc, order="F")
    basin.forcing["rdis"] = np.full(b.shape, drag, order="F")
    basin.dt = dt
    basin.info.update(workload="ridge_basin", n=n, spacing=spacing, seed=seed,
                      ridge_rms=ridge_rms, visc=visc, drag=drag)
    return basin.fill_defaults()


def spherical_metrics(basin: Basin, rlon: float, rlat: float, dxst: float, dyst: float,
                      rotation_on_lat: float = 0.0) -> None:
    """Metrics and Coriolis of an undistorted spherical grid
    (curve_grid = 1), restating Service/basin_parameters.f90:163-296 for a
    regular grid and grid_parameters_spherical (:836-949) for the metric
    factor cos(lat) and the Coriolis sine; rotation_on_lon = 0."""
    b = basin.bounds
    m = np.arange(b.bnd_x1, b.bnd_x2 + 1, dtype=np.float64)
    n = np.arange(b.bnd_y1, b.bnd_y2 + 1, dtype=np.float64)
    xt = rlon + (m - b.mmm) * dxst
    yt = rlat + (n - b.nnn) * dyst
    xu = np.empty_like(xt); xu[:-1] = (xt[:-1] + xt[1:]) / 2.0; xu[-1] = 0.0
    yv = np.empty_like(yt); yv[:-1] = (yt[:-1] + yt[1:]) / 2.0; yv[-1] = 0.0
    stepx = dxst * DPIP180 * RAD_EARTH
    stepy = dyst * DPIP180 * RAD_EARTH
    lat_extr = 89.99999
    sinlat_extr = math.sin(DPIP180 * lat_extr)
    rot = DPIP180 * rotation_on_lat

    def factors(x, y):
        lat_mod = np.clip(y, -lat_extr, lat_extr)
        sin_lat = (np.sin(DPIP180 * y)[None, :] * math.cos(rot)
                   + np.cos(DPIP180 * x)[:, None] * np.cos(DPIP180 * y)[None, :] * math.sin(rot))
        sin_lat = np.clip(sin_lat, -sinlat_extr, sinlat_extr)
        return np.broadcast_to(np.cos(DPIP180 * lat_mod)[None, :], (len(x), len(y))), sin_lat

    vals = {}
    cx_t, _ = factors(xt, yt)       # T grid: dx, dy
    cx_u, _ = factors(xu, yt)       # U grid: dxt, dyh
    cx_v, _ = factors(xt, yv)       # V grid: dxh, dyt
    cx_h, sin_h = factors(xu, yv)   # H grid: dxb, dyb, Coriolis
    vals["dx"] = stepx * cx_t
    vals["dxt"] = stepx * cx_u
    vals["dxh"] = stepx * cx_v
    vals["dxb"] = stepx * cx_h
    for k in ("dy", "dyt", "dyh", "dyb"):
        vals[k] = np.full(b.shape, stepy)
    _set_metric_range(basin, vals)
    rlh = np.full(b.shape, 2.0 * EARTH_ANG_VEL)
    s = b.sl(b.nx_start - 1, b.nx_end + 1, b.ny_start - 1, b.ny_end + 1)
    rlh[s] = rlh[s] * sin_h[s]
    basin.rlh_s = np.asfortranarray(rlh)


def spherical_basin(nx: int = 48, ny: int = 32, rlon: float = 27.5, rlat: float = 40.9,
                    dxst: float = 0.25, dyst: float = 0.2, depth: float = 1500.0,
                    rotation_on_lat: float = 0.0, tau0: float = 0.1, visc: float = 1.0e3,
                    drag: float = 1.0e-6, dt: float = 30.0, seed: int = 3) -> Basin:
    """A small lat-lon basin with the reference's spherical metrics (metrics
    vary along y, Coriolis too; with rotation_on_lat != 0 Coriolis also
    varies along x), random coastline and depth."""
    rng = np.random.default_rng(seed)
    b = Bounds.serial(nx, ny)
    basin = Basin(b, Consts())
    ocean = _largest_ocean(_gaussian_field(rng, (nx, ny), 3.0) > -0.6)
    lu = b.zeros(np.float32)
    lu[b.interior] = ocean.astype(np.float32)
    basin.masks["lu"] = lu
    spherical_metrics(basin, rlon, rlat, dxst, dyst, rotation_on_lat)
    hr = b.zeros()
    hr[b.interior] = np.where(ocean, depth * (0.6 + 0.4 * rng.random((nx, ny))), 0.0)
    basin.hhq_rest = hr
    yt = _y_of_rows(b, 1.0, 0.0)
    basin.taux = np.asfortranarray(np.broadcast_to(tau0 * np.cos(math.pi * yt / b.ny)[None, :], b.shape).copy())
    basin.tauy = np.asfortranarray(0.3 * tau0 * _gaussian_field(rng, b.shape, 4.0))
    basin.forcing["mu"] = np.full(b.shape, visc, order="F")
    basin.forcing["rdis"] = np.full(b.shape, drag, order="F")
    basin.dt = dt
    basin.info.update(workload="spherical_basin", nx=nx, ny=ny, seed=seed,
                      rotation_on_lat=rotation_on_lat)
    return basin.fill_defaults()


WILLIAMSON2_DEPTH = 3000.0        # g*h0 = 2.94e4 m^2/s^2 with g = 9.8
WILLIAMSON2_U0 = 2.0 * math.pi * RAD_EARTH / (12.0 * 86400.0)


def williamson2_fields(basin: Basin):
    """Analytic state of Williamson et al.'s shallow-water test 2 with
    alpha = 0 (steady zonal geostrophic flow) on the basin's T rows and u
    points: eta = -(R*Omega*u0 + u0^2/2) sin^2(lat)/g, u = u0 cos(lat),
    v = 0, with the latitude of each T row as the grid set-up gives it.
    Returns (eta, u) as full arrays, zero off the lu / lcu masks."""
    b = basin.bounds
    info = basin.info
    n = np.arange(b.bnd_y1, b.bnd_y2 + 1, dtype=np.float64)
    lat = info["rlat"] + (n - b.nnn) * info["dyst"]
    s = np.sin(DPIP180 * lat)
    g = basin.consts.free_fall_acc
    u0 = WILLIAMSON2_U0
    eta = -(RAD_EARTH * EARTH_ANG_VEL * u0 + 0.5 * u0 * u0) * s * s / g
    uu = u0 * np.cos(DPIP180 * lat)
    m = basin.masks
    eta2 = np.asfortranarray(np.broadcast_to(eta[None, :], b.shape) * (m["lu"] > 0.5))
    u2 = np.asfortranarray(np.broadcast_to(uu[None, :], b.shape) * (m["lcu"] > 0.5))
    return eta2, u2


def williamson2_basin(dlon: float = 2.5, dlat: float = 2.0, lat_max: float = 80.0,
                      dt: Optional[float] = None, backend=None) -> Basin:
    """Williamson et al.'s shallow-water test 2 (alpha = 0) on the
    reference's spherical grid: a zonally periodic lat-lon band of dlon x
    dlat degrees between -lat_max and lat_max, closed by land rows (the
    exact solution has v = 0, so the walls are consistent with it), flat
    rest depth 3000 m, no viscosity, drag, wind or water flux; the state
    starts at the analytic solution (williamson2_fields) at both time
    levels.  The test the thesis of the reference reports (dipl. p.27):
    relative max-norm error of the level after 5 days, 6.93e-6 on 2.5 x 2.0
    degrees and 1.74e-6 on 1.25 x 1.0.  dt defaults to 60 s per degree of
    latitude spacing (gravity-wave stability number 0.83 for the rest depth
    at the band's edge, 0.52 for the depth there).  backend (gridcon) derives the masks; the state is set
    when it is given."""
    nx = int(round(360.0 / dlon))
    ny = int(round(2.0 * lat_max / dlat))
    b = Bounds.serial(nx, ny, periodicity_x=1)
    basin = Basin(b, Consts())
    lu = b.zeros(np.float32)
    lu[:, b.nnn - b.bnd_y1:b.nn - b.bnd_y1 + 1] = 1.0   # every column: the wrap sees ocean
    basin.masks["lu"] = lu
    rlon, rlat = 0.5 * dlon, -lat_max + 0.5 * dlat
    spherical_metrics(basin, rlon, rlat, dlon, dlat)
    basin.hhq_rest = np.asfortranarray(np.where(lu > 0.5, WILLIAMSON2_DEPTH, 0.0))
    basin.dt = 60.0 * dlat if dt is None else dt
    basin.info.update(workload="williamson2", nx=nx, ny=ny, rlon=rlon, rlat=rlat, dxst=dlon,
                      dyst=dlat, lat_max=lat_max)
    basin.fill_defaults()
    if backend is not None:
        basin.masks.update(backend.gridcon(b, lu))
        eta, u = williamson2_fields(basin)
        for k in ("ssh_e", "sshp_e"):
            basin.state[k][...] = eta
        for k in ("ubrtr_e", "ubrtrp_e"):
            basin.state[k][...] = u
        # the periodic wrap of the initial state (cyclize8_x): gridcon leaves
        # the u mask of the last ring column at land, the wrap fills it
        i0, i1 = b.mmm - b.bnd_x1, b.mm - b.bnd_x1
        for a in basin.state.values():
            a[i0 - 1], a[i1 + 1] = a[i1].copy(), a[i0].copy()
    return basin


def williamson2_error(basin: Basin) -> float:
    """max |h - h_T| / max h_T over the ocean points, h = rest depth + level
    (the thesis's l_inf of the level, normalised by the analytic depth)."""
    b = basin.bounds
    eta, _ = williamson2_fields(basin)
    ocean = basin.masks["lu"][b.interior] > 0.5
    err = np.abs(basin.state["ssh_e"][b.interior] - eta[b.interior])[ocean].max()
    return float(err / (basin.hhq_rest[b.interior] + eta[b.interior])[ocean].max())


def cfl_number(basin: Basin) -> float:
    """2*c*dt*sqrt(1/dx^2+1/dy^2) at the deepest ocean point: the leap-frog
    C-grid gravity-wave stability number (must stay below 1)."""
    b = basin.bounds
    ocean = basin.masks["lu"][b.interior] > 0.5
    h = float(basin.hhq_rest[b.interior][ocean].max())
    dx = basin.metrics["dx"][b.interior][ocean]
    dy = basin.metrics["dy"][b.interior][ocean]
    inv = float(np.sqrt(1.0 / dx ** 2 + 1.0 / dy ** 2).max())
    return 2.0 * math.sqrt(basin.consts.free_fall_acc * h) * basin.dt * inv


def finalize(basin: Basin, backend) -> Basin:
    """Derive the masks (gridcon) and the wind forcing RHSx/RHSy with
    `backend`, which provides gridcon(bounds, lu) -> dict of masks and
    wind_forcing(basin) -> (RHSx, RHSy): the CUDA library for the product,
    the CPU oracle in tests."""
    masks = backend.gridcon(basin.bounds, basin.masks["lu"])
    basin.masks.update(masks)
    if basin.taux is not None:
        rx, ry = backend.wind_forcing(basin)
        basin.forcing["RHSx"], basin.forcing["RHSy"] = rx, ry
    return basin


def vertical_grid(nz: int, seed: int = 0):
    """Sigma-level thicknesses dz (nz, summing to 1) and interface spacings
    hzt (nz + 1: half layers at the surface and the bottom, the mean of the
    two layers between), the steps Service/basin_parameters.f90:113-121
    (vgrid) derives from the level depths; the thicknesses are seeded and
    uneven."""
    rng = np.random.default_rng(seed)
    dz = rng.uniform(0.5, 1.5, nz)
    dz /= dz.sum()
    hzt = np.empty(nz + 1)
    hzt[0], hzt[-1] = dz[0] / 2.0, dz[-1] / 2.0
    hzt[1:-1] = (dz[:-1] + dz[1:]) / 2.0
    return dz, hzt


def column_fields(basin: Basin, nz: int, seed: int = 0, depth: float = 50.0, tau: float = 60.0) -> dict:
    """Seeded synthetic inputs of the 3-D velocity block of the mode-split
    step (Function/vel_ssh.f90:794-1076) on `basin`: the velocity time
    levels uu, uup, vv, vvp (nz levels), the vertical velocity ww and
    viscosity nu (nz + 1 levels), the 3-D RHS terms, the 2-D pressure
    gradient, drag and stresses, and the internal-mode depths (positive
    everywhere).  Magnitudes follow a shelf sea of `depth` metres: the
    velocities are O(0.1 m/s) and every RHS term is a fraction of the time
    term bp*u, so each term moves the solution."""
    rng = np.random.default_rng(seed)
    shp = basin.bounds.shape
    area = float(np.median(basin.metrics["dxt"]) * np.median(basin.metrics["dyh"]))
    scale = depth * area / tau * 0.1          # bp * 0.1 m/s, the RHS unit

    def f3(s, lev=nz):
        return np.asfortranarray(s * rng.standard_normal((*shp, lev)))

    def f2(s):
        return np.asfortranarray(s * rng.standard_normal(shp))

    def pos(lo, hi, lev=None):
        return np.asfortranarray(rng.uniform(lo, hi, shp if lev is None else (*shp, lev)))

    out = dict(uu=f3(0.1), uup=f3(0.1), vv=f3(0.1), vvp=f3(0.1),
               ww=f3(1.0e-3, nz + 1), nu=pos(1.0e-4, 1.0e-2, nz + 1),
               rhsx=f3(0.05 * scale), rhsy=f3(0.05 * scale), rhsx_tran=f3(0.05 * scale),
               rhsy_tran=f3(0.05 * scale), pgrx=f2(0.05 * scale), pgry=f2(0.05 * scale),
               rdis=pos(0.0, 2.0e-5), tx_surf=f2(1.0e-4), ty_surf=f2(1.0e-4), tx_bot=f2(1.0e-4),
               ty_bot=f2(1.0e-4))
    for k in ("hhu", "hhup", "hhun", "hhv", "hhvp", "hhvn", "hhh"):
        out[k] = pos(0.8 * depth, 1.2 * depth)
    out["wflux"] = f2(1.0e-5 * basin.consts.ref_den)
    return out


def tracer_fields(basin: Basin, nz: int, seed: int = 0, depth: float = 50.0) -> dict:
    """Seeded synthetic inputs of one tracer's step (Function/tem_sal.f90):
    a temperature-like tracer ff, ffp (nz levels, about 10 +- 3), the
    transporting velocities uu, vv (nz) and ww (nz + 1), lateral diffusivity
    mu (nz) and vertical nu (nz + 1) with their factors, isopycnal and
    z-level slopes (nz + 1), the isoneutral/GM weights, surface and bottom
    values with boundary-condition types 1 or 2, the short-wave balance and
    source, and the internal-mode depths hhu, hhv, hhqn, hhqp."""
    rng = np.random.default_rng(seed)
    shp = basin.bounds.shape

    def f3(lev, s, loc=0.0):
        return np.asfortranarray(loc + s * rng.standard_normal((*shp, lev)))

    def pos(lo, hi, lev=None):
        return np.asfortranarray(rng.uniform(lo, hi, shp if lev is None else (*shp, lev)))

    out = dict(ff=f3(nz, 3.0, 10.0), ffp=f3(nz, 3.0, 10.0), uu=f3(nz, 0.1), vv=f3(nz, 0.1),
               ww=f3(nz + 1, 1.0e-3), mu=pos(50.0, 500.0, nz), nu=pos(1.0e-5, 1.0e-3, nz + 1),
               slrx=f3(nz + 1, 1.0e-3), slry=f3(nz + 1, 1.0e-3), slzx=f3(nz + 1, 1.0e-3), slzy=f3(nz + 1, 1.0e-3),
               ff_top=f3(1, 2.0, 15.0)[..., 0].copy(order="F"), ff_bot=f3(1, 1.0, 4.0)[..., 0].copy(order="F"),
               ig_top=np.asfortranarray(rng.integers(1, 3, shp, dtype=np.int32)),
               ig_bot=np.asfortranarray(rng.integers(1, 3, shp, dtype=np.int32)),
               swbal=pos(0.0, 1.0), src=f3(nz, 1.0e-6), factor_mu=1.0, factor_nu=1.0, az=0.3, ar=0.7,
               alpha_gm=1.0, src_factor=1.0)
    for k in ("hhu", "hhv", "hhqn", "hhqp"):
        out[k] = pos(0.8 * depth, 1.2 * depth)
    return out
