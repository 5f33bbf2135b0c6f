"""The lateral viscosity of the mode-split step (Control/dyncall.f90:37-43):
3-D stress_components (Function/mixing.f90:115-168) on uup, vvp, then
smagorinsky_coeff (:171-219), then depth_ave of amuv into the barotropic
viscosity.

CPU: the C oracle against a numpy restatement of the same lines, bit for
bit, and a property (a solid-body shear-free, tension-free flow gives the
background viscosity).  GPU: inmsom_stress_components and
inmsom_smagorinsky_coeff against the oracle, bit for bit, with arrays
that hold other values at the points the routines do not set, on a
coastline basin and on periodic ones.
"""
import numpy as np
import pytest

from inmsom_elfs_b200 import basins
from test_baroclinic import coastline, inputs, periodic

NZ = 6
VISC2, DIFT = 1.0e3, 1.0e2
KP = 0.4 / 3.141592653589793


def _case(ora, case):
    return {"coastline": lambda: coastline(ora, nx=40, ny=33), "periodic_xy": lambda: periodic(ora),
            "channel_x": lambda: periodic(ora, px=1, py=0)}[case]()


def _fields(b, nz, seed):
    rng = np.random.default_rng(seed)
    sh = b.bounds.shape + (nz,)
    return {k: np.asfortranarray(rng.standard_normal(sh) * s) for k, s in
            (("u", 0.3), ("v", 0.3), ("str_t", 1e-5), ("str_s", 1e-5), ("amts", 7.0), ("amuv", 9.0))}


def np_stress(b, u, v, str_t, str_s):
    B, M, g = b.bounds, b.masks, b.metrics
    str_t, str_s = str_t.copy(order="F"), str_s.copy(order="F")
    i, j = B.interior
    im, jm = slice(i.start - 1, i.stop - 1), slice(j.start - 1, j.stop - 1)
    ip, jp = slice(i.start + 1, i.stop + 1), slice(j.start + 1, j.stop + 1)
    dx, dy, dxh, dyh = g["dx"], g["dy"], g["dxh"], g["dyh"]
    dxt, dyt, dxb, dyb = g["dxt"], g["dyt"], g["dxb"], g["dyb"]
    for k in range(u.shape[2]):
        uk, vk = u[:, :, k], v[:, :, k]
        t = (dy[i, j] / dx[i, j] * (uk[i, j] / dyh[i, j] - uk[im, j] / dyh[im, j])
             - dx[i, j] / dy[i, j] * (vk[i, j] / dxh[i, j] - vk[i, jm] / dxh[i, jm]))
        s = (dxb[i, j] / dyb[i, j] * (uk[i, jp] / dxt[i, jp] - uk[i, j] / dxt[i, j])
             + dyb[i, j] / dxb[i, j] * (vk[ip, j] / dyt[ip, j] - vk[i, j] / dyt[i, j]))
        str_t[i, j, k] = np.where(M["lu"][i, j] > 0.5, t, str_t[i, j, k])
        str_s[i, j, k] = np.where(M["luu"][i, j] > 0.5, s, str_s[i, j, k])
    return _wrap(B, str_t), _wrap(B, str_s)


def np_smagorinsky(b, str_t, str_s, amts, amuv):
    B, g = b.bounds, b.metrics
    amts, amuv = amts.copy(order="F"), amuv.copy(order="F")
    i, j = B.interior
    im, jm = slice(i.start - 1, i.stop - 1), slice(j.start - 1, j.stop - 1)
    ocean = b.masks["lu"][i, j] > 0.5
    for k in range(str_t.shape[2]):
        s = str_s[:, :, k]
        s2 = (s[i, j] ** 2 + s[im, j] ** 2 + s[i, jm] ** 2 + s[im, jm] ** 2) / 4.0
        mu = KP * KP * g["dx"][i, j] * g["dy"][i, j] * np.sqrt(str_t[i, j, k] ** 2 + s2)
        amuv[i, j, k] = np.where(ocean, VISC2 + mu, amuv[i, j, k])
        amts[i, j, k] = np.where(ocean, DIFT + mu * 0.1, amts[i, j, k])
    return _wrap(B, amts), _wrap(B, amuv)


def _wrap(B, a):
    x0, y0 = B.bnd_x1, B.bnd_y1
    if B.periodicity_x:
        a[B.mmm - 1 - x0], a[B.mm + 1 - x0] = a[B.mm - x0].copy(), a[B.mmm - x0].copy()
    if B.periodicity_y:
        a[:, B.nnn - 1 - y0], a[:, B.nn + 1 - y0] = a[:, B.nn - y0].copy(), a[:, B.nnn - y0].copy()
    return a


@pytest.mark.parametrize("case", ["coastline", "periodic_xy", "channel_x"])
def test_oracle_matches_numpy_restatement(ora, case):
    b = _case(ora, case)
    f = _fields(b, NZ, 3)
    want = np_stress(b, f["u"], f["v"], f["str_t"], f["str_s"])
    got = ora.stress_components(b, f["u"], f["v"], f["str_t"].copy(order="F"), f["str_s"].copy(order="F"))
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)
    want = np_smagorinsky(b, got[0], got[1], f["amts"], f["amuv"])
    mine = ora.smagorinsky_coeff(b, VISC2, DIFT, got[0], got[1], f["amts"].copy(order="F"), f["amuv"].copy(order="F"))
    for g_, w_ in zip(mine, want):
        assert np.array_equal(g_, w_)


def test_still_water_gives_the_background_viscosity(ora):
    """No flow: no tension, no shear, so amuv = visc2 and amts = dift at
    every ocean point of the interior."""
    b = _case(ora, "coastline")
    f = _fields(b, 2, 4)
    zero = np.zeros_like(f["u"])
    st, ss = ora.stress_components(b, zero, zero, np.zeros_like(zero), np.zeros_like(zero))
    amts, amuv = ora.smagorinsky_coeff(b, VISC2, DIFT, st, ss, f["amts"].copy(order="F"), f["amuv"].copy(order="F"))
    i, j = b.bounds.interior
    ocean = b.masks["lu"][i, j] > 0.5
    assert np.all(amuv[i, j][ocean] == VISC2) and np.all(amts[i, j][ocean] == DIFT)
    assert np.array_equal(amuv[i, j][~ocean], f["amuv"][i, j][~ocean])


@pytest.mark.gpu
@pytest.mark.parametrize("case,nz", [("coastline", NZ), ("coastline", 1), ("periodic_xy", NZ), ("channel_x", 3)])
def test_lateral_viscosity_bitexact(gpu, ora, case, nz):
    """stress_components -> smagorinsky_coeff -> depth_ave(amuv), the chain
    of Control/dyncall.f90:37-43, through the C ABI against the oracle."""
    b = _case(ora, case)
    f = _fields(b, nz, 10 + nz)
    dz, _, _ = inputs(b, nz=nz, seed=nz)
    w_st, w_ss = ora.stress_components(b, f["u"], f["v"], f["str_t"].copy(order="F"), f["str_s"].copy(order="F"))
    w_ts, w_uv = ora.smagorinsky_coeff(b, VISC2, DIFT, w_st, w_ss, f["amts"].copy(order="F"),
                                       f["amuv"].copy(order="F"))
    mu0 = basins.column_fields(b, 1, seed=4)["pgrx"]
    _, w_mu = ora.depth_ave(b, dz, w_uv.copy(order="F"), mu0.copy(order="F"), b.masks["lu"], 0)
    with gpu.BarotropicSolver(b, resident=False) as s:
        g_st, g_ss = s.stress_components(f["u"], f["v"], f["str_t"].copy(order="F"), f["str_s"].copy(order="F"))
        g_ts, g_uv = s.smagorinsky_coeff(VISC2, DIFT, g_st, g_ss, f["amts"].copy(order="F"),
                                         f["amuv"].copy(order="F"))
        _, g_mu = s.depth_ave(dz, g_uv.copy(order="F"), mu0.copy(order="F"), b.masks["lu"], 0)
    for name, g_, w_ in (("str_t", g_st, w_st), ("str_s", g_ss, w_ss), ("amts", g_ts, w_ts),
                         ("amuv", g_uv, w_uv), ("mu", g_mu, w_mu)):
        assert np.array_equal(g_, w_), f"{name}: max diff {np.max(np.abs(g_ - w_))}"
    assert not np.array_equal(g_uv, f["amuv"])
