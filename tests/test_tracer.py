"""One tracer's transport-diffusion step, tracer_tran_diff
(Function/tem_sal.f90:1-422).

CPU: the C oracle against a second, vectorised numpy restatement of the
same lines (bit for bit) on a coastline basin and on periodic basins, and
properties (a uniform tracer with no flux stays uniform; the tridiagonal
solve's residual).  GPU: inmsom_tracer_tran_diff against the oracle, bit
for bit, including the flux diagnostics.
"""
import numpy as np
import pytest

from inmsom_elfs_b200 import basins
from test_baroclinic import NZ, TAU, _views, coastline, periodic


def inputs(b, nz=NZ, seed=0):
    dz, hzt = basins.vertical_grid(nz, seed)
    return dz, hzt, basins.tracer_fields(b, nz, seed=seed + 1)


def _wrap_x(B, a):
    x0 = B.bnd_x1
    left, right = a[B.mm - x0].copy(), a[B.mmm - x0].copy()
    a[B.mmm - 1 - x0], a[B.mm + 1 - x0] = left, right


def _wrap_y(B, a):
    y0 = B.bnd_y1
    a[:, B.nnn - 1 - y0] = a[:, B.nn - y0]
    a[:, B.nn + 1 - y0] = a[:, B.nnn - y0]


def np_tracer(b, dz, hzt, tau, f):
    B, mt = b.bounds, b.metrics
    sh = _views(B)
    nz = len(dz)
    shp = B.shape
    ff, ffp = f["ff"], f["ffp"]
    Z = lambda lev: np.zeros((*shp, lev), order="F")
    F = {k: Z(nz) for k in ("x", "y")}
    FZ, CO, SG = ({k: Z(nz + 1) for k in ("x", "y")} for _ in range(3))
    FO = {k: Z(4) for k in ("x", "y")}
    for d in ("x", "y"):
        V = d == "y"
        e = (0, 1) if V else (1, 0)
        mask = sh(b.masks["lcv" if V else "lcu"]) > 0.5
        hh = sh(f["hhv" if V else "hhu"])
        slr, slz = f["slry" if V else "slrx"], f["slzy" if V else "slzx"]
        vel = f["vv" if V else "uu"]
        dside, dnorm = sh(mt["dxh" if V else "dyh"]), sh(mt["dyt" if V else "dxt"])
        f1d = np.zeros(mask.shape + (nz + 2,))
        for k in range(2, nz + 1):
            a0, a1 = k - 1, k - 2
            dfdz = (sh(ffp)[..., a0] - sh(ffp)[..., a1] + sh(ffp, *e)[..., a0] - sh(ffp, *e)[..., a1]) / 2.0
            dfdh = (sh(ffp, *e)[..., a0] - sh(ffp)[..., a0] + sh(ffp, *e)[..., a1] - sh(ffp)[..., a1]) / 2.0
            mu1 = ((sh(f["mu"])[..., a0] + sh(f["mu"])[..., a1] + sh(f["mu"], *e)[..., a0] + sh(f["mu"], *e)[..., a1])
                   / 4.0 * f["factor_mu"] * dside / dnorm)
            slope = f["ar"] * sh(slr)[..., a0] + f["az"] * sh(slz)[..., a0]
            f1d[..., k] = np.where(mask, mu1 * (hh * dfdh * hzt[k - 1] - slope * dfdz), 0.0)
            sh(FZ[d])[..., a0] = np.where(mask, mu1 * slope * dfdh, 0.0)
            sh(CO[d])[..., a0] = np.where(mask, mu1 * (slope * slope) / hh / hzt[k - 1], 0.0)
            sh(SG[d])[..., a0] = np.where(mask, mu1 * (sh(slr)[..., a0] - sh(slz)[..., a0]) * f["alpha_gm"], 0.0)
        for k in range(1, nz + 1):
            q = k - 1
            if k == 1:
                fd = f1d[..., 2] / hzt[1]
            elif k < nz:
                fd = (f1d[..., k] + f1d[..., k + 1]) / dz[q] / 2.0
            else:
                fd = f1d[..., k] / hzt[k - 1]
            s2 = sh(ff)[..., q] + sh(ff, *e)[..., q]
            fa = -(sh(vel)[..., q] * hh * dside * s2 / 2.0)
            vg = (sh(SG[d])[..., k] - sh(SG[d])[..., q]) / dz[q]
            fg = -(vg * s2 / 2.0)
            sh(F[d])[..., q] = np.where(mask, fa + fd + fg, 0.0)
            o = sh(FO[d])
            o[..., 0] = np.where(mask, o[..., 0] + dz[q] * (fa + fd + fg), o[..., 0])
            o[..., 1] = np.where(mask, o[..., 1] + dz[q] * fa, o[..., 1])
            o[..., 2] = np.where(mask, o[..., 2] + dz[q] * fd, o[..., 2])
            o[..., 3] = np.where(mask, o[..., 3] + dz[q] * fg, o[..., 3])
    if B.periodicity_x:
        for a in (F["x"], FZ["x"], CO["x"], SG["x"]):
            _wrap_x(B, a)
    if B.periodicity_y:
        for a in (F["y"], FZ["y"], CO["y"], SG["y"]):
            _wrap_y(B, a)
    # the column solves
    lu = sh(b.masks["lu"]) > 0.5
    dxv, dyv = sh(mt["dx"]), sh(mt["dy"])
    hn, hp = sh(f["hhqn"]), sh(f["hhqp"])
    bp, bp0 = hn * dxv * dyv / tau / 2.0, hp * dxv * dyv / tau / 2.0
    cu = np.maximum(sh(b.masks["lcu"]) + sh(b.masks["lcu"], -1), np.float32(1e-10)).astype(np.float64)
    cv = np.maximum(sh(b.masks["lcv"]) + sh(b.masks["lcv"], 0, -1), np.float32(1e-10)).astype(np.float64)
    A, Bd, C, E = (np.zeros(lu.shape + (nz,)) for _ in range(4))
    fz_p = np.zeros(lu.shape)
    dp = np.zeros(lu.shape)
    for k in range(1, nz + 1):
        q = k - 1
        fz_m = fz_p
        if k < nz:
            vg = -(sh(SG["x"])[..., k] - sh(SG["x"], -1)[..., k] + sh(SG["y"])[..., k] - sh(SG["y"], 0, -1)[..., k])
            fz_p = (-((sh(FZ["x"])[..., k] + sh(FZ["x"], -1)[..., k]) / cu)
                    - (sh(FZ["y"])[..., k] + sh(FZ["y"], 0, -1)[..., k]) / cv
                    + (sh(CO["x"])[..., k] * (sh(ffp, 1)[..., k] - sh(ffp, 1)[..., q])
                       + sh(CO["x"], -1)[..., k] * (sh(ffp, -1)[..., k] - sh(ffp, -1)[..., q])) / cu / 2.0
                    + (sh(CO["y"])[..., k] * (sh(ffp, 0, 1)[..., k] - sh(ffp, 0, 1)[..., q])
                       + sh(CO["y"], 0, -1)[..., k] * (sh(ffp, 0, -1)[..., k] - sh(ffp, 0, -1)[..., q])) / cv / 2.0
                    - (sh(f["ww"])[..., k] * dxv * dyv + vg) * (sh(ff)[..., q] + sh(ff)[..., k]) / 2.0)
        else:
            fz_p = np.zeros(lu.shape)
        nu_p = sh(f["nu"])[..., k] * f["factor_nu"]
        dm = sh(f["nu"])[..., 0] * f["factor_nu"] * dxv * dyv / hn / hzt[0] if k == 1 else dp
        if k < nz:
            dp = ((sh(CO["x"])[..., k] + sh(CO["x"], -1)[..., k]) / cu / 2.0
                  + (sh(CO["y"])[..., k] + sh(CO["y"], 0, -1)[..., k]) / cv / 2.0
                  + nu_p * dxv * dyv / hn / hzt[k])
        else:
            dp = nu_p * dxv * dyv / hn / hzt[k]
        rhs = (sh(F["x"])[..., q] - sh(F["x"], -1)[..., q] + sh(F["y"])[..., q] - sh(F["y"], 0, -1)[..., q]
               + (fz_p - fz_m) / dz[q]
               + sh(f["src"])[..., q] * sh(b.hhq_rest) * sh(f["swbal"]) * f["src_factor"] * dxv * dyv)
        base = bp0 * sh(ffp)[..., q] + rhs
        if k == 1:
            t1 = sh(f["ig_top"]) == 1
            C[..., q] = -dp / dz[q]
            Bd[..., q] = np.where(t1, bp + (dp + dm) / dz[q], bp + dp / dz[q])
            E[..., q] = np.where(t1, base + dm * sh(f["ff_top"]) / dz[q], base + sh(f["ff_top"]) / dz[q] * dxv * dyv)
        elif k < nz:
            C[..., q], A[..., q] = -dp / dz[q], -dm / dz[q]
            Bd[..., q] = bp + (dp + dm) / dz[q]
            E[..., q] = base
        else:
            t1 = sh(f["ig_bot"]) == 1
            A[..., q] = -dm / dz[q]
            Bd[..., q] = np.where(t1, bp + (dp + dm) / dz[q], bp + dm / dz[q])
            E[..., q] = np.where(t1, base + dp * sh(f["ff_bot"]) / dz[q], base + sh(f["ff_bot"]) / dz[q] * dxv * dyv)
    x, y = np.zeros_like(E), np.zeros_like(E)
    x[..., 0], y[..., 0] = -C[..., 0] / Bd[..., 0], E[..., 0] / Bd[..., 0]
    for j in range(1, nz):
        scr = 1.0 / (A[..., j] * x[..., j - 1] + Bd[..., j])
        x[..., j], y[..., j] = -C[..., j] * scr, (E[..., j] - A[..., j] * y[..., j - 1]) * scr
    r = np.zeros_like(E)
    r[..., -1] = y[..., -1]
    for j in range(nz - 2, -1, -1):
        r[..., j] = x[..., j] * r[..., j + 1] + y[..., j]
    fn = Z(nz)
    sh(fn)[...] = np.where(lu[..., None], r, 0.0)
    if B.periodicity_x:
        _wrap_x(B, fn)
    if B.periodicity_y:
        _wrap_y(B, fn)
    x0, y0 = B.bnd_x1, B.bnd_y1
    ring = (slice(B.nx_start - 1 - x0, B.nx_end + 2 - x0), slice(B.ny_start - 1 - y0, B.ny_end + 2 - y0))
    m = (b.masks["lu"][ring] > 0.5)[..., None]
    ts = b.consts.time_smooth
    ff2, ffp2 = ff.copy(order="F"), ffp.copy(order="F")
    ffp2[ring] = np.where(m, ff[ring] + ts * (fn[ring] - 2.0 * ff[ring] + ffp[ring]) / 2.0, ffp[ring])
    ff2[ring] = np.where(m, fn[ring], ff[ring])
    return ff2, ffp2, FO["x"], FO["y"]


def _oracle(ora, b, dz, hzt, f, tau=TAU):
    ff, ffp = f["ff"].copy(order="F"), f["ffp"].copy(order="F")
    fx = np.full((*b.bounds.shape, 4), 7.0, order="F")     # the call zeroes them first
    fy = np.full((*b.bounds.shape, 4), 7.0, order="F")
    return ora.tracer_tran_diff(b, dz, hzt, tau, ff, ffp, fx, fy, f)


CASES = {"coastline": lambda ora: coastline(ora), "periodic_xy": lambda ora: periodic(ora),
         "channel_x": lambda ora: periodic(ora, px=1, py=0)}


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_matches_numpy_restatement(ora, case):
    b = CASES[case](ora)
    dz, hzt, f = inputs(b)
    got = _oracle(ora, b, dz, hzt, f)
    with np.errstate(all="ignore"):
        want = np_tracer(b, dz, hzt, TAU, f)
    for name, g_, w_ in zip(("ff", "ffp", "flux_f_x", "flux_f_y"), got, want):
        assert np.array_equal(g_, w_), f"{name}: max diff {np.nanmax(np.abs(g_ - w_))}"
    assert not np.array_equal(got[0], f["ff"])


def test_uniform_tracer_without_fluxes_stays_uniform(ora):
    """No velocity, no source, insulating top and bottom (type 2 with zero
    flux) and a uniform tracer at both time levels: ff stays uniform."""
    b = coastline(ora, nx=40, ny=30)
    dz, hzt, f = inputs(b, nz=8)
    for k in ("uu", "vv", "ww", "src", "ff_top", "ff_bot"):
        f[k] = np.zeros_like(f[k])
    f["ig_top"][:] = 2
    f["ig_bot"][:] = 2
    f["ff"][:] = 12.5
    f["ffp"][:] = 12.5
    f["hhqp"] = f["hhqn"].copy(order="F")
    ff, ffp, fx, fy = _oracle(ora, b, dz, hzt, f)
    sh = _views(b.bounds)
    m = sh(b.masks["lu"]) > 0.5
    assert np.allclose(sh(ff)[m], 12.5, rtol=1e-13, atol=0)
    assert np.allclose(sh(ffp)[m], 12.5, rtol=1e-13, atol=0)
    assert np.all(np.abs(fx) < 1e-9) and np.all(np.abs(fy) < 1e-9)


def test_tracer_content_is_conserved(ora):
    """Closed basin, no source, zero-flux surface and bottom (type 2): the
    step only moves the tracer, sum over ocean columns and levels of
    dz*hhqn*dx*dy*ff(new) equals that of dz*hhqp*dx*dy*ffp (the lateral
    fluxes cancel between neighbours, the vertical parts and the diffusion
    telescope in the column)."""
    b = coastline(ora)
    dz, hzt, f = inputs(b, nz=12, seed=5)
    f["src"] = np.zeros_like(f["src"])
    f["ig_top"][:] = 2
    f["ig_bot"][:] = 2
    f["ff_top"] = np.zeros_like(f["ff_top"])
    f["ff_bot"] = np.zeros_like(f["ff_bot"])
    ff, ffp, _, _ = _oracle(ora, b, dz, hzt, f)
    sh = _views(b.bounds)
    m = (sh(b.masks["lu"]) > 0.5)[..., None]
    area = (sh(b.metrics["dx"]) * sh(b.metrics["dy"]))[..., None]
    new = np.sum(np.where(m, dz * sh(f["hhqn"])[..., None] * area * sh(ff), 0.0))
    old = np.sum(np.where(m, dz * sh(f["hhqp"])[..., None] * area * sh(f["ffp"]), 0.0))
    assert abs(new - old) / abs(old) < 1e-12
    assert not np.allclose(sh(ff)[m[..., 0]], sh(f["ffp"])[m[..., 0]])   # but it does move


# ---- GPU ------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("case,nz", [("coastline", NZ), ("coastline", 2), ("coastline", 41), ("periodic_xy", NZ),
                                     ("channel_x", 7)])
def test_tracer_bitexact(gpu, ora, case, nz):
    b = CASES[case](ora)
    dz, hzt, f = inputs(b, nz=nz, seed=nz)
    want = _oracle(ora, b, dz, hzt, f)
    ff, ffp = f["ff"].copy(order="F"), f["ffp"].copy(order="F")
    fx = np.full((*b.bounds.shape, 4), 7.0, order="F")
    fy = np.full((*b.bounds.shape, 4), 7.0, order="F")
    with gpu.BarotropicSolver(b, resident=False) as s:
        got = s.tracer_tran_diff(dz, hzt, TAU, ff, ffp, fx, fy, f)
        phases = s.last_phases()
    for name, g_, w_ in zip(("ff", "ffp", "flux_f_x", "flux_f_y"), got, want):
        assert np.array_equal(g_, w_), f"{name}: max diff {np.nanmax(np.abs(g_ - w_))}"
    assert phases[1] > 0.0


@pytest.mark.gpu
def test_tracer_rejects_bad_arguments(gpu, ora):
    from inmsom_elfs_b200._lib import InmsomError
    b = coastline(ora, nx=40, ny=30)
    dz, hzt, f = inputs(b, nz=6)
    f["ig_top"][b.masks["lu"] > 0.5] = 3
    with gpu.BarotropicSolver(b, resident=False) as s:
        with pytest.raises(InmsomError) as e:
            s.tracer_tran_diff(dz, hzt, TAU, f["ff"].copy(order="F"), f["ffp"].copy(order="F"),
                               np.zeros((*b.bounds.shape, 4), order="F"), np.zeros((*b.bounds.shape, 4), order="F"), f)
    assert e.value.code == 2


@pytest.mark.gpu
def test_tracer_and_baroclinic_share_a_context(gpu, ora):
    """Both blocks on one context, with the level count changing in between:
    each keeps its own device block and stays bit-exact."""
    from test_baroclinic import _run_oracle as baro_oracle
    from test_baroclinic import inputs as baro_inputs
    b = coastline(ora, nx=60, ny=50)
    with gpu.BarotropicSolver(b, resident=False) as s:
        for nz in (NZ, 7, NZ):
            dz, hzt, f = inputs(b, nz=nz, seed=nz)
            want = _oracle(ora, b, dz, hzt, f)
            ff, ffp = f["ff"].copy(order="F"), f["ffp"].copy(order="F")
            fx, fy = np.zeros((*b.bounds.shape, 4), order="F"), np.zeros((*b.bounds.shape, 4), order="F")
            got = s.tracer_tran_diff(dz, hzt, TAU, ff, ffp, fx, fy, f)
            for g_, w_ in zip(got, want):
                assert np.array_equal(g_, w_)
            dzb, hztb, fb = baro_inputs(b, nz=nz + 3, seed=nz)
            wb = baro_oracle(ora, b, dzb, hztb, fb)
            st = [fb[k].copy(order="F") for k in ("uu", "uup", "vv", "vvp")]
            s.baroclinic_dynamics(dzb, hztb, TAU, *st, **{k: fb[k] for k in s.BAROCLINIC_FIELDS})
            for g_, w_ in zip(st, wb):
                assert np.array_equal(g_, w_)
