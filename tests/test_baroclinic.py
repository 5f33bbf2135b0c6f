"""The 3-D velocity block of the mode-split step: baroclinic_dynamics
(Function/vel_ssh.f90:794-1027, with the tridiagonal sweep factor8 of
Service/oc_algorithms.f90:494-524) and vertical_velocity
(Function/vel_ssh.f90:1030-1076).

CPU: the C oracle against a second, vectorised numpy restatement of the
same lines (bit for bit), and against properties of the equations (the
solution satisfies its tridiagonal system; with no coupling each level is
eta/bp; w integrates the divergence).  GPU: inmsom_baroclinic_dynamics and
inmsom_vertical_velocity against the oracle, bit for bit, on a coastline
basin, at the smallest nz, and on periodic basins whose ring points are
ocean.
"""
import numpy as np
import pytest
from conftest import rel_err

from inmsom_elfs_b200 import basins
from inmsom_elfs_b200.grid import Basin, Bounds, Consts

NZ = 20          # Inc/basinpar.fi:6
TAU = 60.0


def prep(b, ora):
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    return b


def coastline(ora, nx=90, ny=70, seed=31):
    return prep(basins.regional_basin(nx=nx, ny=ny, seed=seed), ora)


def periodic(ora, nx=24, ny=18, px=1, py=1, seed=5):
    """A basin that wraps in x (and y): ocean everywhere but a seeded
    island, with lu copied across the wrap so that ring points are ocean."""
    rng = np.random.default_rng(seed)
    b = Bounds.serial(nx, ny, periodicity_x=px, periodicity_y=py)
    basin = Basin(b, Consts())
    lu = np.ones(b.shape, dtype=np.float32, order="F")
    if not py:
        lu[:, : b.nnn - b.bnd_y1 + 1] = 0.0
        lu[:, b.nn - b.bnd_y1:] = 0.0
    i0, j0 = b.mmm - b.bnd_x1 + nx // 3, b.nnn - b.bnd_y1 + ny // 3
    lu[i0:i0 + 3, j0:j0 + 2] = 0.0
    basin.masks["lu"] = np.asfortranarray(lu)
    basins.uniform_metrics(basin, 2.0e3)
    basin.rlh_s = np.asfortranarray(1.0e-4 + 1.0e-5 * rng.standard_normal(b.shape))
    basin.hhq_rest = np.asfortranarray(np.where(lu > 0.5, 60.0 * (0.8 + 0.4 * rng.random(b.shape)), 0.0))
    basin.taux = np.full(b.shape, 0.1, order="F")
    basin.tauy = b.zeros()
    basin.forcing["mu"] = np.full(b.shape, 100.0, order="F")
    basin.forcing["rdis"] = np.full(b.shape, 1.0e-6, order="F")
    basin.dt = 10.0
    return prep(basin.fill_defaults(), ora)


def inputs(basin, nz=NZ, seed=0):
    dz, hzt = basins.vertical_grid(nz, seed)
    f = basins.column_fields(basin, nz, seed=seed + 1, tau=TAU)
    return dz, hzt, f


# ---- a second restatement, vectorised over the interior columns -----------

def _views(B):
    x0, y0 = B.bnd_x1, B.bnd_y1

    def sh(a, dm=0, dn=0):
        return a[B.nx_start - x0 + dm:B.nx_end - x0 + 1 + dm, B.ny_start - y0 + dn:B.ny_end - y0 + 1 + dn]
    return sh


def _wrap(B, a):
    """cyclize8_x then cyclize8_y on every level (Service/oc_algorithms.f90)."""
    x0, y0 = B.bnd_x1, B.bnd_y1
    if B.periodicity_x:
        left, right = a[B.mm - x0].copy(), a[B.mmm - x0].copy()
        a[B.mmm - 1 - x0], a[B.mm + 1 - x0] = left, right
    if B.periodicity_y:
        a[:, B.nnn - 1 - y0] = a[:, B.nn - y0]
        a[:, B.nn + 1 - y0] = a[:, B.nnn - y0]


def np_baroclinic(basin, dz, hzt, tau, uu, uup, vv, vvp, f, want_system=False):
    B, g, mt = basin.bounds, basin, basin.metrics
    sh = _views(B)
    nz = len(dz)
    ts = basin.consts.time_smooth
    systems = {}
    new = {}
    for comp in ("u", "v"):
        V = comp == "v"
        e = (0, 1) if V else (1, 0)                 # far end of the velocity point
        p = (-1, 0) if V else (0, -1)               # partner of the Coriolis average
        self_, selfp, other = (vv, vvp, uu) if V else (uu, uup, vv)
        f1 = sh(mt["dxh" if V else "dxt"])
        f2 = sh(mt["dyt" if V else "dyh"])
        hn = sh(f["hhvn" if V else "hhun"])
        bp = hn * f1 * f2 / tau / 2.0
        bp0 = sh(f["hhvp" if V else "hhup"]) * f1 * f2 / tau / 2.0
        hc = sh(f["hhv" if V else "hhu"])
        pg = sh(f["pgry" if V else "pgrx"])
        rhs, rhst = f["rhsy" if V else "rhsx"], f["rhsy_tran" if V else "rhsx_tran"]
        ts_, tb_ = sh(f["ty_surf" if V else "tx_surf"]), sh(f["ty_bot" if V else "tx_bot"])
        dx, dy = mt["dx"], mt["dy"]
        cor = lambda d: sh(g.rlh_s, *d) * sh(f["hhh"], *d) * sh(mt["dxb"], *d) * sh(mt["dyb"], *d)
        cor0, cor1 = cor((0, 0)), cor(p)
        drag = (sh(f["rdis"]) + sh(f["rdis"], *e)) / 2.0
        A, Bd, C, E = (np.zeros(bp.shape + (nz,)) for _ in range(4))
        dp = np.zeros(bp.shape)
        fz_p = np.zeros(bp.shape)
        for k in range(1, nz + 1):
            q = k - 1
            dm, fz_m = dp, fz_p
            if k < nz:
                dp = (sh(f["nu"])[..., k] + sh(f["nu"], *e)[..., k]) / 2.0 / hn / hzt[k] * f1 * f2
                fz_p = ((sh(f["ww"])[..., k] * sh(dx) * sh(dy) + sh(f["ww"], *e)[..., k] * sh(dx, *e) * sh(dy, *e))
                        / 2.0 * (sh(self_)[..., q] + sh(self_)[..., k]) / 2.0)
            else:
                dp = np.zeros(bp.shape)
                fz_p = np.zeros(bp.shape)
            C[..., q] = -dp / dz[q] if k < nz else 0.0
            A[..., q] = -dm / dz[q] if k > 1 else 0.0
            Bd[..., q] = (bp + dp / dz[q] if k == 1 else (bp + (dp + dm) / dz[q] if k < nz else bp + dm / dz[q]))
            c_ = (cor0 * (sh(other, *e)[..., q] + sh(other)[..., q])
                  + cor1 * (sh(other, e[0] + p[0], e[1] + p[1])[..., q] + sh(other, *p)[..., q])) / 4.0
            eta = bp0 * sh(selfp)[..., q] + sh(rhs)[..., q] + sh(rhst)[..., q] + pg - (fz_p - fz_m) / dz[q]
            eta = eta - c_ if V else eta + c_
            eta = eta - drag * sh(selfp)[..., q] * f1 * f2 * hc
            if k == 1:
                eta = eta + ts_ / dz[q] * f1 * f2
            if k == nz:
                eta = eta + tb_ / dz[q] * f1 * f2
            E[..., q] = eta
        # factor8
        x = np.zeros_like(E)
        y = np.zeros_like(E)
        x[..., 0] = -C[..., 0] / Bd[..., 0]
        y[..., 0] = E[..., 0] / Bd[..., 0]
        for j in range(1, nz):
            scr = 1.0 / (A[..., j] * x[..., j - 1] + Bd[..., j])
            x[..., j] = -C[..., j] * scr
            y[..., j] = (E[..., j] - A[..., j] * y[..., j - 1]) * scr
        r = np.zeros_like(E)
        r[..., nz - 1] = y[..., nz - 1]
        for j in range(nz - 2, -1, -1):
            r[..., j] = x[..., j] * r[..., j + 1] + y[..., j]
        mask = sh(g.masks["lcv" if V else "lcu"]) > 0.5
        full = np.zeros(self_.shape, order="F")
        sh(full)[...] = np.where(mask[..., None], r, 0.0)
        _wrap(B, full)
        new[comp] = full
        systems[comp] = (A, Bd, C, E, r, mask)
    out = []
    x0, y0 = B.bnd_x1, B.bnd_y1
    ring = (slice(B.nx_start - 1 - x0, B.nx_end + 2 - x0), slice(B.ny_start - 1 - y0, B.ny_end + 2 - y0))
    for comp, cur, prev in (("u", uu, uup), ("v", vv, vvp)):
        m = (g.masks["lcu" if comp == "u" else "lcv"][ring] > 0.5)[..., None]
        c2, p2 = cur.copy(order="F"), prev.copy(order="F")
        un = new[comp][ring]
        p2[ring] = np.where(m, cur[ring] + ts * (un - 2.0 * cur[ring] + prev[ring]) / 2.0, prev[ring])
        c2[ring] = np.where(m, un, cur[ring])
        out += [c2, p2]
    return (out, systems) if want_system else out


def np_vertical_velocity(basin, dz, u, v, w, hu, hv, wflux):
    B, mt = basin.bounds, basin.metrics
    sh = _views(B)
    nz = len(dz)
    c = basin.consts
    lu = sh(basin.masks["lu"]) > 0.5
    w = w.copy(order="F")
    acc = np.zeros(lu.shape)
    cols = np.zeros(lu.shape + (nz + 1,))
    for k in range(nz, 0, -1):
        q = k - 1
        acc = acc + dz[q] / (sh(mt["dx"]) * sh(mt["dy"])) * (
            sh(u)[..., q] * sh(hu) * sh(mt["dyh"]) - sh(u, -1)[..., q] * sh(hu, -1) * sh(mt["dyh"], -1)
            + sh(v)[..., q] * sh(hv) * sh(mt["dxh"]) - sh(v, 0, -1)[..., q] * sh(hv, 0, -1) * sh(mt["dxh"], 0, -1)
            + sh(wflux) / c.ref_den * float(c.full_free_surface))
        cols[..., q] = acc
    sh(w)[...] = np.where(lu[..., None], cols, sh(w))
    _wrap(B, w)
    return w


def _run_oracle(ora, basin, dz, hzt, f, tau=TAU):
    st = [f[k].copy(order="F") for k in ("uu", "uup", "vv", "vvp")]
    ora.baroclinic_dynamics(basin, dz, hzt, tau, *st, **{k: f[k] for k in ora.BAROCLINIC_FIELDS})
    return st


# ---- CPU ------------------------------------------------------------------

@pytest.mark.parametrize("case", ["coastline", "periodic_xy", "channel_x"])
def test_oracle_matches_numpy_restatement(ora, case):
    b = {"coastline": lambda: coastline(ora), "periodic_xy": lambda: periodic(ora),
         "channel_x": lambda: periodic(ora, px=1, py=0)}[case]()
    dz, hzt, f = inputs(b)
    got = _run_oracle(ora, b, dz, hzt, f)
    with np.errstate(all="ignore"):
        want = np_baroclinic(b, dz, hzt, TAU, f["uu"], f["uup"], f["vv"], f["vvp"], f)
    for name, g_, w_ in zip(("uu", "uup", "vv", "vvp"), got, want):
        assert np.array_equal(g_, w_), f"{name}: max diff {np.max(np.abs(g_ - w_))}"
    assert not np.array_equal(got[0], f["uu"])


def test_solution_satisfies_its_tridiagonal_system(ora):
    b = coastline(ora)
    dz, hzt, f = inputs(b)
    with np.errstate(all="ignore"):
        _, systems = np_baroclinic(b, dz, hzt, TAU, f["uu"], f["uup"], f["vv"], f["vvp"], f, want_system=True)
    for comp, (A, Bd, C, E, r, mask) in systems.items():
        res = Bd * r - E
        res[..., 1:] += A[..., 1:] * r[..., :-1]
        res[..., :-1] += C[..., :-1] * r[..., 1:]
        scale = np.abs(Bd * r) + np.abs(E)
        rel = np.abs(res)[mask] / scale[mask]
        assert rel.max() < 1e-12, comp


def test_uncoupled_levels_are_eta_over_bp(ora):
    """No viscosity, vertical velocity, Coriolis, drag or stress: every
    level solves bp*un = bp0*uup + RHS + pgr on its own."""
    b = coastline(ora, nx=40, ny=30)
    b.rlh_s = np.zeros(b.bounds.shape, order="F")
    dz, hzt, f = inputs(b, nz=6)
    for k in ("ww", "rdis", "tx_surf", "ty_surf", "tx_bot", "ty_bot"):
        f[k] = np.zeros_like(f[k])
    f["nu"] = np.zeros_like(f["nu"])
    uu, uup, vv, vvp = _run_oracle(ora, b, dz, hzt, f)
    sh = _views(b.bounds)
    area = sh(b.metrics["dxt"]) * sh(b.metrics["dyh"])
    bp = sh(f["hhun"]) * area / TAU / 2.0
    bp0 = sh(f["hhup"]) * area / TAU / 2.0
    un = (bp0[..., None] * sh(f["uup"]) + sh(f["rhsx"]) + sh(f["rhsx_tran"]) + sh(f["pgrx"])[..., None]) / bp[..., None]
    m = sh(b.masks["lcu"]) > 0.5
    # the terms are summed in another order here: normwise, a few ulps
    assert rel_err(sh(uu)[m], un[m]) < 1e-14
    ts = b.consts.time_smooth
    filt = sh(f["uu"]) + ts * (un - 2.0 * sh(f["uu"]) + sh(f["uup"])) / 2.0
    assert rel_err(sh(uup)[m], filt[m]) < 1e-14
    # land points keep their values
    assert np.array_equal(sh(uu)[~m], sh(f["uu"])[~m])


def test_vertical_viscosity_conserves_column_momentum(ora):
    """With only the vertical viscosity acting (no advection, Coriolis, drag,
    stress or RHS), each water column keeps sum_k dz*bp*un = sum_k dz*bp0*uup:
    the implicit diffusion moves momentum between levels only."""
    b = coastline(ora, nx=50, ny=40)
    b.rlh_s = np.zeros(b.bounds.shape, order="F")
    dz, hzt, f = inputs(b, nz=15, seed=4)
    for k in ("ww", "rdis", "tx_surf", "ty_surf", "tx_bot", "ty_bot", "pgrx", "pgry", "rhsx", "rhsy",
              "rhsx_tran", "rhsy_tran"):
        f[k] = np.zeros_like(f[k])
    uu, uup, vv, vvp = _run_oracle(ora, b, dz, hzt, f)
    sh = _views(b.bounds)
    for comp, new, prev, hn, hp, mask in (("u", uu, "uup", "hhun", "hhup", "lcu"), ("v", vv, "vvp", "hhvn", "hhvp", "lcv")):
        m = sh(b.masks[mask]) > 0.5
        lhs = np.sum(dz * sh(new), axis=2) * sh(f[hn])
        rhs = np.sum(dz * sh(f[prev]), axis=2) * sh(f[hp])
        scale = np.sum(dz * np.abs(sh(f[prev])), axis=2) * sh(f[hp])
        assert np.max(np.abs(lhs - rhs)[m] / scale[m]) < 1e-12, comp
        assert not np.allclose(sh(new)[m], sh(f[prev])[m])


@pytest.mark.parametrize("case", ["coastline", "periodic_xy"])
def test_vertical_velocity_oracle_matches_numpy(ora, case):
    b = coastline(ora) if case == "coastline" else periodic(ora)
    dz, _, f = inputs(b)
    w0 = basins.column_fields(b, NZ, seed=9)["ww"]
    got = ora.vertical_velocity(b, dz, f["uu"], f["vv"], w0.copy(order="F"), f["hhu"], f["hhv"], f["wflux"])
    with np.errstate(all="ignore"):
        want = np_vertical_velocity(b, dz, f["uu"], f["vv"], w0, f["hhu"], f["hhv"], f["wflux"])
    assert np.array_equal(got, want)
    sh = _views(b.bounds)
    m = sh(b.masks["lu"]) > 0.5
    assert np.all(sh(got)[..., NZ][m] == 0.0)          # w(nz+1) = 0 at ocean points
    assert np.array_equal(sh(got)[~m], sh(w0)[~m])     # land columns untouched


# ---- GPU ------------------------------------------------------------------

def _gpu_run(gpu, basin, dz, hzt, f, tau=TAU):
    st = [f[k].copy(order="F") for k in ("uu", "uup", "vv", "vvp")]
    with gpu.BarotropicSolver(basin, resident=False) as s:
        s.baroclinic_dynamics(dz, hzt, tau, *st, **{k: f[k] for k in s.BAROCLINIC_FIELDS})
        phases = s.last_phases()
    return st, phases


@pytest.mark.gpu
@pytest.mark.parametrize("case,nz", [("coastline", NZ), ("coastline", 2), ("coastline", 57), ("coastline", 96),
                                     ("coastline", 97), ("coastline", 150), ("periodic_xy", NZ), ("channel_x", 7)])
def test_baroclinic_bitexact(gpu, ora, case, nz):
    """From the smallest nz to one whose column sweep far exceeds a ring
slot's worth of levels; the drop-in call splits the rows into bands."""
    b = {"coastline": lambda: coastline(ora), "periodic_xy": lambda: periodic(ora),
         "channel_x": lambda: periodic(ora, px=1, py=0)}[case]()
    dz, hzt, f = inputs(b, nz=nz, seed=nz)
    want = _run_oracle(ora, b, dz, hzt, f)
    got, phases = _gpu_run(gpu, b, dz, hzt, f)
    for name, g_, w_ in zip(("uu", "uup", "vv", "vvp"), got, want):
        assert np.array_equal(g_, w_), f"{name}: max diff {np.max(np.abs(g_ - w_))}"
    assert not np.array_equal(got[0], f["uu"])
    assert all(t >= 0.0 for t in phases) and phases[1] > 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["coastline", "periodic_xy"])
def test_vertical_velocity_bitexact(gpu, ora, case):
    b = coastline(ora) if case == "coastline" else periodic(ora)
    dz, _, f = inputs(b)
    w0 = basins.column_fields(b, NZ, seed=9)["ww"]
    want = ora.vertical_velocity(b, dz, f["uu"], f["vv"], w0.copy(order="F"), f["hhu"], f["hhv"], f["wflux"])
    with gpu.BarotropicSolver(b, resident=False) as s:
        got = s.vertical_velocity(dz, f["uu"], f["vv"], w0.copy(order="F"), f["hhu"], f["hhv"], f["wflux"])
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_baroclinic_rejects_bad_levels(gpu, ora):
    from inmsom_elfs_b200._lib import InmsomError
    b = coastline(ora, nx=40, ny=30)
    for nz in (1, 201):
        dz, hzt, f = inputs(b, nz=nz)
        with gpu.BarotropicSolver(b, resident=False) as s:
            with pytest.raises(InmsomError) as e:
                s.baroclinic_dynamics(dz, hzt, TAU, f["uu"], f["uup"], f["vv"], f["vvp"],
                                      **{k: f[k] for k in s.BAROCLINIC_FIELDS})
        assert e.value.code == 2


@pytest.mark.gpu
def test_repeated_calls_and_level_change(gpu, ora):
    """The device block is reused across calls and rebuilt when nz changes."""
    b = coastline(ora, nx=60, ny=50)
    with gpu.BarotropicSolver(b, resident=False) as s:
        for nz in (NZ, NZ, 5, NZ):
            dz, hzt, f = inputs(b, nz=nz, seed=3 * nz)
            want = _run_oracle(ora, b, dz, hzt, f)
            st = [f[k].copy(order="F") for k in ("uu", "uup", "vv", "vvp")]
            s.baroclinic_dynamics(dz, hzt, TAU, *st, **{k: f[k] for k in s.BAROCLINIC_FIELDS})
            for g_, w_ in zip(st, want):
                assert np.array_equal(g_, w_)


# ---- the 2-D/3-D coupling loops of the mode-split step ----------------------

def np_depth_ave(basin, dz, u, utr, mask, kbcl):
    B = basin.bounds
    u, utr = u.copy(order="F"), utr.copy(order="F")
    inner = (slice(1, -1), slice(1, -1))
    m = mask[inner] > 0.5
    ff0 = np.zeros(m.shape)
    for k in range(len(dz)):
        ff0 = ff0 + u[inner][..., k] * dz[k]
    utr[inner] = np.where(m, ff0, utr[inner])
    sub = u[inner]
    sub[...] = np.where(m[..., None], sub - float(kbcl) * ff0[..., None], sub)
    return u, utr


@pytest.mark.parametrize("kbcl", [0, 1])
def test_depth_ave_oracle_matches_numpy(ora, kbcl):
    b = coastline(ora)
    dz, _, f = inputs(b)
    for mname, field in (("llu", "rhsx"), ("llv", "rhsy")):
        utr0 = basins.column_fields(b, 1, seed=4)["pgrx"]
        got = ora.depth_ave(b, dz, f[field].copy(order="F"), utr0.copy(order="F"), b.masks[mname], kbcl)
        want = np_depth_ave(b, dz, f[field], utr0, b.masks[mname], kbcl)
        for g_, w_ in zip(got, want):
            assert np.array_equal(g_, w_)
    # the depth mean of a level-independent field is the field (sum dz = 1)
    u = np.repeat(f["pgrx"][..., None], NZ, axis=2).copy(order="F")
    _, utr = ora.depth_ave(b, dz, u, b.bounds.zeros(), b.masks["llu"], 0)
    m = b.masks["llu"][1:-1, 1:-1] > 0.5
    assert np.allclose(utr[1:-1, 1:-1][m], f["pgrx"][1:-1, 1:-1][m], rtol=1e-14, atol=0)


def test_shift_barotropic_oracle_round_trip(ora):
    """Removing then restoring uu2d returns uu up to the rounding of x - s + s;
    the ring's ocean points are shifted, land points are not."""
    b = periodic(ora)
    _, _, f = inputs(b)
    s2 = {k: np.asfortranarray(0.1 * v / np.abs(v).max()) for k, v in basins.column_fields(b, 1, seed=6).items()
          if k in ("pgrx", "pgry")}            # velocities of the same size as uu
    uu, vv = f["uu"].copy(order="F"), f["vv"].copy(order="F")
    ora.shift_barotropic(b, NZ, uu, vv, s2["pgrx"], s2["pgry"], -1)
    B = b.bounds
    x0, y0 = B.bnd_x1, B.bnd_y1
    ring = (slice(B.nx_start - 1 - x0, B.nx_end + 2 - x0), slice(B.ny_start - 1 - y0, B.ny_end + 2 - y0))
    m = (b.masks["lcu"][ring] > 0.5)[..., None]
    want = np.where(m, f["uu"][ring] - s2["pgrx"][ring][..., None], f["uu"][ring])
    assert np.array_equal(uu[ring], want)
    ora.shift_barotropic(b, NZ, uu, vv, s2["pgrx"], s2["pgry"], 1)
    assert rel_err(uu, f["uu"]) < 1e-15 * 8 and rel_err(vv, f["vv"]) < 1e-15 * 8


@pytest.mark.gpu
@pytest.mark.parametrize("kbcl", [0, 1])
def test_depth_ave_bitexact(gpu, ora, kbcl):
    b = coastline(ora)
    dz, _, f = inputs(b)
    utr0 = basins.column_fields(b, 1, seed=4)["pgrx"]
    want = ora.depth_ave(b, dz, f["rhsx"].copy(order="F"), utr0.copy(order="F"), b.masks["llu"], kbcl)
    with gpu.BarotropicSolver(b, resident=False) as s:
        got = s.depth_ave(dz, f["rhsx"].copy(order="F"), utr0.copy(order="F"), b.masks["llu"], kbcl)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)


@pytest.mark.gpu
@pytest.mark.parametrize("sign", [-1, 1])
def test_shift_barotropic_bitexact(gpu, ora, sign):
    b = periodic(ora)
    _, _, f = inputs(b, nz=9)
    s2 = basins.column_fields(b, 1, seed=6)
    want = ora.shift_barotropic(b, 9, f["uu"].copy(order="F"), f["vv"].copy(order="F"), s2["pgrx"], s2["pgry"], sign)
    with gpu.BarotropicSolver(b, resident=False) as s:
        got = s.shift_barotropic(f["uu"].copy(order="F"), f["vv"].copy(order="F"), s2["pgrx"], s2["pgry"], sign)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)
