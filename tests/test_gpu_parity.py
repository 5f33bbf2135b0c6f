"""Parity of the CUDA library with the CPU oracle, through the C ABI.

Tolerances:
  * general (per-loop) path: bit-exact (np.array_equal) for every state,
    time-mean, depth and scratch array -- it is compiled with
    --fmad=false and keeps the Fortran expression order;
  * fused path: normwise relative difference max|gpu-oracle|/max|oracle|
    <= 1e-12 after 10 steps and <= 1e-10 after 1000 steps on SSH, u and v
    (the contract for the FP64 plain form), and the same bound on the
    time means;
  * masks, index ranges and untouched (land / halo) points: bit-exact.
"""
import numpy as np
import pytest

from conftest import rel_err
from inmsom_elfs_b200 import basins
from inmsom_elfs_b200.grid import DEPTHS, MEANS, SCRATCH, STATE, Bounds

pytestmark = pytest.mark.gpu

TOL10 = 1e-12
TOL1000 = 1e-10


def prep(b, ora):
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    return b


def run_pair(gpu, ora, b, calls, tau, nstep, ksw4=0, force_general=False, resident=False):
    """Run `calls` barotropic_dynamics calls on the oracle and on the GPU
    from copies of the same basin; return (oracle basin, gpu basin, path)."""
    bo, bg = b.copy(), b.copy()
    for _ in range(calls):
        ora.barotropic_dynamics(bo, tau, nstep, ksw4)
    with gpu.BarotropicSolver(bg, resident=resident, force_general=force_general) as s:
        for _ in range(calls):
            s.barotropic_dynamics(tau, nstep, ksw4)
        if resident:
            s.sync_to_host(0x1 | 0x2 | 0x4)
        path = s.path()
    return bo, bg, path


def assert_bitexact(bo, bg, groups=("state", "means", "depths", "scratch")):
    for grp in groups:
        for k, v in getattr(bo, grp).items():
            w = getattr(bg, grp)[k]
            assert np.array_equal(v, w), f"{grp}.{k}: max diff {np.max(np.abs(v - w))}"


def assert_close(bo, bg, tol, names=("ssh_e", "ubrtr_e", "vbrtr_e", "sshp_e", "ubrtrp_e", "vbrtrp_e")):
    for k in names:
        e = rel_err(bg.state[k], bo.state[k])
        assert e <= tol, f"{k}: {e:.3e} > {tol:.0e}"


# ---------------------------------------------------------------- set-up
def test_gridcon_bitexact(gpu, ora):
    rng = np.random.default_rng(0)
    for nx, ny in ((5, 4), (37, 29), (130, 70)):
        b = Bounds.serial(nx, ny)
        lu = b.zeros(np.float32)
        lu[...] = (rng.random(b.shape) > 0.3).astype(np.float32)   # halo included
        mo = ora.gridcon(b, lu)
        mg = gpu.gridcon(b, lu)
        for k in mo:
            assert np.array_equal(mo[k], mg[k]), k


def test_wind_forcing_and_r_diss_bitexact(gpu, ora):
    b = prep(basins.regional_basin(nx=150, ny=97, seed=4), ora)
    with gpu.BarotropicSolver(b) as s:
        rx, ry = s.wind_forcing(b.taux, b.tauy)
        assert np.array_equal(rx, b.forcing["RHSx"])
        assert np.array_equal(ry, b.forcing["RHSy"])
        # Control/init_pars.f90:465,467 divide by lcu(m)+lcu(m-1) (lcv sums):
        # 0/0 = NaN at ocean points without an ocean neighbour along an axis,
        # on both sides alike
        ro, rg = ora.r_diss(b, 1e-4), s.r_diss(1e-4)
        assert np.array_equal(rg, ro, equal_nan=True)
        assert np.array_equal(np.isnan(rg), np.isnan(ro))


# ---------------------------------------------------------- general path
@pytest.mark.parametrize("nstep,calls,ksw4", [(1, 10, 0), (3, 4, 0), (2, 3, 1)])
def test_general_bitexact_beta_plane(gpu, ora, nstep, calls, ksw4):
    b = prep(basins.beta_plane_basin(n=48, ny=40, seed=7), ora)
    if ksw4:
        b.forcing["mu4"][...] = 3.0e8 * (1.0 + 0.1 * np.random.default_rng(1).random(b.bounds.shape))
    bo, bg, path = run_pair(gpu, ora, b, calls, nstep * b.dt, nstep, ksw4, force_general=True)
    assert path[0] == 0
    assert_bitexact(bo, bg)


def test_general_bitexact_spherical_rotated(gpu, ora):
    # rotated sphere: Coriolis varies along x -> general path by eligibility
    b = prep(basins.spherical_basin(nx=40, ny=30, rotation_on_lat=20.0), ora)
    bo, bg, path = run_pair(gpu, ora, b, 8, b.dt, 1)
    assert path[0] == 0 and "vary" in path[1]
    assert_bitexact(bo, bg)


def test_general_bitexact_ocean_halo(gpu, ora):
    # ocean in the halo ring: the Asselin/hh_shift ranges reach the ring
    b = basins.beta_plane_basin(n=30, ny=26, seed=8)
    b.masks["lu"][...] = 1.0
    b.hhq_rest[...] = 3000.0
    prep(b, ora)
    bo, bg, path = run_pair(gpu, ora, b, 6, 2 * b.dt, 2)
    assert path[0] == 0 and "halo" in path[1]
    assert_bitexact(bo, bg)


def test_general_bitexact_2d_metrics(gpu, ora):
    b = basins.beta_plane_basin(n=33, ny=27, seed=9)
    rng = np.random.default_rng(3)
    for k, v in b.metrics.items():
        v *= 1.0 + 0.05 * rng.random(v.shape)
    prep(b, ora)
    bo, bg, path = run_pair(gpu, ora, b, 6, b.dt, 1)
    assert path[0] == 0
    assert_bitexact(bo, bg)


def test_general_resident_matches_copy_mode(gpu, ora):
    b = prep(basins.beta_plane_basin(n=40, seed=12), ora)
    bo, bg, _ = run_pair(gpu, ora, b, 5, b.dt, 1, force_general=True, resident=True)
    assert_bitexact(bo, bg, groups=("state", "means", "depths"))


def test_ssh_internal_bitexact(gpu, ora):
    b = prep(basins.beta_plane_basin(n=36, seed=13), ora)
    rng = np.random.default_rng(2)
    bd = b.bounds
    arrays = [rng.standard_normal(bd.shape) * s for s in (0.1, 0.1, 50.0, 50.0, 1e-3)]
    arrays = [np.asfortranarray(a) for a in arrays] + [bd.zeros() for _ in range(4)]
    ao = [a.copy(order="F") for a in arrays]
    ag = [a.copy(order="F") for a in arrays]
    ora.ssh_internal(b, 300.0, *ao)
    with gpu.BarotropicSolver(b) as s:
        s.ssh_internal(300.0, *ag)
    for x, y in zip(ao, ag):
        assert np.array_equal(x, y)


# ------------------------------------------------------------ fused path
def test_fused_parity_10_and_1000_steps(gpu, ora):
    # 300 x 200: three column strips and several row chunks
    b = prep(basins.beta_plane_basin(n=300, ny=200, seed=14), ora)
    bo, bg = b.copy(), b.copy()
    with gpu.BarotropicSolver(bg, resident=True) as s:
        assert s.path() == (1, "eligible")
        for _ in range(10):
            ora.barotropic_dynamics(bo, b.dt, 1)
            s.barotropic_dynamics(b.dt, 1)
        s.sync_to_host()
        assert_close(bo, bg, TOL10)
        for k in MEANS:
            assert rel_err(bg.means[k], bo.means[k]) <= TOL10, k
        for _ in range(990):
            ora.barotropic_dynamics(bo, b.dt, 1)
            s.barotropic_dynamics(b.dt, 1)
        s.sync_to_host(0x1 | 0x2)
    assert_close(bo, bg, TOL1000)
    for k in DEPTHS:
        assert rel_err(bg.depths[k], bo.depths[k]) <= TOL1000, k


def test_fused_dynamics_nstep(gpu, ora):
    # 2*nstep substeps, state saved at nstep, time means over all of them
    b = prep(basins.regional_basin(nx=270, ny=140, seed=15), ora)
    bo, bg, path = run_pair(gpu, ora, b, 3, 6 * b.dt, 6)
    assert path[0] == 1
    assert_close(bo, bg, TOL10)
    for k in MEANS:
        assert rel_err(bg.means[k], bo.means[k]) <= TOL10, k


@pytest.mark.parametrize("force_general", [False, True])
def test_run_substeps_with_wind_cycle(gpu, ora, force_general):
    b = prep(basins.regional_basin(nx=260, ny=200, seed=16), ora)
    scale = basins.wind_cycle(200, b.dt, t0=1800.0, period=600.0)
    bo, bg = b.copy(), b.copy()
    ora.run_substeps(bo, 200, b.dt, scale)
    with gpu.BarotropicSolver(bg, resident=True, force_general=force_general) as s:
        s.load_state()
        s.run_substeps(200, b.dt, scale)
        s.sync_to_host()
        assert s.path()[0] == (0 if force_general else 1)
    if force_general:
        assert_bitexact(bo, bg, groups=("state",))
    else:
        assert_close(bo, bg, TOL10 * 10)


def test_fused_spherical_metrics(gpu, ora):
    # metrics vary along y: per-row coefficients, non-zero metric vorticity
    b = prep(basins.spherical_basin(nx=140, ny=90, seed=17), ora)
    bo, bg, path = run_pair(gpu, ora, b, 10, b.dt, 1)
    assert path[0] == 1
    assert_close(bo, bg, TOL10)


def test_fused_nonuniform_forcing(gpu, ora):
    # viscosity, drag and water flux vary in space: the 2-D-forcing variant
    b = basins.beta_plane_basin(n=140, ny=100, seed=18)
    rng = np.random.default_rng(4)
    b.forcing["mu"] *= 1.0 + 0.5 * rng.random(b.bounds.shape)
    b.forcing["rdis"] *= 1.0 + rng.random(b.bounds.shape)
    b.forcing["wflux"][...] = 1e-5 * rng.standard_normal(b.bounds.shape)
    prep(b, ora)
    bo, bg, path = run_pair(gpu, ora, b, 10, b.dt, 1)
    assert path[0] == 1
    assert_close(bo, bg, TOL10)


@pytest.mark.parametrize("force_general", [False, True])
def test_untouched_points_keep_their_values(gpu, ora, force_general):
    # values at land u/v/T points and in the halo are never written by the
    # reference (vel_ssh.f90:589-612 masks); poison them and compare exactly
    b = prep(basins.beta_plane_basin(n=150, ny=60, seed=19), ora)
    for k in STATE:
        m = b.masks["lu"] if k.startswith("ssh") else (b.masks["lcu"] if k.startswith("u") else b.masks["lcv"])
        b.state[k][m < 0.5] = 0.125
    ora.hh_init_external(b)
    bo, bg, path = run_pair(gpu, ora, b, 5, b.dt, 1, force_general=force_general)
    assert path[0] == (0 if force_general else 1)
    for k in STATE:
        m = b.masks["lu"] if k.startswith("ssh") else (b.masks["lcu"] if k.startswith("u") else b.masks["lcv"])
        assert np.array_equal(bg.state[k][m < 0.5], bo.state[k][m < 0.5]), k
    if force_general:
        assert_bitexact(bo, bg)
    else:
        assert_close(bo, bg, TOL10)


# -------------------------------------------------------- diagnostics
def test_diag_and_guard(gpu, ora):
    b = prep(basins.beta_plane_basin(n=100, seed=20), ora)
    for _ in range(20):
        ora.barotropic_dynamics(b, b.dt, 1)
    with gpu.BarotropicSolver(b, resident=True) as s:
        s.load_state()
        v, e = s.diag()
        vo, eo = ora.diag(b)
        assert abs(v - vo) / vo < 1e-13
        assert abs(e - eo) / eo < 1e-12
        assert s.guard() == 0


def test_guard_trips_and_context_survives(gpu, ora):
    from inmsom_elfs_b200 import InmsomError
    b = prep(basins.beta_plane_basin(n=64, seed=21), ora)
    bad = b.copy()
    bad.state["ssh_e"][b.masks["lu"] > 0.5] = 11.0    # both levels: a sea at rest
    bad.state["sshp_e"][b.masks["lu"] > 0.5] = 11.0
    with gpu.BarotropicSolver(bad, guard=True) as s:
        with pytest.raises(InmsomError) as ei:
            s.barotropic_dynamics(b.dt, 1)
        assert ei.value.code == 3
        # the same context keeps working once the state is sane again
        for k in STATE:
            bad.state[k][...] = b.state[k]
        s.sync_from_host()       # resident context: re-upload the sane state
        s.barotropic_dynamics(b.dt, 1)


def test_last_phases_cover_the_call(gpu, ora):
    """inmsom_gpu_last_phases: upload, substeps and download of the last
    barotropic_dynamics call, each positive, together within the call's
    wall time; before any call it is an argument error."""
    import time
    from inmsom_elfs_b200 import InmsomError, _lib
    b = prep(basins.regional_basin(nx=200, ny=150, seed=17), ora)
    with gpu.BarotropicSolver(b, resident=True) as s:
        with pytest.raises(InmsomError) as e:
            s.last_phases()
        assert e.value.code == _lib.EARG
        s.barotropic_dynamics(4 * b.dt, 4)
        t0 = time.perf_counter()
        s.barotropic_dynamics(4 * b.dt, 4)
        wall = (time.perf_counter() - t0) * 1e3
        up, comp, down = s.last_phases()
        assert up > 0 and comp > 0 and down > 0
        assert up + comp + down <= wall * 1.05 + 0.05


@pytest.mark.parametrize("with_all", [True, False])
def test_rhs2d_bitexact(gpu, ora, with_all):
    """inmsom_rhs2d (Control/dyncall.f90:110-130) against the oracle's
    restatement, bit for bit, with every term given or with some absent."""
    b = prep(basins.regional_basin(nx=180, ny=130, seed=18), ora)
    rng = np.random.default_rng(19)
    f = lambda: np.asfortranarray(rng.standard_normal(b.bounds.shape))
    args = dict(diff_disp=(f(), f()), tran=(f(), f()), tran_disp=(f(), f()), surf_stress=(f(), f()),
                bot_stress=(f(), f()), slpr=f(), hhu=np.abs(f()) * 100.0, hhv=np.abs(f()) * 100.0)
    if not with_all:
        args.update(tran=(None, None), bot_stress=(f(), None), slpr=None)
    rx, ry = f(), f()
    ox, oy = ora.rhs2d(b, rx.copy(order="F"), ry.copy(order="F"), **args)
    with gpu.BarotropicSolver(b, resident=True) as s:
        gx, gy = s.rhs2d(rx.copy(order="F"), ry.copy(order="F"), **args)
    assert np.array_equal(gx, ox) and np.array_equal(gy, oy)
    assert not np.array_equal(gx, rx)


def test_velocity2d_bitexact(gpu, ora):
    """inmsom_velocity2d (Control/dyncall.f90:188-201) against the oracle's
    restatement, bit for bit, after a call of barotropic_dynamics."""
    b = prep(basins.regional_basin(nx=170, ny=140, seed=20), ora)
    with gpu.BarotropicSolver(b, resident=True) as s:
        s.barotropic_dynamics(4 * b.dt, 4)
        s.sync_to_host(0x1 | 0x2)
        rng = np.random.default_rng(21)
        f = lambda: np.asfortranarray(rng.standard_normal(b.bounds.shape))
        slpr = f()
        hhu = np.asfortranarray(b.depths["hhu_e"] + 1.0)   # no zero depth at masked points
        hhv = np.asfortranarray(b.depths["hhv_e"] + 1.0)
        args = [b.means["ubrtr_i"], b.means["vbrtr_i"], slpr, hhu, hhv]
        outs = [f(), f(), f(), f()]
        got = s.velocity2d(*[o.copy(order="F") for o in outs], *args)
    ref = ora.velocity2d(b, *[o.copy(order="F") for o in outs], *args)
    for g_, r_ in zip(got, ref):
        assert np.array_equal(g_, r_)
    assert not np.array_equal(got[0], outs[0])


def test_static_coeffs_stay_resident(gpu, ora):
    # INMSOM_STATIC_COEFFS: wflux, mu and rdis are copied in by the first
    # call and kept; a change on the host reaches the device only after
    # inmsom_gpu_sync_from_host(INMSOM_SYNC_COEFFS)
    from inmsom_elfs_b200 import _lib
    b = prep(basins.regional_basin(nx=200, ny=120, seed=21), ora)
    bo, bg = b.copy(), b.copy()
    with gpu.BarotropicSolver(bg, resident=True, static_coeffs=True) as s:
        ora.barotropic_dynamics(bo, 4 * b.dt, 4)
        s.barotropic_dynamics(4 * b.dt, 4)
        bg.forcing["mu"][...] *= 3.0                    # not seen by the device
        ora.barotropic_dynamics(bo, 4 * b.dt, 4)
        s.barotropic_dynamics(4 * b.dt, 4)
        s.sync_to_host()
        assert_close(bo, bg, TOL10)
        bo.forcing["mu"][...] *= 3.0
        s.sync_from_host(_lib.SYNC_COEFFS)
        ora.barotropic_dynamics(bo, 4 * b.dt, 4)
        s.barotropic_dynamics(4 * b.dt, 4)
        s.sync_to_host()
    assert_close(bo, bg, TOL10)
    for k in MEANS:
        assert rel_err(bg.means[k], bo.means[k]) <= TOL10, k


@pytest.mark.parametrize("nx,ny", [(3, 3), (5, 4), (17, 9), (29, 6), (31, 5), (61, 3), (7, 40)])
def test_tiny_and_ragged_basins(gpu, ora, nx, ny):
    """Basins smaller than a strip (30 columns) or a work item (4 rows), one
    ocean cell upward, and strips cut one or two columns into the next: the
    fused path against the oracle after 10 steps (1e-12) and the per-loop
    path bit for bit."""
    b = prep(basins.beta_plane_basin(n=nx, ny=ny, seed=nx * 100 + ny), ora)
    bo, bg, path = run_pair(gpu, ora, b, 10, b.dt, 1)
    assert path[0] == 1, path
    assert_close(bo, bg, TOL10)
    bo, bg, path = run_pair(gpu, ora, b, 10, b.dt, 1, force_general=True)
    assert path[0] == 0
    assert_bitexact(bo, bg, groups=("state",))


@pytest.mark.parametrize("force_general", [False, True])
def test_all_land_basin_keeps_its_state(gpu, ora, force_general):
    """An empty ocean (every point land): both paths run and leave every
    state array as it was, as the oracle does."""
    b = basins.beta_plane_basin(n=40, ny=30, seed=5)
    b.masks["lu"][...] = 0.0
    b.hhq_rest[...] = 0.0
    prep(b, ora)
    bo, bg, path = run_pair(gpu, ora, b, 5, b.dt, 1, force_general=force_general)
    assert path[0] == (0 if force_general else 1), path
    for k in STATE:
        assert np.array_equal(bg.state[k], b.state[k]), k
        assert np.array_equal(bo.state[k], b.state[k]), k


@pytest.mark.parametrize("force_general", [False, True])
def test_land_values_do_not_reach_the_ocean(gpu, ora, force_general):
    """Random values at every land and halo point of the state (the
    reference never writes them, and its stencils weight them by masks):
    the ocean points match the oracle (fused 1e-12, per-loop bit for bit)
    and the land points keep their values."""
    b = basins.regional_basin(nx=120, ny=90, seed=23)
    prep(b, ora)
    rng = np.random.default_rng(24)
    land = b.masks["lu"] < 0.5
    for k in STATE:
        b.state[k] = np.asfortranarray(np.where(land, rng.standard_normal(b.bounds.shape), b.state[k]))
    bo, bg, path = run_pair(gpu, ora, b, 10, b.dt, 1, force_general=force_general)
    assert path[0] == (0 if force_general else 1), path
    if force_general:
        assert_bitexact(bo, bg, groups=("state",))
    else:
        assert_close(bo, bg, TOL10)
    for k in STATE:
        assert np.array_equal(bg.state[k][land], b.state[k][land]), k


def test_fixed_depth_free_surface_off(gpu, ora):
    """full_free_surface = 0 (Inc/basinpar.fi: the depths stay at the rest
    depth and the water flux leaves the continuity): the fused path refuses
    it and the per-loop path follows the oracle bit for bit, time means and
    depths included."""
    import dataclasses
    b = basins.regional_basin(nx=90, ny=70, seed=29)
    b.consts = dataclasses.replace(b.consts, full_free_surface=0)
    b.forcing["wflux"] = np.asfortranarray(1e-4 * np.random.default_rng(30).standard_normal(b.bounds.shape))
    prep(b, ora)
    bo, bg, path = run_pair(gpu, ora, b, 4, 3 * b.dt, 3)
    assert path[0] == 0 and "full_free_surface" in path[1], path
    assert_bitexact(bo, bg, groups=("state", "means", "depths"))


@pytest.mark.parametrize("px,py", [(1, 0), (0, 1), (1, 1)])
def test_general_bitexact_periodic(gpu, ora, px, py):
    """Periodic wraps of the barotropic step (Service/oc_algorithms.f90:50-135
    after every field update) in x, y and both, on a basin with a seeded
    island and a non-uniform Coriolis field: the per-loop path bit for bit
    with the oracle, time means and depths included."""
    from inmsom_elfs_b200.grid import Basin, Consts
    rng = np.random.default_rng(40 + 2 * px + py)
    nx, ny = 36, 28
    bd = Bounds.serial(nx, ny, periodicity_x=px, periodicity_y=py)
    b = Basin(bd, Consts())
    lu = np.ones(bd.shape, dtype=np.float32, order="F")
    if not py:
        lu[:, : bd.nnn - bd.bnd_y1] = 0.0
        lu[:, bd.nn - bd.bnd_y1 + 1:] = 0.0
    if not px:
        lu[: bd.mmm - bd.bnd_x1, :] = 0.0
        lu[bd.mm - bd.bnd_x1 + 1:, :] = 0.0
    i0, j0 = bd.mmm - bd.bnd_x1 + nx // 3, bd.nnn - bd.bnd_y1 + ny // 3
    lu[i0:i0 + 3, j0:j0 + 2] = 0.0
    b.masks["lu"] = np.asfortranarray(lu)
    basins.uniform_metrics(b, 5.0e3)
    b.rlh_s = np.asfortranarray(1.0e-4 + 1.0e-5 * rng.standard_normal(bd.shape))
    b.hhq_rest = np.asfortranarray(np.where(lu > 0.5, 200.0 * (0.8 + 0.4 * rng.random(bd.shape)), 0.0))
    b.taux = np.asfortranarray(0.1 * rng.standard_normal(bd.shape))
    b.tauy = np.asfortranarray(0.1 * rng.standard_normal(bd.shape))
    b.forcing["mu"] = np.full(bd.shape, 300.0, order="F")
    b.forcing["rdis"] = np.full(bd.shape, 1.0e-6, order="F")
    b.dt = 20.0
    prep(b.fill_defaults(), ora)
    bo, bg, path = run_pair(gpu, ora, b, 5, 2 * b.dt, 2)
    assert path[0] == 0 and "periodic" in path[1], path
    assert_bitexact(bo, bg, groups=("state", "means", "depths"))
