"""Parity at the sizes of the path's workload configurations.

* 256 x 256 beta-plane basin (10 km, f0 = 1e-4, beta = 2e-11, 4000 m minus
  Gaussian bumps, land ring, tau_x = 0.1 cos(pi y/Ly), A = 1e3, r = 1e-6,
  Asselin 0.05): the fused GPU path against the oracle after 10 and 1000
  steps, through the drop-in call and through the standalone run.  The
  configuration names dt = 20 s; at 4000 m and 10 km that violates the
  leap-frog gravity-wave limit (stability number 1.12), and a CPU test
  shows the oracle -- the reference's scheme -- tripping the range guard of
  Control/dyncall.f90:452-516 there, while at 15 s (0.84) it stays in
  range for the configuration's 1000 steps.  The GPU tests use 15 s.
* 2048 x 1536 regional basin (1 km, fractal coastline, log-normal depth,
  wind with a 6-hour cycle, dt = 2 s), the benchmark workload: masks
  bit-exact, the fused standalone run against the oracle after 10 and 1000
  steps, and 10,000 steps on the GPU conserving the volume to 1e-12.

Tolerances (Function/vel_ssh.f90:484-648 restated by the oracle): normwise
relative max|gpu - oracle| / max|oracle| <= 1e-12 after 10 steps and
<= 1e-10 after 1000 for SSH, u and v at both levels.
"""
import numpy as np
import pytest

from conftest import rel_err
from inmsom_elfs_b200 import basins

TOL10 = 1e-12
TOL1000 = 1e-10
STATE = ("ssh_e", "ubrtr_e", "vbrtr_e", "sshp_e", "ubrtrp_e", "vbrtrp_e")


def _close(bo, bg, tol):
    for k in STATE:
        e = rel_err(bg.state[k], bo.state[k])
        assert e <= tol, f"{k}: {e:.3e} > {tol:.0e}"


def test_beta_plane_256_dt20_violates_the_gravity_wave_limit(ora):
    b = basins.beta_plane_basin(n=256, dt=20.0)
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    assert basins.cfl_number(b) > 1.1
    tripped = None
    for k in range(400):
        ora.barotropic_dynamics(b, b.dt, 1, 0)
        if ora.guard(b) > 0:
            tripped = k + 1
            break
    assert tripped is not None and tripped < 400, tripped


def test_beta_plane_256_dt15_stays_in_range(ora):
    b = basins.beta_plane_basin(n=256)
    assert b.dt == 15.0 and basins.cfl_number(b) < 0.9
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    for _ in range(1000):
        ora.barotropic_dynamics(b, b.dt, 1, 0)
    assert ora.guard(b) == 0
    assert np.abs(b.state["ubrtr_e"]).max() > 1e-4     # the wind has spun up a flow


@pytest.mark.gpu
def test_beta_plane_256_drop_in_parity_10_and_1000(gpu, ora):
    b = basins.beta_plane_basin(n=256)
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    bo, bg = b.copy(), b.copy()
    with gpu.BarotropicSolver(bg, resident=True) as s:
        assert s.path() == (1, "eligible")
        for n in (10, 990):
            for _ in range(n):
                ora.barotropic_dynamics(bo, b.dt, 1)
                s.barotropic_dynamics(b.dt, 1)
            s.sync_to_host()
            _close(bo, bg, TOL10 if n == 10 else TOL1000)


@pytest.mark.gpu
def test_beta_plane_256_standalone_parity_10_and_1000(gpu, ora):
    b = basins.beta_plane_basin(n=256)
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    bo, bg = b.copy(), b.copy()
    with gpu.BarotropicSolver(bg, resident=True) as s:
        s.load_state()
        for n in (10, 990):
            ora.run_substeps(bo, n, b.dt)
            s.run_substeps(n, b.dt)
            s.sync_to_host()
            _close(bo, bg, TOL10 if n == 10 else TOL1000)


@pytest.fixture(scope="module")
def regional(gpu, ora):
    """The 2048 x 1536 benchmark basin with its masks and forcing from the
    oracle, and the GPU's gridcon of the same coastline."""
    b = basins.regional_basin()
    lu = b.masks["lu"]
    g = gpu.gridcon(b.bounds, lu)
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    return b, g


@pytest.mark.gpu
def test_regional_2048x1536_masks_bitexact(regional):
    b, g = regional
    for k, v in g.items():
        assert np.array_equal(v, b.masks[k]), k


@pytest.mark.gpu
def test_regional_2048x1536_parity_10_and_1000(gpu, ora, regional):
    b, _ = regional
    bo, bg = b.copy(), b.copy()
    scale = basins.wind_cycle(1000, b.dt)
    with gpu.BarotropicSolver(bg, resident=True) as s:
        assert s.path() == (1, "eligible")
        s.load_state()
        done = 0
        for n in (10, 990):
            ora.run_substeps(bo, n, b.dt, scale[done:done + n])
            s.run_substeps(n, b.dt, scale[done:done + n])
            done += n
            s.sync_to_host()
            _close(bo, bg, TOL10 if n == 10 else TOL1000)


@pytest.mark.gpu
def test_regional_2048x1536_volume_over_10000_steps(gpu, regional):
    b, _ = regional
    bg = b.copy()
    with gpu.BarotropicSolver(bg, resident=True) as s:
        s.load_state()
        v0, _ = s.diag()
        s.run_substeps(10000, b.dt, basins.wind_cycle(10000, b.dt))
        v1, e1 = s.diag()
        assert s.guard() == 0
    assert e1 > 0.0
    assert abs(v1 - v0) <= 1e-12 * abs(v0), (v1 - v0) / v0


@pytest.mark.gpu
def test_regional_2048x1536_drop_in_call_with_time_means(gpu, ora, regional):
    """The call the end-to-end measurement makes, at the benchmark basin's
    size: barotropic_dynamics(tau = 10 dt, nstep = 10) through the drop-in
    entry point (20 substeps, the state saved at the tenth, the four time
    means over all of them), twice, on a resident context with static
    coefficients, against the oracle: state and time means within 1e-12."""
    b, _ = regional
    bo, bg = b.copy(), b.copy()
    for _ in range(2):
        ora.barotropic_dynamics(bo, 10 * b.dt, 10)
    with gpu.BarotropicSolver(bg, resident=True, static_coeffs=True) as s:
        for _ in range(2):
            s.barotropic_dynamics(10 * b.dt, 10)
        s.sync_to_host(0x1 | 0x2)
        assert s.path() == (1, "eligible")
    _close(bo, bg, TOL10)
    for k in ("ubrtr_i", "vbrtr_i", "ssh4gradx", "ssh4grady"):
        e = rel_err(bg.means[k], bo.means[k])
        assert e <= TOL10, f"{k}: {e:.3e}"


@pytest.mark.gpu
def test_ridge_4096_fp64_parity_10(gpu, ora):
    """The 4096 x 4096 double-gyre ridge basin (2 km, dt 3 s), the FP32
    variant's reference run, in FP64 on the fused path against the oracle
    after 10 steps (1e-12); 16.8 M cells, the largest configuration."""
    b = basins.ridge_basin(n=4096)
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    bo, bg = b.copy(), b.copy()
    scale = basins.wind_cycle(10, b.dt)
    ora.run_substeps(bo, 10, b.dt, scale)
    with gpu.BarotropicSolver(bg, resident=True) as s:
        assert s.path() == (1, "eligible")
        s.load_state()
        s.run_substeps(10, b.dt, scale)
        s.sync_to_host()
    _close(bo, bg, TOL10)
