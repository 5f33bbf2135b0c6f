"""Known-answer and property tests of the CPU oracle (no GPU).

The reference ships no tests or golden vectors and cannot be built here
(no Fortran compiler, no MPI), so the oracle is checked by physics that
the reference scheme satisfies exactly or to rounding, and by restating
small pieces of the reference independently in numpy.
"""
import math

import numpy as np
import pytest

from conftest import rel_err
from inmsom_elfs_b200 import basins
from inmsom_elfs_b200.grid import Basin, Bounds, Consts


def _prep(b, ora):
    basins.finalize(b, ora.OracleBackend())
    ora.hh_init_external(b)
    return b


def test_gridcon_matches_definition(ora):
    # Service/grid_construction.f90:59-112 restated with numpy slicing
    rng = np.random.default_rng(5)
    b = Bounds.serial(23, 17)
    lu = b.zeros(np.float32)
    lu[b.interior] = (rng.random((b.nx, b.ny)) > 0.35).astype(np.float32)
    m = ora.gridcon(b, lu)
    s = b.sl(b.nx_start - 1, b.nx_end, b.ny_start - 1, b.ny_end)
    a = lu[s]
    r = lu[b.sl(b.nx_start, b.nx_end + 1, b.ny_start - 1, b.ny_end)]
    u = lu[b.sl(b.nx_start - 1, b.nx_end, b.ny_start, b.ny_end + 1)]
    ru = lu[b.sl(b.nx_start, b.nx_end + 1, b.ny_start, b.ny_end + 1)]
    expect = {
        "luh": (a + r + u + ru) > 0.5, "luu": (a * r * u * ru) > 0.5,
        "llu": (a + r) > 0.5, "llv": (a + u) > 0.5, "lcu": (a * r) > 0.5, "lcv": (a * u) > 0.5,
    }
    for k, e in expect.items():
        full = b.zeros(np.float32)
        full[s] = e.astype(np.float32)
        assert np.array_equal(m[k], full), k


def test_lake_at_rest_is_exact(ora):
    # zero wind, zero state, random topography: every field stays exactly 0
    b = basins.beta_plane_basin(n=40, seed=11)
    b.taux[...] = 0.0
    _prep(b, ora)
    for _ in range(30):
        ora.barotropic_dynamics(b, b.dt, 1, 0)
    for k, v in b.state.items():
        assert not np.any(v), k
    for k, v in b.means.items():
        assert not np.any(v), k


def test_volume_conserved(ora):
    # flux-form continuity telescopes; the Asselin filter is linear
    b = _prep(basins.beta_plane_basin(n=48, seed=2), ora)
    v0, _ = ora.diag(b)
    for _ in range(200):
        ora.barotropic_dynamics(b, b.dt, 1, 0)
    v1, e1 = ora.diag(b)
    assert abs(v1 - v0) / v0 < 1e-13
    assert e1 > 0.0
    assert ora.guard(b) == 0


def test_mirror_symmetry(ora):
    # flat bottom, f = 0, no wind, an x-symmetric SSH bump: the solution
    # stays mirror symmetric in x (u antisymmetric), to rounding
    b = basins.beta_plane_basin(n=31, ny=24, nbumps=0, seed=0)
    b.taux[...] = 0.0
    b.rlh_s[...] = 0.0
    _prep(b, ora)
    bd = b.bounds
    m = np.arange(bd.bnd_x1, bd.bnd_x2 + 1)[:, None]
    n = np.arange(bd.bnd_y1, bd.bnd_y2 + 1)[None, :]
    mc = 0.5 * (bd.nx_start + bd.nx_end)
    bump = 0.1 * np.exp(-((m - mc) ** 2 + (n - 12.0) ** 2) / 8.0) * (b.masks["lu"] > 0.5)
    b.state["ssh_e"][...] = bump
    b.state["sshp_e"][...] = bump
    ora.hh_init_external(b)
    for _ in range(40):
        ora.barotropic_dynamics(b, b.dt, 1, 0)
    s = b.state["ssh_e"][bd.interior]
    assert rel_err(s[::-1, :], s) < 1e-11
    u = b.state["ubrtr_e"][bd.sl(bd.nx_start, bd.nx_end - 1, bd.ny_start, bd.ny_end)]
    assert rel_err(-u[::-1, :], u) < 1e-10


def test_seiche_period(ora):
    # gravest seiche of a closed flat 1-D channel: period 2L/sqrt(gH) up to
    # the C-grid and leap-frog dispersion corrections (< 1 % here)
    nx, h, dx, dt = 64, 100.0, 1000.0, 10.0
    b = basins.beta_plane_basin(n=nx, ny=3, nbumps=0, spacing=dx, depth=h, dt=dt, drag=0.0,
                                visc=0.0, seed=0)
    b.taux[...] = 0.0
    b.rlh_s[...] = 0.0
    bd = b.bounds
    lu = bd.zeros(np.float32)
    lu[bd.sl(bd.nx_start, bd.nx_end, bd.ny_start + 1, bd.ny_start + 1)] = 1.0
    b.masks["lu"] = lu
    b.hhq_rest = np.asfortranarray(np.where(lu > 0.5, h, 0.0))
    _prep(b, ora)
    m = np.arange(bd.bnd_x1, bd.bnd_x2 + 1)[:, None]
    L = nx * dx
    x = (m - bd.nx_start + 0.5) * dx
    eta = 0.01 * np.cos(math.pi * x / L) * (lu > 0.5)
    b.state["ssh_e"][...] = eta
    b.state["sshp_e"][...] = eta
    ora.hh_init_external(b)
    probe = bd.sl(bd.nx_start, bd.nx_start, bd.ny_start + 1, bd.ny_start + 1)
    series = []
    for _ in range(2000):
        ora.barotropic_dynamics(b, dt, 1, 0)
        series.append(float(b.state["ssh_e"][probe][0, 0]))
    s = np.array(series)
    up = np.nonzero((s[:-1] < 0) & (s[1:] >= 0))[0]
    period = np.mean(np.diff(up)) * dt
    expect = 2 * L / math.sqrt(9.8 * h)
    assert abs(period / expect - 1.0) < 0.01


def test_r_diss_linear_slope(ora):
    # Control/init_pars.f90:459-481 on a uniform slope: r_fric*|grad H|
    b = basins.beta_plane_basin(n=20, seed=0)
    _prep(b, ora)
    bd = b.bounds
    m = np.arange(bd.bnd_x1, bd.bnd_x2 + 1)[:, None] * 1.0
    n = np.arange(bd.bnd_y1, bd.bnd_y2 + 1)[None, :] * 1.0
    b.hhq_rest = np.asfortranarray(1000.0 + 3.0 * m + 4.0 * n)
    r = ora.r_diss(b, 1e-4)
    # interior points whose four neighbours are ocean
    s = bd.sl(bd.nx_start + 2, bd.nx_end - 2, bd.ny_start + 2, bd.ny_end - 2)
    np.testing.assert_allclose(r[s], 1e-4 * 5.0 / 1.0e4, rtol=1e-14)


def test_ssh_internal_continuity(ora):
    # Function/vel_ssh.f90:707-719: a uniform transport divergence-free
    # field leaves SSH at sshp; the Asselin step then mixes levels
    b = _prep(basins.beta_plane_basin(n=16, seed=0), ora)
    bd = b.bounds
    ssh, sshp = bd.zeros(), bd.zeros()
    sshp[...] = 0.2 * (b.masks["lu"] > 0.5)
    u, v, wf = bd.zeros(), bd.zeros(), bd.zeros()
    hq = {k: bd.zeros() for k in ("q", "u", "v", "h")}
    ora.ssh_internal(b, 100.0, ssh, sshp, u, v, wf, hq["q"], hq["u"], hq["v"], hq["h"])
    ocean = b.masks["lu"] > 0.5
    assert np.all(ssh[ocean] == 0.2)
    # sshp_i = ssh + ts*(ssh_new - 2 ssh + sshp)/2 with ssh = 0
    np.testing.assert_array_equal(sshp[ocean], 0.0 + 0.05 * (0.2 - 0.0 + 0.2) / 2.0)


def test_guard_counts_nan_and_range(ora):
    b = _prep(basins.beta_plane_basin(n=16, seed=0), ora)
    bd = b.bounds
    i = (bd.nx_start + 3 - bd.bnd_x1, bd.ny_start + 3 - bd.bnd_y1)
    b.state["ssh_e"][i] = 12.0
    b.state["ubrtr_e"][i] = np.nan
    assert ora.guard(b) == 2
