"""FP32 velocity storage (INMSOM_FP32_VELOCITY) for inmsom_run_substeps.

u, up, v, vp live in FP32 on the device during a run and the momentum
arithmetic is FP32; SSH, its time levels and the continuity stay FP64.
Tolerances against the FP64 fused run and against the FP64 CPU oracle
(normwise relative, max|a-b|/max|b|), written here:
  * after 300 substeps of the 400 x 300 regional basin: SSH <= 1e-6,
    u and v (both levels) <= 2e-6;
  * the closed-basin volume is conserved to 1e-13 relative, as in FP64:
    the continuity differences the FP32 transports in FP64 (exactly), so
    each face's flux leaves one cell and enters the other;
  * land and halo points of the FP64 state are never written;
  * runs split by a change of the forcing continue as one run does.
"""
import numpy as np
import pytest

from conftest import rel_err
from inmsom_elfs_b200 import basins

pytestmark = pytest.mark.gpu

TOL_SSH = 1e-6
TOL_UV = 2e-6


def _run(gpu, b, nsub, fp32, scale=None):
    bg = b.copy()
    with gpu.BarotropicSolver(bg, resident=True, fp32_velocity=fp32) as s:
        s.load_state()
        s.run_substeps(nsub, b.dt, scale)
        s.sync_to_host()
        vol, en = s.diag()
    return bg, vol, en


def _prep(gpu, b):
    basins.finalize(b, gpu.GpuBackend(0))
    return b


def test_fp32_velocity_close_to_fp64(gpu):
    b = _prep(gpu, basins.regional_basin(nx=400, ny=300, seed=41))
    scale = basins.wind_cycle(300, b.dt, t0=0.0, period=1800.0)
    b64, _, _ = _run(gpu, b, 300, False, scale)
    b32, _, _ = _run(gpu, b, 300, True, scale)
    errs = {k: rel_err(b32.state[k], b64.state[k]) for k in b64.state}
    print("fp32 velocity normwise relative errors:", errs)
    assert errs["ssh_e"] <= TOL_SSH and errs["sshp_e"] <= TOL_SSH, errs
    for k in ("ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e"):
        assert errs[k] <= TOL_UV, (k, errs[k])
    # the velocities came back through FP32
    u = b32.state["ubrtr_e"]
    assert np.array_equal(u, u.astype(np.float32).astype(np.float64))


def test_fp32_velocity_against_the_fp64_oracle(gpu, ora):
    # the errors of the variant against the FP64 CPU oracle (the reference's
    # scheme): the same bounds as against the FP64 GPU run, which itself
    # stays within 1e-12 of the oracle over this many steps
    b = _prep(gpu, basins.regional_basin(nx=400, ny=300, seed=41))
    ora.hh_init_external(b)
    scale = basins.wind_cycle(300, b.dt, t0=0.0, period=1800.0)
    bo = b.copy()
    ora.run_substeps(bo, 300, b.dt, scale)
    b32, _, _ = _run(gpu, b, 300, True, scale)
    ocean = b.masks["lu"] > 0.5
    errs = {k: rel_err(b32.state[k], bo.state[k]) for k in bo.state}
    rms = {k: float(np.sqrt(np.mean((b32.state[k] - bo.state[k])[ocean] ** 2))) for k in bo.state}
    print("fp32 velocity vs FP64 oracle: normwise", errs, "rms", rms)
    assert errs["ssh_e"] <= TOL_SSH and errs["sshp_e"] <= TOL_SSH, errs
    for k in ("ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e"):
        assert errs[k] <= TOL_UV, (k, errs[k])


def test_fp32_velocity_runs_split_by_a_forcing_change(gpu):
    """An odd run (the state moves to the other ping-pong set), a new
    forcing, then two runs with it unchanged: against the FP64 runs of the
    same sequence, within the tolerances of one run -- a stale FP32 copy of
    the forcing or of either set would be far outside them."""
    b = _prep(gpu, basins.regional_basin(nx=400, ny=300, seed=45))
    out = {}
    for fp32 in (False, True):
        bg = b.copy()
        with gpu.BarotropicSolver(bg, resident=True, fp32_velocity=fp32) as s:
            s.load_state()
            s.run_substeps(7, b.dt)
            s.sync_to_host()
            for k in ("RHSx", "RHSy"):
                bg.forcing[k] *= 1.3
            s.load_state()
            s.run_substeps(6, b.dt)
            s.run_substeps(5, b.dt)
            s.sync_to_host()
        out[fp32] = bg
    errs = {k: rel_err(out[True].state[k], out[False].state[k]) for k in b.state}
    print("fp32 velocity split runs:", errs)
    assert errs["ssh_e"] <= TOL_SSH and errs["sshp_e"] <= TOL_SSH, errs
    for k in ("ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e"):
        assert errs[k] <= TOL_UV, (k, errs[k])


def test_fp32_velocity_at_the_4096_ridge_basin_size(gpu):
    """The configuration's own case: the 4096 x 4096 double-gyre ridge basin
    (2 km, dt 3 s, wind with a 6-hour cycle), 5000 steps of the FP32-velocity
    variant against the FP64 run.  Bounds (max over ocean points of |diff| /
    max |FP64|): u 1e-4, v 2e-4, SSH 1e-4 (measured on a B200: 3.7e-5, 1.0e-4,
    4.6e-5); the volume change as small as the FP64 run's (1e-13)."""
    b = _prep(gpu, basins.ridge_basin(n=4096))
    steps = 5000
    scale = basins.wind_cycle(steps, b.dt)
    out, dvol = {}, {}
    for fp32 in (False, True):
        bg = b.copy()
        with gpu.BarotropicSolver(bg, resident=True, fp32_velocity=fp32) as s:
            s.load_state()
            v0, _ = s.diag()
            s.run_substeps(steps, b.dt, scale)
            v1, _ = s.diag()
            s.sync_to_host()
        out[fp32], dvol[fp32] = bg, abs(v1 - v0) / v0
    ocean = b.masks["lu"] > 0.5
    err = {}
    for k in b.state:
        d = (out[True].state[k] - out[False].state[k])[ocean]
        err[k] = float(np.abs(d).max() / np.abs(out[False].state[k][ocean]).max())
    print("4096^2 ridge basin, 5000 steps, FP32 velocity vs FP64:", err, "volume change", dvol)
    assert err["ubrtr_e"] <= 1e-4 and err["ubrtrp_e"] <= 1e-4, err
    assert err["vbrtr_e"] <= 2e-4 and err["vbrtrp_e"] <= 2e-4, err
    assert err["ssh_e"] <= 1e-4 and err["sshp_e"] <= 1e-4, err
    assert dvol[True] <= 1e-13 and dvol[False] <= 1e-13, dvol


def test_fp32_velocity_conserves_volume(gpu):
    b = _prep(gpu, basins.beta_plane_basin(n=200, seed=42))
    lu = b.masks["lu"] > 0.5
    bump = 0.3 * np.exp(-((np.arange(b.bounds.shape[0])[:, None] - 90.0) ** 2 +
                          (np.arange(b.bounds.shape[1])[None, :] - 110.0) ** 2) / 200.0)
    b.state["ssh_e"] = np.asfortranarray(np.where(lu, bump, 0.0))
    b.state["sshp_e"] = b.state["ssh_e"].copy(order="F")
    with gpu.BarotropicSolver(b, resident=True, fp32_velocity=True) as s:
        s.load_state()
        v0, _ = s.diag()
        s.run_substeps(500, b.dt)
        v1, e1 = s.diag()
    assert abs(v1 - v0) / v0 <= 1e-13
    assert np.isfinite(e1) and e1 > 0.0


def test_fp32_velocity_leaves_land_untouched(gpu):
    b = _prep(gpu, basins.regional_basin(nx=260, ny=200, seed=43))
    rng = np.random.default_rng(44)
    land = b.masks["lu"] < 0.5
    for k in b.state:
        b.state[k] = np.asfortranarray(np.where(land, rng.standard_normal(b.bounds.shape), b.state[k]))
    b32, _, _ = _run(gpu, b, 51, True)
    for k in b.state:
        assert np.array_equal(b32.state[k][land], b.state[k][land]), k


def test_fp32_velocity_needs_uniform_variant(gpu):
    from inmsom_elfs_b200 import InmsomError
    from inmsom_elfs_b200 import _lib
    b = _prep(gpu, basins.spherical_basin(nx=64, ny=48))
    with gpu.BarotropicSolver(b, resident=True, fp32_velocity=True) as s:
        s.load_state()
        with pytest.raises(InmsomError) as e:
            s.run_substeps(4, b.dt)
        assert e.value.code == _lib.EUNSUPPORTED
