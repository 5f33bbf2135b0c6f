"""Ensemble runs (inmsom_ens_*): members of different sizes and both fused
variants advanced by CUDA-graph launches -- one launch per member and
substep, or one persistent launch per group of substeps -- must end bit for
bit where each member run alone with inmsom_run_substeps ends: the same
work items and arithmetic on the same data; the work partition (changed by
the autotuner) does not change any value."""
import numpy as np
import pytest

from inmsom_elfs_b200 import basins

pytestmark = pytest.mark.gpu


def _members(gpu):
    out = []
    for k, (nx, ny) in enumerate(((96, 80), (130, 120), (200, 150), (64, 64))):
        b = basins.regional_basin(nx=nx, ny=ny, seed=60 + k)
        if k == 2:   # a 2-D viscosity: the general fused variant
            rng = np.random.default_rng(70)
            b.forcing["mu"] = np.asfortranarray(700.0 + 500.0 * rng.random(b.bounds.shape))
        b.taux *= 0.8 + 0.1 * k
        basins.finalize(b, gpu.GpuBackend(0))
        out.append(b)
    return out


def _alone(gpu, b, nsub, scale):
    bg = b.copy()
    with gpu.BarotropicSolver(bg, resident=True) as s:
        s.load_state()
        s.run_substeps(nsub, b.dt, scale)
        s.sync_to_host()
    return bg


def _ensemble(gpu, bs, nsub, scale, group, tune=False, persistent=False):
    cps = [b.copy() for b in bs]
    solvers = [gpu.BarotropicSolver(b, resident=True) for b in cps]
    for s in solvers:
        s.load_state()
    dts = [b.dt for b in cps]
    with gpu.Ensemble(solvers, group=group, persistent=persistent) as e:
        rows = None
        if tune:
            rows = e.tune(dts, trial_groups=1)
            for s in solvers:
                s.load_state()        # back to the initial state; the tuned partition stays
        e.run(nsub, dts, scale)
    for s in solvers:
        s.sync_to_host()
        s.close()
    return cps, rows


@pytest.mark.parametrize("tune,persistent", [(False, False), (True, False), (False, True), (True, True)])
def test_ensemble_matches_members_run_alone(gpu, tune, persistent):
    bs = _members(gpu)
    nsub = 22                                   # 5 graph launches of 4 and 2 direct substeps
    scale = basins.wind_cycle(nsub, 2.0, t0=300.0, period=600.0)
    ref = [_alone(gpu, b, nsub, scale) for b in bs]
    got, rows = _ensemble(gpu, bs, nsub, scale, group=4, tune=tune, persistent=persistent)
    for r, g in zip(ref, got):
        for k in r.state:
            assert np.array_equal(r.state[k], g.state[k]), k
    if tune:
        assert len(rows) == len(bs) and all(x in (0, 96, 64, 48, 32) for x in rows)


def test_ensemble_rejects_odd_group(gpu):
    from inmsom_elfs_b200 import InmsomError
    b = _members(gpu)[0]
    with gpu.BarotropicSolver(b.copy(), resident=True) as s:
        s.load_state()
        with pytest.raises(InmsomError):
            gpu.Ensemble([s], group=3)


def test_ensemble_rejects_a_member_given_twice(gpu):
    """Both entries would advance the same state in the same group."""
    from inmsom_elfs_b200 import InmsomError
    b = _members(gpu)[0]
    with gpu.BarotropicSolver(b.copy(), resident=True) as s:
        s.load_state()
        with pytest.raises(InmsomError, match="again"):
            gpu.Ensemble([s, s], group=4)


@pytest.mark.parametrize("persistent", [False, True])
def test_ensemble_odd_runs_back_to_back(gpu, persistent):
    """An odd run moves each member's state to its other ping-pong set; the
    next run must notice (recapture) and continue from there."""
    bs = _members(gpu)
    scale = basins.wind_cycle(10, 2.0, t0=100.0, period=600.0)
    ref = [_alone(gpu, b, 10, scale) for b in bs]
    cps = [b.copy() for b in bs]
    solvers = [gpu.BarotropicSolver(b, resident=True) for b in cps]
    for s in solvers:
        s.load_state()
    dts = [b.dt for b in cps]
    with gpu.Ensemble(solvers, group=4, persistent=persistent) as e:
        e.run(5, dts, scale[:5])       # one graph launch and one direct substep
        e.run(5, dts, scale[5:])
    for s in solvers:
        s.sync_to_host()
        s.close()
    for r, g in zip(ref, cps):
        for k in r.state:
            assert np.array_equal(r.state[k], g.state[k]), k


def test_ensemble_members_match_the_oracle(gpu, ora):
    """Every member of a mixed ensemble (both fused variants) against the
    CPU oracle run of the same member: normwise relative 1e-12 after 22
    substeps, as the single-basin fused path."""
    from conftest import rel_err
    bs = _members(gpu)
    nsub = 22
    scale = basins.wind_cycle(nsub, 2.0, t0=300.0, period=600.0)
    got, _ = _ensemble(gpu, bs, nsub, scale, group=4)
    for b, g in zip(bs, got):
        bo = b.copy()
        ora.hh_init_external(bo)
        ora.run_substeps(bo, nsub, b.dt, scale)
        for k in ("ssh_e", "ubrtr_e", "vbrtr_e", "sshp_e", "ubrtrp_e", "vbrtrp_e"):
            assert rel_err(g.state[k], bo.state[k]) <= 1e-12, (b.bounds.nx, k)


@pytest.mark.parametrize("persistent", [False, True])
def test_sixty_four_members_match_members_run_alone(gpu, persistent):
    """The configuration's member count: 64 regional basins of sides drawn
    from 64..256 in steps of 64 (seeded), wind amplitude +-20 %, 10 substeps
    (two replays of a group of 4 and two direct substeps), every member bit
    for bit its run alone."""
    rng = np.random.default_rng(64)
    bs = []
    for i, (n, a) in enumerate(zip(rng.choice([64, 128, 192, 256], size=64), rng.uniform(0.8, 1.2, size=64))):
        b = basins.regional_basin(nx=int(n), ny=int(n), seed=200 + i)
        b.taux *= a
        b.tauy *= a
        basins.finalize(b, gpu.GpuBackend(0))
        bs.append(b)
    nsub = 10
    scale = basins.wind_cycle(nsub, 2.0, t0=50.0, period=600.0)
    ref = [_alone(gpu, b, nsub, scale) for b in bs]
    got, _ = _ensemble(gpu, bs, nsub, scale, group=4, persistent=persistent)
    for r, g in zip(ref, got):
        for k in r.state:
            assert np.array_equal(r.state[k], g.state[k]), k
