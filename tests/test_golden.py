"""Golden regression fixtures (tests/golden/*.npz, made by
tests/golden/make_golden.py): four small seeded basins -- beta plane,
rotated spherical grid, regional coastline with 2-D forcing and the
biharmonic term, zonally periodic channel -- with every input and the
oracle's outputs after two barotropic_dynamics calls.

  * the oracle reproduces every stored output bit for bit (CPU);
  * the per-loop CUDA path reproduces them bit for bit (GPU);
  * the default path (fused where the basin is eligible) stays within the
    fused tolerance, 1e-12 normwise relative, on state, time means and
    depths.
"""
import numpy as np
import pytest

from conftest import rel_err
from golden.make_golden import CASE_NAMES, case_path, load_case

TOL = 1e-12


def test_fixtures_present():
    for name in CASE_NAMES:
        assert case_path(name).exists(), f"missing fixture {name}: run tests/golden/make_golden.py"


def _check_exact(basin, expected):
    for key, want in expected.items():
        grp, name = key.split(".", 1)
        got = getattr(basin, grp)[name]
        assert np.array_equal(got, want), f"{key}: max diff {np.max(np.abs(got - want))}"


@pytest.mark.parametrize("name", CASE_NAMES)
def test_oracle_matches_golden(ora, name):
    basin, p, expected = load_case(name)
    for _ in range(p["calls"]):
        ora.barotropic_dynamics(basin, p["tau"], p["nstep"], p["ksw4"])
    _check_exact(basin, expected)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASE_NAMES)
def test_general_path_matches_golden(gpu, name):
    basin, p, expected = load_case(name)
    with gpu.BarotropicSolver(basin, resident=False, force_general=True) as s:
        for _ in range(p["calls"]):
            s.barotropic_dynamics(p["tau"], p["nstep"], p["ksw4"])
        assert s.path()[0] == 0
    _check_exact(basin, expected)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASE_NAMES)
def test_default_path_matches_golden(gpu, name):
    basin, p, expected = load_case(name)
    with gpu.BarotropicSolver(basin, resident=True) as s:
        for _ in range(p["calls"]):
            s.barotropic_dynamics(p["tau"], p["nstep"], p["ksw4"])
        s.sync_to_host(0x1 | 0x2)
    for key, want in expected.items():
        grp, k = key.split(".", 1)
        assert rel_err(getattr(basin, grp)[k], want) <= TOL, key
