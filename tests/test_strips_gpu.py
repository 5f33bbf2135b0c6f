"""Row strips on one GPU (inmsom_strips_*): a basin split into strips, one
context each, advanced with one halo-row exchange per substep -- or, with
halos of 2k rows, k substeps per exchange computing into the halos -- must
end bit for bit where the single-domain fused run ends (both fused
variants)."""
import numpy as np
import pytest

from inmsom_elfs_b200 import basins
from inmsom_elfs_b200.strips import gather_state, split_basin

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nstrips,general,halo", [(3, False, 2), (2, True, 2), (4, False, 2),
                                                  (3, False, 4), (2, True, 6), (4, False, 8)])
def test_strips_match_single_domain(gpu, nstrips, general, halo):
    b = basins.regional_basin(nx=180, ny=170, seed=91)
    if general:
        rng = np.random.default_rng(92)
        b.forcing["mu"] = np.asfortranarray(600.0 + 600.0 * rng.random(b.bounds.shape))
    basins.finalize(b, gpu.GpuBackend(0))
    nsub = 41
    scale = basins.wind_cycle(nsub, b.dt, t0=100.0, period=700.0)
    ref = b.copy()
    with gpu.BarotropicSolver(ref, resident=True) as s:
        s.load_state()
        s.run_substeps(nsub, b.dt, scale)
        s.sync_to_host()
        assert s.path()[0] == 1
    parts = split_basin(b, nstrips, halo)
    solvers = [gpu.BarotropicSolver(p, resident=True) for p in parts]
    for s in solvers:
        assert s.path()[0] == 1, s.path()[1]
        s.load_state()
    with gpu.Strips(solvers) as g:
        g.run(nsub, b.dt, scale)
    for s in solvers:
        s.sync_to_host()
        s.close()
    got = gather_state(parts, b)
    for k, v in ref.state.items():
        assert np.array_equal(got.state[k], v), k
