"""inmsom_run_substeps replays a captured CUDA graph of 50 substeps (FP64
and FP32 velocity storage).  An odd number of substeps leaves the state in
the other ping-pong set; runs of odd and even lengths, graph-replayed or
launched directly, one after another must end bit for bit where one run of
the total length ends."""
import numpy as np
import pytest

from inmsom_elfs_b200 import basins

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fp32", [False, True])
def test_odd_runs_back_to_back(gpu, fp32):
    b = basins.regional_basin(nx=200, ny=150, seed=81)
    basins.finalize(b, gpu.GpuBackend(0))
    parts = (151, 9, 151, 100)            # graph + odd rest, direct, graph + odd rest, graph
    total = sum(parts)
    scale = basins.wind_cycle(total, b.dt, t0=0.0, period=1800.0)
    ref = b.copy()
    with gpu.BarotropicSolver(ref, resident=True, fp32_velocity=fp32) as s:
        s.load_state()
        s.run_substeps(total, b.dt, scale)
        s.sync_to_host()
    got = b.copy()
    with gpu.BarotropicSolver(got, resident=True, fp32_velocity=fp32) as s:
        s.load_state()
        k = 0
        for n in parts:
            s.run_substeps(n, b.dt, scale[k:k + n])
            k += n
        s.sync_to_host()
    for key in ref.state:
        assert np.array_equal(got.state[key], ref.state[key]), key
