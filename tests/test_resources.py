"""Contexts and ensembles give back what they take: after one warm-up
round (the library's module is loaded and its one-time allocations made),
rounds that create a context on the fused path, run the drop-in call, the
standalone run (CUDA graphs), the FP32-velocity variant and an ensemble in
both forms, then destroy everything, leave the device's free memory where
it was (within 8 MiB: the driver's own bookkeeping)."""
import pytest

from inmsom_elfs_b200 import basins

pytestmark = pytest.mark.gpu


def _round(gpu, bs):
    for i, b in enumerate(bs):
        bg = b.copy()
        with gpu.BarotropicSolver(bg, resident=True, fp32_velocity=bool(i % 2)) as s:
            s.load_state()
            s.run_substeps(8, b.dt)
            s.run_substeps(3, b.dt)
            if not i % 2:
                s.barotropic_dynamics(4 * b.dt, 4)
            s.sync_to_host()
    solvers = [gpu.BarotropicSolver(b.copy(), resident=True) for b in bs]
    for s in solvers:
        s.load_state()
    dts = [b.dt for b in bs]
    for persistent in (False, True):
        with gpu.Ensemble(solvers, group=4, persistent=persistent) as e:
            e.run(10, dts)
    for s in solvers:
        s.close()


def test_contexts_and_ensembles_release_their_memory(gpu):
    import torch
    bs = []
    for k, (nx, ny) in enumerate(((300, 200), (180, 150), (256, 96))):
        b = basins.regional_basin(nx=nx, ny=ny, seed=80 + k)
        basins.finalize(b, gpu.GpuBackend(0))
        bs.append(b)
    _round(gpu, bs)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        _round(gpu, bs)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    assert free0 - free1 <= 8 << 20, (free0 - free1) / 2**20
