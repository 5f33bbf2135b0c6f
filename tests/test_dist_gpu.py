"""One process per strip on the GPU (inmsom_step_*, inmsom_halo_*,
inmsom_elfs_b200.dist): two ranks, each with its own context for its strip,
advance with one halo exchange per substep, or with halos of 2k rows k
substeps per exchange (gloo, staged through host memory; both ranks on the one GPU this test gets -- their kernels never
wait for each other, the host exchange orders them) and must end bit for
bit where the single-domain fused run ends; the all-reduced volume and
energy equal the single-domain diagnostics to 1e-13 / 1e-12 relative."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
NSUB = 23


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _basin():
    from inmsom_elfs_b200 import basins, solver
    b = basins.regional_basin(nx=160, ny=150, seed=93)
    basins.finalize(b, solver.GpuBackend(0))
    return b


def _rank(rank, world, port, q, halo):
    import torch
    import torch.distributed as dist
    from inmsom_elfs_b200 import basins, solver
    from inmsom_elfs_b200.dist import GpuStripStepper, run_strip
    from inmsom_elfs_b200.strips import split_basin
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        b = _basin()
        loc = split_basin(b, world, halo)[rank]
        scale = basins.wind_cycle(NSUB, b.dt, t0=50.0, period=900.0)
        from inmsom_elfs_b200.dist import diag
        with solver.BarotropicSolver(loc, resident=True) as s:
            s.load_state()
            run_strip(GpuStripStepper(s, host_staging=True), rank, world, NSUB, b.dt, scale)
            s.sync_to_host()
            vol, en = diag(s)
        q.put((rank, {k: v for k, v in loc.state.items()}, (vol, en)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("halo", [2, 6])
def test_two_ranks_match_single_domain(gpu, halo):
    from inmsom_elfs_b200 import basins
    from inmsom_elfs_b200.strips import gather_state, split_basin
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q, halo)) for r in range(2)]
    for p in procs:
        p.start()
    got, dg = {}, {}
    for _ in range(2):
        r, st, d = q.get(timeout=300)
        got[r], dg[r] = st, d
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    b = _basin()
    scale = basins.wind_cycle(NSUB, b.dt, t0=50.0, period=900.0)
    ref = b.copy()
    with gpu.BarotropicSolver(ref, resident=True) as s:
        s.load_state()
        s.run_substeps(NSUB, b.dt, scale)
        s.sync_to_host()
        vol, en = s.diag()
    # the all-reduced diagnostics: the same on both ranks, the single-domain
    # sums up to the order of the additions
    assert dg[0] == dg[1]
    assert abs(dg[0][0] - vol) <= 1e-13 * abs(vol) and abs(dg[0][1] - en) <= 1e-12 * abs(en)
    parts = split_basin(b, 2, halo)
    for r in range(2):
        parts[r].state.update(got[r])
    merged = gather_state(parts, b)
    for k, v in ref.state.items():
        assert np.array_equal(merged.state[k], v), k


def test_step_entry_points_check_their_arguments(gpu):
    import ctypes
    from inmsom_elfs_b200 import InmsomError, _lib
    b = _basin()
    with gpu.BarotropicSolver(b, resident=True) as s:
        lib = _lib.load()
        with pytest.raises(InmsomError):           # no resident state yet
            _lib.check(lib.inmsom_step_begin(s._ctx))
        s.load_state()
        with pytest.raises(InmsomError):           # not begun
            _lib.check(lib.inmsom_step_launch(s._ctx, b.dt, 1.0))
        with pytest.raises(InmsomError):
            _lib.check(lib.inmsom_halo_pack(s._ctx, 2, ctypes.c_void_p(1)))
        _lib.check(lib.inmsom_step_begin(s._ctx))
        with pytest.raises(InmsomError):           # rows beyond a basin edge
            _lib.check(lib.inmsom_step_launch_rows(s._ctx, b.dt, 1.0, 2, 0))
        _lib.check(lib.inmsom_step_end(s._ctx))
        assert lib.inmsom_gpu_pitch(s._ctx) % 32 == 0
