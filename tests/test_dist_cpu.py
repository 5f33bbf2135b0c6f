"""One process per strip (inmsom_elfs_b200.dist): the halo exchange between
gloo ranks on CPU, with a radius-2 numpy stencil standing in for the GPU
substep, must reproduce the single-domain run bit for bit (2 and 3 ranks),
with the reference's two halo rows (an exchange per substep) and with wide
halos of 2k rows (k substeps per exchange, computing into the halo, the
last block of a run shorter); the FP64 all-reduce of the diagnostics (dist.diag) must
give every rank the single-domain volume and energy.  The GPU side of the
same exchange is tested in test_dist_gpu.py."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

NX, ROWS, NSUB = 19, 41, 7      # global rows incl. 2 halo rows each side


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fields():
    rng = np.random.default_rng(5)
    return rng.standard_normal((6, NX, ROWS))


def _split(world):
    """interior rows [2, ROWS-3] cut into `world` strips: (first, last) global rows"""
    ny = ROWS - 4
    locn = ny // world
    out = []
    for k in range(world):
        a = 2 + k * locn
        b = a + locn - 1 if k < world - 1 else ROWS - 3
        out.append((a, b))
    return out


def _rank(rank, world, port, q, halo):
    import torch.distributed as dist
    from inmsom_elfs_b200.dist import NumpyStripStepper, run_strip, substeps_per_exchange
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a, b = _split(world)[rank]
        hs = halo if rank > 0 else 2
        hn = halo if rank + 1 < world else 2
        f = _fields()[:, :, a - hs:b + hn + 1]
        st = NumpyStripStepper(f, (hs, b - a + hs))
        assert substeps_per_exchange(st, rank, world) == halo // 2
        run_strip(st, rank, world, NSUB, 0.5, np.linspace(0.5, 1.5, NSUB))
        q.put((rank, st.f[:, :, hs:b - a + hs + 1]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,halo", [(2, 2), (3, 2), (2, 4), (3, 6)])
def test_gloo_ranks_reproduce_one_domain(world, halo):
    from inmsom_elfs_b200.dist import NumpyStripStepper, run_strip
    ref = NumpyStripStepper(_fields(), (2, ROWS - 3))
    run_strip(ref, 0, 1, NSUB, 0.5, np.linspace(0.5, 1.5, NSUB))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, halo)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    merged = np.concatenate([got[r] for r in range(world)], axis=2)
    assert np.array_equal(merged, ref.f[:, :, 2:ROWS - 2])


class _StripDiag:
    """Stands in for a strip's solver: diag() is the oracle's volume and
    energy over the strip's interior rows."""

    def __init__(self, basin):
        self.basin = basin

    def diag(self):
        from oracle import oracle as ora
        return ora.diag(self.basin)


def _basin():
    from inmsom_elfs_b200 import basins
    from oracle import oracle as ora
    b = basins.regional_basin(nx=48, ny=41, seed=93)
    basins.finalize(b, ora.OracleBackend())
    rng = np.random.default_rng(7)
    for k in ("ssh_e", "ubrtr_e", "vbrtr_e"):
        b.state[k] = np.asfortranarray(0.1 * rng.standard_normal(b.bounds.shape))
    return b


def _diag_rank(rank, world, port, q):
    import torch.distributed as dist
    from inmsom_elfs_b200.dist import diag
    from inmsom_elfs_b200.strips import split_basin
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        strip = split_basin(_basin(), world)[rank]
        q.put((rank, diag(_StripDiag(strip))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_diag_sums_the_strips(world):
    """dist.diag: every rank gets the sum of the strips' volume and energy
    (FP64 all-reduce), equal to the single-domain diagnostics up to the
    order of the sums."""
    from oracle import oracle as ora
    vol, en = ora.diag(_basin())
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_diag_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert len({got[r] for r in range(world)}) == 1          # the same on every rank
    v, e = got[0]
    assert abs(v - vol) <= 1e-13 * abs(vol) and abs(e - en) <= 1e-12 * abs(en)
