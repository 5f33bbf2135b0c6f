"""Row-strip decomposition on the CPU: two gloo ranks, each running the
oracle on its strip with the reference's halo exchange (syncborder_real8:
one row sent north and one south after every field update, for a 1 x 2
process grid), must reproduce the single-domain oracle run bit for bit.
This checks the decomposition (strip_bounds / split_basin / gather_state)
and the exchange pattern the GPU strips reproduce."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _basin():
    from inmsom_elfs_b200 import basins
    from oracle import oracle as ora
    b = basins.regional_basin(nx=70, ny=57, seed=81)
    basins.finalize(b, ora.OracleBackend())
    lu = b.masks["lu"] > 0.5
    m = np.arange(b.bounds.shape[0])[:, None]
    n = np.arange(b.bounds.shape[1])[None, :]
    b.state["ssh_e"] = np.asfortranarray(np.where(lu, 0.2 * np.exp(-((m - 35.0) ** 2 + (n - 30.0) ** 2) / 60.0), 0.0))
    b.state["sshp_e"] = b.state["ssh_e"].copy(order="F")
    ora.hh_init_external(b)
    return b


CALLS, NSTEP = 3, 4


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from oracle import oracle as ora
    from inmsom_elfs_b200.strips import split_basin
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        glob = _basin()
        loc = split_basin(glob, world)[rank]
        lb = loc.bounds
        nxa, nya = lb.bnd_x2 - lb.bnd_x1 + 1, lb.bnd_y2 - lb.bnd_y1 + 1
        c0, c1 = lb.nx_start - lb.bnd_x1, lb.nx_end - lb.bnd_x1 + 1
        row = lambda n: n - lb.bnd_y1

        def exchange(ptr):
            f = np.ctypeslib.as_array(ptr, shape=(nya * nxa,)).reshape(nya, nxa).T
            # Modules/mod_mpi_parallel_tools.f90:187-207: ny+ then ny-
            for send_row, recv_row, to, frm in ((lb.ny_end, lb.bnd_y1 + 1, rank + 1, rank - 1),
                                                (lb.ny_start, lb.bnd_y2 - 1, rank - 1, rank + 1)):
                reqs, buf = [], None
                if 0 <= to < world:
                    reqs.append(dist.isend(torch.from_numpy(f[c0:c1, row(send_row)].copy()), to))
                if 0 <= frm < world:
                    buf = torch.empty(c1 - c0, dtype=torch.float64)
                    reqs.append(dist.irecv(buf, frm))
                for r in reqs:
                    r.wait()
                if buf is not None:
                    f[c0:c1, row(recv_row)] = buf.numpy()

        ora.set_exchange(exchange)
        for _ in range(CALLS):
            ora.barotropic_dynamics(loc, NSTEP * loc.dt, NSTEP)
        ora.set_exchange(None)
        q.put((rank, {k: v for k, v in loc.state.items()}, {k: v for k, v in loc.means.items()}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_strips_reproduce_one_domain():
    from oracle import oracle as ora
    from inmsom_elfs_b200.strips import gather_state, split_basin, strip_bounds
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    glob = _basin()
    strips = split_basin(glob, 2)
    for rank, st, means in got:
        strips[rank].state.update(st)
        strips[rank].means.update(means)
    merged = gather_state(strips, glob, groups=("state", "means"))
    ref = glob.copy()
    for _ in range(CALLS):
        ora.barotropic_dynamics(ref, NSTEP * ref.dt, NSTEP)
    b = glob.bounds
    inner = (slice(None), slice(b.ny_start - b.bnd_y1, b.ny_end - b.bnd_y1 + 1))
    for grp in ("state", "means"):
        for k, v in getattr(ref, grp).items():
            assert np.array_equal(getattr(merged, grp)[k][inner], v[inner]), (grp, k)
    assert len(strip_bounds(b, 2)) == 2


def test_strip_bounds_follow_the_reference_formula():
    from inmsom_elfs_b200.grid import Bounds
    from inmsom_elfs_b200.strips import strip_bounds
    g = Bounds.serial(100, 103)            # rows 1..107, interior 3..105
    s = strip_bounds(g, 4)
    locn = (107 - 4) // 4
    assert [x.ny_start for x in s] == [3 + locn * k for k in range(4)]
    assert s[-1].ny_end == 105 and all(x.bnd_y1 == x.ny_start - 2 and x.bnd_y2 == x.ny_end + 2 for x in s)
    assert all(s[k].ny_end + 1 == s[k + 1].ny_start for k in range(3))
    assert all(x.nx_start == g.nx_start and x.nx_end == g.nx_end for x in s)
    with pytest.raises(ValueError):
        strip_bounds(Bounds.serial(10, 3), 4)


def test_stacked_strip_equals_split_of_the_stack(ora):
    from inmsom_elfs_b200 import basins
    """strips.stacked_strip (the multi-GPU benchmark's strips: N basins
    stacked along y, each finalized on its own) gives exactly what
    split_basin gives on the explicitly stacked global basin, for the
    reference's 2-row halos and for wide ones."""
    from dataclasses import replace
    from inmsom_elfs_b200.grid import Basin
    from inmsom_elfs_b200.strips import split_basin, stacked_strip
    n, ny = 3, 30
    parts = {q: basins.finalize(basins.regional_basin(nx=40, ny=ny, seed=5 + q), ora.OracleBackend())
             for q in range(n)}
    for q, p in parts.items():
        p.state["ssh_e"][...] = np.random.default_rng(q).standard_normal(p.bounds.shape)
    own = parts[0]
    b = own.bounds
    glob = replace(b, ny_end=b.ny_start + n * ny - 1, bnd_y2=b.ny_start + n * ny + 1, nn=b.nnn + n * ny - 1)

    def stack(get):
        cols = [get(parts[0])[:, :2]] + [get(parts[q])[:, 2:-2] for q in range(n)] + [get(parts[n - 1])[:, -2:]]
        return np.asfortranarray(np.concatenate(cols, axis=1))

    def grp(name):
        return {k: stack(lambda p, k=k: getattr(p, name)[k]) for k in getattr(own, name)}

    g = Basin(glob, own.consts, grp("masks"), grp("metrics"), stack(lambda p: p.rlh_s),
              stack(lambda p: p.hhq_rest), grp("depths"), grp("state"), grp("means"), grp("forcing"),
              grp("scratch"), None, None, own.dt)
    for halo in (2, 6):
        sp = split_basin(g, n, halo)
        for r in range(n):
            loc = stacked_strip({q: parts[q] for q in (r - 1, r, r + 1) if 0 <= q < n}, n, r, halo)
            assert loc.bounds == sp[r].bounds
            for name in ("masks", "metrics", "state", "forcing", "depths"):
                for k, v in getattr(loc, name).items():
                    assert np.array_equal(v, getattr(sp[r], name)[k]), (name, k, r)
            assert np.array_equal(loc.hhq_rest, sp[r].hhq_rest) and np.array_equal(loc.rlh_s, sp[r].rlh_s)
