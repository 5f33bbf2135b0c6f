"""Row strips with one process (rank) per GPU.

The reference runs its barotropic step on a 2-D MPI process grid and
exchanges one halo row or column per field update with syncborder_real8
(Modules/mod_mpi_parallel_tools.f90:179-252).  Here a 1 x P grid of row
strips (strips.strip_bounds, the reference's decomposition) runs one strip
per rank, each in its own context on its own GPU, and the ranks exchange
ONE pair of halo messages per substep: after a substep, the two
northernmost interior rows of the six state fields go to the northern
neighbour's southern halo rows and the two southernmost to the southern
neighbour's northern halo rows.  The fused kernel recomputes the
intermediates it needs in its halo rows, so this gives the single-domain
result bit for bit.  With halos of 2k rows between the strips (the GPU
form of the reference's wide-halo exchange mode) a rank advances k
substeps per exchange of 2k rows, computing 2(k-i) rows into each shared
halo in substep i of a block, as its neighbour does from the same values:
the same result with k times fewer exchanges.

Transport: torch.distributed point-to-point (batch_isend_irecv).  With NCCL
the device buffers go directly, ordered on the context's CUDA stream; with
gloo they are staged through host memory (tests, and a GPU without peers).
Every rank takes the same collective steps in the same order.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, load


class GpuStripStepper:
    """The per-rank side of the C ABI (inmsom_step_*, inmsom_halo_*) on a
    resident BarotropicSolver whose basin is this rank's strip."""

    def __init__(self, solver, host_staging: bool):
        import torch
        self.torch = torch
        self.solver = solver
        ctx = solver._ctx
        lib = load()
        hs, hn = ctypes.c_int(), ctypes.c_int()
        check(lib.inmsom_gpu_halo(ctx, ctypes.byref(hs), ctypes.byref(hn)))
        self.halo = (hs.value, hn.value)
        pitch = int(lib.inmsom_gpu_pitch(ctx))
        sizes = [6 * w * pitch for w in (hs.value, hn.value)] * 2   # send s/n, receive s/n
        dev = torch.device("cuda", solver.device)
        self.dev = [torch.empty(n, dtype=torch.float64, device=dev) for n in sizes]
        self.stream = torch.cuda.ExternalStream(lib.inmsom_gpu_stream(ctx), device=dev)
        self.host = host_staging
        if host_staging:
            self.cpu = [torch.empty(n, dtype=torch.float64).pin_memory() for n in sizes]

    # buffers: 0 send south, 1 send north, 2 receive south, 3 receive north
    def buffer(self, k: int):
        return self.cpu[k] if self.host else self.dev[k]

    def begin(self) -> None:
        check(load().inmsom_step_begin(self.solver._ctx))

    def launch(self, dt: float, rs: float, rows_south: int = 0, rows_north: int = 0) -> None:
        check(load().inmsom_step_launch_rows(self.solver._ctx, float(dt), float(rs), int(rows_south),
                                             int(rows_north)))

    def pack(self, side: int) -> None:
        check(load().inmsom_halo_pack(self.solver._ctx, side, ctypes.c_void_p(self.dev[side].data_ptr())))
        if self.host:
            with self.torch.cuda.stream(self.stream):
                self.cpu[side].copy_(self.dev[side])     # waits for the pack

    def unpack(self, side: int) -> None:
        k = 2 + side
        if self.host:
            with self.torch.cuda.stream(self.stream):
                self.dev[k].copy_(self.cpu[k])
        check(load().inmsom_halo_unpack(self.solver._ctx, side, ctypes.c_void_p(self.dev[k].data_ptr())))

    def sync(self) -> None:
        """Make the packed device buffers visible to the transport's stream
        (NCCL): the caller's current stream waits for the context's."""
        if not self.host:
            self.torch.cuda.current_stream(self.dev[0].device).wait_stream(self.stream)

    def after_receive(self) -> None:
        if not self.host:
            self.stream.wait_stream(self.torch.cuda.current_stream(self.dev[0].device))

    def end(self) -> None:
        check(load().inmsom_step_end(self.solver._ctx))


def exchange(stepper, rank: int, world: int, group=None) -> None:
    """One halo exchange with the neighbouring ranks (after a substep)."""
    import torch.distributed as dist
    ops = []
    if rank > 0:
        stepper.pack(0)
    if rank + 1 < world:
        stepper.pack(1)
    stepper.sync()
    if rank + 1 < world:
        ops.append(dist.P2POp(dist.isend, stepper.buffer(1), rank + 1, group))
        ops.append(dist.P2POp(dist.irecv, stepper.buffer(3), rank + 1, group))
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, stepper.buffer(0), rank - 1, group))
        ops.append(dist.P2POp(dist.irecv, stepper.buffer(2), rank - 1, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    stepper.after_receive()
    if rank > 0:
        stepper.unpack(0)
    if rank + 1 < world:
        stepper.unpack(1)


def substeps_per_exchange(stepper, rank: int, world: int) -> int:
    """k of a strip whose halos shared with other strips are 2k rows (every
    rank computes the same k from the common halo width)."""
    hs, hn = stepper.halo
    shared = ([hs] if rank > 0 else []) + ([hn] if rank + 1 < world else [])
    if not shared:
        return 1
    if len(set(shared)) != 1 or shared[0] < 2 or shared[0] % 2:
        raise ValueError(f"rank {rank}: shared halos {shared} must be one even width >= 2")
    return shared[0] // 2


def run_strip(stepper, rank: int, world: int, nsub: int, dt: float,
              rhs_scale: Optional[Sequence[float]] = None, group=None) -> None:
    """nsub substeps of this rank's strip: blocks of k substeps (k from the
    halo width, 1 with the reference's two rows), the i-th computing 2(k-i)
    rows into each shared halo, and one halo exchange after each block."""
    k = substeps_per_exchange(stepper, rank, world)
    stepper.begin()
    step = 0
    while step < nsub:
        n = min(k, nsub - step)
        for i in range(1, n + 1):
            e = 2 * (n - i)
            stepper.launch(dt, 1.0 if rhs_scale is None else float(rhs_scale[step]),
                           e if rank > 0 else 0, e if rank + 1 < world else 0)
            step += 1
        exchange(stepper, rank, world, group)
    stepper.end()


class NumpyStripStepper:
    """A stand-in with the same interface for testing the exchange on CPU:
    six fields on the strip's rows (halo rows each side), a radius-2
    row/column stencil that, like the fused kernel, needs only the state's
    halo rows.  Rows outside the global interior are never written."""

    def __init__(self, fields: np.ndarray, local_rows: tuple):
        self.f = fields.copy()                       # [6, nx, rows]
        self.l0, self.l1 = local_rows                # first/last interior rows of this strip (local index)
        self.halo = (self.l0, self.f.shape[2] - 1 - self.l1)
        w = self.halo * 2
        self.buf = [np.zeros((6, self.f.shape[1], w[k])) for k in range(4)]

    def buffer(self, k):
        import torch
        return torch.from_numpy(self.buf[k])

    def begin(self):
        pass

    def launch(self, dt, rs, rows_south=0, rows_north=0):
        f = self.f
        new = f.copy()
        for j in range(self.l0 - rows_south, self.l1 + rows_north + 1):
            for q in range(6):
                a = f[q, 2:-2, j]
                new[q, 2:-2, j] = (0.4 * a + 0.15 * (f[q, 2:-2, j - 1] + f[q, 2:-2, j + 1])
                                   + 0.05 * (f[q, 2:-2, j - 2] + f[q, 2:-2, j + 2])
                                   + 0.1 * (f[q, 1:-3, j] + f[q, 3:-1, j])
                                   + 0.01 * rs * f[(q + 1) % 6, 2:-2, j] * dt)
        self.f = new

    def pack(self, side):
        w = self.halo[side]
        r = self.l0 if side == 0 else self.l1 - w + 1
        self.buf[side][...] = self.f[:, :, r:r + w]

    def sync(self):
        pass

    def after_receive(self):
        pass

    def unpack(self, side):
        w = self.halo[side]
        r = self.l0 - w if side == 0 else self.l1 + 1
        self.f[:, :, r:r + w] = self.buf[2 + side]

    def end(self):
        pass


def diag(solver, group=None, device_tensor: bool = False):
    """Volume and energy of the whole basin: each rank's inmsom_gpu_diag
    over its strip's interior rows, summed over the ranks by an FP64
    all-reduce (two scalars; NCCL with device_tensor, else on the host)."""
    import torch
    import torch.distributed as dist
    v, e = solver.diag()
    t = torch.tensor([v, e], dtype=torch.float64)
    if device_tensor:
        t = t.to(torch.device("cuda", solver.device))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t[0].item()), float(t[1].item())
