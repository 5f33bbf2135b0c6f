"""inmsom_diag_noalloc: the volume/energy diagnostic for callers that cannot
allocate GPU memory, with its scratch in a fixed array of the library.

Collected last on purpose: the GPU test must also pass after every other
test has used the library on the same device.  It calls the entry point
through the C ABI on caller-owned device arrays, twice in a row on two
different basins (the second with fewer rows, so stale partials of the first
call would show) and once more on the first basin with a padded row pitch,
and compares each result with inmsom_gpu_diag of a context holding the same
state, within the diagnostic's tolerance; the device's free memory is the
same before and after each call but the first.
"""
import ctypes

import numpy as np
import pytest

from inmsom_elfs_b200 import basins
from inmsom_elfs_b200.grid import Bounds, Consts

TOL = 1e-12   # relative tolerance of the volume/energy diagnostic tests


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _call(lib, bounds, consts, ld, fields, out, stream):
    from inmsom_elfs_b200 import _lib
    names = ("lu", "lcu", "lcv", "dx", "dy", "dxt", "dyt", "dxh", "dyh", "hhq_rest",
             "ssh", "u", "v", "hu", "hv")
    return lib.inmsom_diag_noalloc(ctypes.byref(_lib.cbounds(bounds)),
                                   ctypes.byref(_lib.cconsts(consts)), ld,
                                   *[_ptr(fields[k]) for k in names], _ptr(out),
                                   ctypes.c_void_p(stream))


def _to_device(torch, a, ld):
    """Host Fortran array f(bnd_x1:bnd_x2, bnd_y1:bnd_y2) -> device rows of
    ld elements (x fastest), padding zero."""
    nxa, nya = a.shape
    dt = torch.float32 if a.dtype == np.float32 else torch.float64
    t = torch.zeros((nya, ld), dtype=dt, device="cuda:0")
    t[:, :nxa] = torch.from_numpy(np.ascontiguousarray(a.T)).to("cuda:0")
    return t


def _evolved(gpu, basin, calls):
    """Run a resident context for `calls` barotropic_dynamics calls; return
    (volume, energy) from inmsom_gpu_diag and the host basin holding the
    same state and u/v depths."""
    basins.finalize(basin, gpu.GpuBackend(0))
    with gpu.BarotropicSolver(basin, resident=True) as s:
        s.hh_init_external()
        for _ in range(calls):
            s.barotropic_dynamics(5 * basin.dt, 5)
        vol, en = s.diag()
        s.sync_to_host(0x1 | 0x2)
    return (vol, en), basin


def _fields(torch, basin, ld):
    m, g, st, d = basin.masks, basin.metrics, basin.state, basin.depths
    host = {"lu": m["lu"], "lcu": m["lcu"], "lcv": m["lcv"],
            **{k: g[k] for k in ("dx", "dy", "dxt", "dyt", "dxh", "dyh")},
            "hhq_rest": basin.hhq_rest, "ssh": st["ssh_e"], "u": st["ubrtr_e"],
            "v": st["vbrtr_e"], "hu": d["hhu_e"], "hv": d["hhv_e"]}
    return {k: _to_device(torch, a, ld) for k, a in host.items()}


@pytest.mark.gpu
def test_noalloc_diag_matches_context_diag(gpu):
    import torch
    from inmsom_elfs_b200 import _lib
    lib = _lib.load()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream(0)

    want_a, a = _evolved(gpu, basins.beta_plane_basin(n=120, seed=31), 4)
    want_b, b = _evolved(gpu, basins.regional_basin(nx=150, ny=61, seed=32), 4)
    assert b.bounds.ny < a.bounds.ny
    nxa_a = a.bounds.bnd_x2 - a.bounds.bnd_x1 + 1
    nxa_b = b.bounds.bnd_x2 - b.bounds.bnd_x1 + 1

    calls = ((a, nxa_a, want_a), (b, nxa_b, want_b), (a, nxa_a + 37, want_a))
    for i, (basin, ld, (vol, en)) in enumerate(calls):
        fields = _fields(torch, basin, ld)
        out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(0)[0]
        rc = _call(lib, basin.bounds, basin.consts, ld, fields, out, stream.cuda_stream)
        assert rc == 0, lib.inmsom_gpu_last_error().decode()
        got = out.cpu().numpy()          # waits for the stream
        if i > 0:
            # after the first call (which may load the device code and the
            # array), a call takes no device memory at all
            assert torch.cuda.mem_get_info(0)[0] == free0
        assert abs(got[0] - vol) <= TOL * abs(vol), (got[0], vol)
        assert abs(got[1] - en) <= TOL * abs(en), (got[1], en)
        assert en > 0.0


@pytest.mark.gpu
def test_noalloc_diag_rejects_too_many_rows_on_gpu(gpu):
    import torch
    from inmsom_elfs_b200 import _lib
    lib = _lib.load()
    torch.cuda.set_device(0)
    b = Bounds.serial(8, _lib.DIAG_NOALLOC_MAX_ROWS + 1)
    one = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    rc = lib.inmsom_diag_noalloc(ctypes.byref(_lib.cbounds(b)), ctypes.byref(_lib.cconsts(Consts())),
                                 12, *[_ptr(one)] * 16, None)
    assert rc == _lib.EARG
    assert b"INMSOM_DIAG_NOALLOC_MAX_ROWS" in lib.inmsom_gpu_last_error()


def test_noalloc_diag_argument_checks_without_gpu():
    """Host-side checks return before the first CUDA call (no GPU needed)."""
    from inmsom_elfs_b200 import _lib
    lib = _lib.load()
    fake = ctypes.c_void_p(0x1000)      # never dereferenced: every call below is rejected
    k = ctypes.byref(_lib.cconsts(Consts()))
    big = Bounds.serial(8, _lib.DIAG_NOALLOC_MAX_ROWS + 1)
    rc = lib.inmsom_diag_noalloc(ctypes.byref(_lib.cbounds(big)), k, 12, *[fake] * 16, None)
    assert rc == _lib.EARG
    assert b"exceed INMSOM_DIAG_NOALLOC_MAX_ROWS" in lib.inmsom_gpu_last_error()
    ok = Bounds.serial(8, _lib.DIAG_NOALLOC_MAX_ROWS)
    assert lib.inmsom_diag_noalloc(ctypes.byref(_lib.cbounds(ok)), k, 11, *[fake] * 16,
                                   None) == _lib.EARG     # ld below the row length (12)
    assert lib.inmsom_diag_noalloc(ctypes.byref(_lib.cbounds(ok)), k, 12, *[fake] * 15, None,
                                   None) == _lib.EARG     # NULL output
    assert lib.inmsom_diag_noalloc(None, k, 12, *[fake] * 16, None) == _lib.EARG
