"""ctypes binding of libinmsom_gpu.so (include/inmsom_gpu.h).

The library is the product: there is no Python or CPU fallback.  Loading
fails loudly if the shared object has not been built.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().with_name("libinmsom_gpu.so")

OK, ECUDA, EARG, EGUARD, ETIMEOUT, EUNSUPPORTED = 0, 1, 2, 3, 4, 5
RESIDENT, FORCE_GENERAL, GUARD, FP32_VELOCITY, STATIC_COEFFS = 0x1, 0x2, 0x4, 0x8, 0x10
SYNC_STATE, SYNC_DEPTHS, SYNC_SCRATCH, SYNC_COEFFS = 0x1, 0x2, 0x4, 0x8

# every exported entry point declared in include/inmsom_gpu.h
EXPORTS = (
    "inmsom_gpu_init", "inmsom_gpu_register_grid", "inmsom_barotropic_dynamics",
    "inmsom_ssh_internal", "inmsom_gridcon", "inmsom_r_diss", "inmsom_wind_forcing",
    "inmsom_hh_init_external", "inmsom_guard", "inmsom_gpu_diag",
    "inmsom_gpu_sync_to_host", "inmsom_gpu_sync_from_host", "inmsom_run_substeps",
    "inmsom_gpu_path", "inmsom_gpu_finalize", "inmsom_gpu_last_error", "inmsom_load_state",
    "inmsom_diag_noalloc", "inmsom_ens_create", "inmsom_ens_run", "inmsom_ens_tune",
    "inmsom_ens_destroy", "inmsom_strips_create", "inmsom_strips_run", "inmsom_strips_destroy",
    "inmsom_mlp_pack", "inmsom_mlp_forward", "inmsom_mlp_grad", "inmsom_mlp_adam", "inmsom_mlp_batch_indices",
    "inmsom_closure_features", "inmsom_run_closure", "inmsom_closure_tendency", "inmsom_gpu_last_phases",
    "inmsom_step_begin", "inmsom_step_launch", "inmsom_halo_pack", "inmsom_halo_unpack", "inmsom_step_end",
    "inmsom_gpu_stream", "inmsom_gpu_pitch", "inmsom_rhs2d", "inmsom_velocity2d",
    "inmsom_baroclinic_dynamics", "inmsom_vertical_velocity", "inmsom_depth_ave", "inmsom_shift_barotropic",
    "inmsom_wdstd8", "inmsom_wdstd", "inmsom_rdstd8", "inmsom_rdstd", "inmsom_ctl_file_write",
    "inmsom_write_checkpoint", "inmsom_read_checkpoint", "inmsom_tracer_tran_diff", "inmsom_ctl_file_read",
    "inmsom_pwdstd", "inmsom_prdstd", "inmsom_ocpwrite", "inmsom_ocpread",
    "inmsom_compare_grids", "inmsom_stress_components", "inmsom_smagorinsky_coeff",
    "inmsom_test_hold_copy", "inmsom_step_launch_rows", "inmsom_gpu_halo", "inmsom_ens_persistent",
)

# include/inmsom_gpu.h: INMSOM_MLP_*
MLP_NPARAM, MLP_NBF16, MLP_PARTIAL = 7816, 7680, 7817

# include/inmsom_gpu.h: INMSOM_DIAG_NOALLOC_MAX_ROWS
DIAG_NOALLOC_MAX_ROWS = 16384


class CCtlAxes(ctypes.Structure):
    """include/inmsom_gpu.h: inmsom_ctl_axes."""
    _fields_ = [("xgr_type", ctypes.c_int), ("ygr_type", ctypes.c_int),
                ("xt", ctypes.POINTER(ctypes.c_double)), ("xu", ctypes.POINTER(ctypes.c_double)),
                ("yt", ctypes.POINTER(ctypes.c_double)), ("yv", ctypes.POINTER(ctypes.c_double)),
                ("dxst", ctypes.c_double), ("dyst", ctypes.c_double),
                ("calendar", ctypes.c_int), ("year", ctypes.c_int), ("month", ctypes.c_int), ("day", ctypes.c_int),
                ("hour", ctypes.c_int), ("minute", ctypes.c_int), ("tstep", ctypes.c_float)]


OCEAN_STATE_FIELDS = ("tt", "ttp", "ss", "ssp", "uu", "uup", "vv", "vvp", "q2", "q2p", "q2l", "q2lp", "ssh_i",
                      "sshp_i", "ssh_e", "sshp_e", "ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e")


class COceanState(ctypes.Structure):
    """include/inmsom_gpu.h: inmsom_ocean_state."""
    _fields_ = [(n, ctypes.POINTER(ctypes.c_double)) for n in OCEAN_STATE_FIELDS]


class InmsomError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class CBounds(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "nx_start", "nx_end", "ny_start", "ny_end", "bnd_x1", "bnd_x2", "bnd_y1", "bnd_y2",
        "mmm", "mm", "nnn", "nn", "periodicity_x", "periodicity_y")]


class CClosureNorm(ctypes.Structure):
    """inmsom_closure_norm"""
    _fields_ = [("mean", ctypes.c_float * 5), ("inv_std", ctypes.c_float * 5),
                ("out_scale", ctypes.c_float * 2)]


class CConsts(ctypes.Structure):
    _fields_ = [("time_smooth", ctypes.c_double), ("free_fall_acc", ctypes.c_double),
                ("ref_den", ctypes.c_double), ("full_free_surface", ctypes.c_int)]


DP = ctypes.POINTER(ctypes.c_double)
FP = ctypes.POINTER(ctypes.c_float)
VP = ctypes.c_void_p

_lib = None


def load() -> ctypes.CDLL:
    """Load the CUDA library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with inmsom_elfs_b200.build.build() "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    i, d, u = ctypes.c_int, ctypes.c_double, ctypes.c_uint
    lib.inmsom_gpu_last_error.restype = ctypes.c_char_p
    lib.inmsom_gpu_init.argtypes = [ctypes.POINTER(VP), ctypes.POINTER(CBounds),
                                    ctypes.POINTER(CConsts), i, u]
    lib.inmsom_gpu_register_grid.argtypes = [VP] + [FP] * 7 + [DP] * 10 + [DP] * 12
    lib.inmsom_barotropic_dynamics.argtypes = [VP, d, i, i] + [DP] * 25
    lib.inmsom_ssh_internal.argtypes = [VP, d] + [DP] * 9
    lib.inmsom_gridcon.argtypes = [ctypes.POINTER(CBounds)] + [FP] * 7 + [i]
    lib.inmsom_r_diss.argtypes = [VP, d, DP]
    lib.inmsom_wind_forcing.argtypes = [VP, DP, DP, DP, DP]
    lib.inmsom_hh_init_external.argtypes = [VP, DP, DP]
    lib.inmsom_guard.argtypes = [VP, ctypes.POINTER(ctypes.c_long)]
    lib.inmsom_gpu_diag.argtypes = [VP, DP, DP]
    lib.inmsom_gpu_sync_to_host.argtypes = [VP, u]
    lib.inmsom_gpu_sync_from_host.argtypes = [VP, u]
    lib.inmsom_run_substeps.argtypes = [VP, i, d, DP, ctypes.POINTER(ctypes.c_float)]
    lib.inmsom_load_state.argtypes = [VP] + [DP] * 12
    lib.inmsom_gpu_path.argtypes = [VP, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_char_p)]
    lib.inmsom_test_hold_copy.argtypes = [VP, i, i, ctypes.c_uint]
    lib.inmsom_gpu_finalize.argtypes = [VP]
    lib.inmsom_ens_create.argtypes = [ctypes.POINTER(VP), ctypes.POINTER(VP), i, i]
    lib.inmsom_ens_run.argtypes = [VP, i, DP, DP, ctypes.POINTER(ctypes.c_float)]
    lib.inmsom_ens_tune.argtypes = [VP, DP, i, ctypes.POINTER(i)]
    lib.inmsom_ens_destroy.argtypes = [VP]
    lib.inmsom_ens_persistent.argtypes = [VP, i]
    lib.inmsom_strips_create.argtypes = [ctypes.POINTER(VP), ctypes.POINTER(VP), i]
    lib.inmsom_strips_run.argtypes = [VP, i, d, DP, ctypes.POINTER(ctypes.c_float)]
    lib.inmsom_strips_destroy.argtypes = [VP]
    F = ctypes.POINTER(ctypes.c_float)
    IP = ctypes.POINTER(ctypes.c_int)
    lib.inmsom_mlp_pack.argtypes = [VP, VP, VP]
    lib.inmsom_mlp_forward.argtypes = [VP, ctypes.c_longlong, VP, VP, VP, VP]
    lib.inmsom_mlp_grad.argtypes = [VP, VP, VP, i, VP, VP, VP, VP, VP]
    lib.inmsom_mlp_adam.argtypes = [VP, VP, VP, VP, VP, i, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, VP]
    lib.inmsom_mlp_batch_indices.argtypes = [VP, i, ctypes.c_longlong, ctypes.c_ulonglong, i, VP]
    NP = ctypes.POINTER(CClosureNorm)
    lib.inmsom_closure_features.argtypes = [VP, NP, VP]
    lib.inmsom_run_closure.argtypes = [VP, i, d, i, VP, VP, NP, ctypes.POINTER(ctypes.c_float)]
    lib.inmsom_closure_tendency.argtypes = [VP, VP, VP, NP, DP, DP]
    FPP = ctypes.POINTER(ctypes.c_float)
    lib.inmsom_gpu_last_phases.argtypes = [VP, FPP, FPP, FPP]
    lib.inmsom_rhs2d.argtypes = [VP] + [DP] * 15
    lib.inmsom_velocity2d.argtypes = [VP] + [DP] * 9
    lib.inmsom_baroclinic_dynamics.argtypes = [VP, i, DP, DP, d] + [DP] * 24
    lib.inmsom_vertical_velocity.argtypes = [VP, i] + [DP] * 7
    lib.inmsom_depth_ave.argtypes = [VP, i, DP, DP, DP, FP, i]
    lib.inmsom_shift_barotropic.argtypes = [VP, i, DP, DP, DP, DP, i]
    lib.inmsom_stress_components.argtypes = [VP, i, DP, DP, DP, DP]
    lib.inmsom_smagorinsky_coeff.argtypes = [VP, i, d, d, DP, DP, DP, DP]
    cp = ctypes.c_char_p
    for nm, ptr in (("inmsom_wdstd8", DP), ("inmsom_wdstd", FP), ("inmsom_rdstd8", DP), ("inmsom_rdstd", FP)):
        getattr(lib, nm).argtypes = [cp, cp, i, ptr, FP] + [i] * 9
    lib.inmsom_ocpwrite.argtypes = [cp, ctypes.POINTER(CBounds), i, FP, FP, FP, DP, DP, ctypes.POINTER(CCtlAxes),
                                    ctypes.POINTER(COceanState)]
    lib.inmsom_ocpread.argtypes = [cp, ctypes.POINTER(CBounds), i, FP, FP, FP, d, ctypes.POINTER(COceanState)]
    grid = [ctypes.c_float, i, i, i, i, DP, d, DP, d, ctypes.c_float, ctypes.c_float, DP, d]
    lib.inmsom_compare_grids.argtypes = [i, ctypes.POINTER(ctypes.c_int)] + grid + grid
    for nm in ("inmsom_pwdstd", "inmsom_prdstd"):
        getattr(lib, nm).argtypes = [ctypes.POINTER(CBounds), cp, cp, i, FP, FP] + [i] * 9
    lib.inmsom_ctl_file_write.argtypes = [cp, ctypes.c_float, i, i, i, i, i, DP, d, i, DP, d, i, DP, d,
                                          i, i, i, i, i, i, ctypes.c_float, cp, cp]
    lib.inmsom_write_checkpoint.argtypes = [VP, cp, ctypes.POINTER(CCtlAxes)]
    IP, FPn = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)
    lib.inmsom_ctl_file_read.argtypes = [cp, cp, i, FPn, IP, IP, IP, IP, IP, DP, i, DP, IP, DP, i, DP, IP, DP, i,
                                         DP, IP, IP, IP, IP, IP, IP, IP, FPn, cp, i, cp, i, i, IP]
    IPP = ctypes.POINTER(ctypes.c_int)
    lib.inmsom_tracer_tran_diff.argtypes = ([VP, i, DP, DP, DP, DP, d, DP, DP, DP, DP, d, DP, d, DP, DP, DP, DP,
                                             d, d, d, DP, DP, IPP, IPP, DP, DP, DP, i, i, IPP, IPP, cp, FP, DP, d]
                                            + [DP] * 4)
    lib.inmsom_read_checkpoint.argtypes = [VP, cp] + [DP] * 6
    lib.inmsom_step_begin.argtypes = [VP]
    lib.inmsom_step_launch.argtypes = [VP, d, d]
    lib.inmsom_step_launch_rows.argtypes = [VP, d, d, i, i]
    lib.inmsom_gpu_halo.argtypes = [VP, ctypes.POINTER(i), ctypes.POINTER(i)]
    lib.inmsom_halo_pack.argtypes = [VP, i, VP]
    lib.inmsom_halo_unpack.argtypes = [VP, i, VP]
    lib.inmsom_step_end.argtypes = [VP]
    lib.inmsom_gpu_stream.argtypes = [VP]
    lib.inmsom_gpu_pitch.argtypes = [VP]
    lib.inmsom_diag_noalloc.argtypes = ([ctypes.POINTER(CBounds), ctypes.POINTER(CConsts),
                                         ctypes.c_longlong] + [VP] * 16 + [VP])
    for name in EXPORTS:
        if name not in ("inmsom_gpu_last_error", "inmsom_gpu_stream", "inmsom_gpu_pitch"):
            getattr(lib, name).restype = i
    lib.inmsom_gpu_stream.restype = VP
    lib.inmsom_gpu_pitch.restype = ctypes.c_longlong
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != OK:
        raise InmsomError(rc, load().inmsom_gpu_last_error().decode(errors="replace"))


def dptr(a):
    """double* of a Fortran-contiguous float64 array (None -> NULL)."""
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags.f_contiguous:
        raise TypeError("expected a Fortran-contiguous float64 array")
    return a.ctypes.data_as(DP)


def fptr(a):
    if a.dtype != np.float32 or not a.flags.f_contiguous:
        raise TypeError("expected a Fortran-contiguous float32 array")
    return a.ctypes.data_as(FP)


def cbounds(b) -> CBounds:
    return CBounds(*b.astuple())


def cconsts(c) -> CConsts:
    return CConsts(c.time_smooth, c.free_fall_acc, c.ref_den, c.full_free_surface)
