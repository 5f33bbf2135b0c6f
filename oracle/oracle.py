"""ctypes front end of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
use this module, always as the checker or the timed CPU reference, never as
the product path.  Functions take the same Basin objects and argument
orders as inmsom_elfs_b200.solver, so a test can run the same call on both.
Parity with the Fortran reference itself is unpinned (see oracle.h).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

DP = ctypes.POINTER(ctypes.c_double)
FP = ctypes.POINTER(ctypes.c_float)

MASKS = ("lu", "luu", "luh", "lcu", "lcv", "llu", "llv")
METRICS = ("dx", "dy", "dxt", "dyt", "dxh", "dyh", "dxb", "dyb")
DEPTHS = ("hhq_e", "hhqp_e", "hhqn_e", "hhu_e", "hhup_e", "hhun_e",
          "hhv_e", "hhvp_e", "hhvn_e", "hhh_e", "hhhp_e", "hhhn_e")
DYN_ARGS = ("ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e", "ssh_e", "sshp_e",
            "ubrtr_i", "vbrtr_i", "ssh4gradx", "ssh4grady", "RHSx", "RHSy", "wflux",
            "mu", "mu4", "vort", "str_t2d", "str_s2d", "fx", "fy", "rdis",
            "RHSx_adv", "RHSy_adv", "RHSx_dif", "RHSy_dif")


class OraBounds(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "nx_start", "nx_end", "ny_start", "ny_end", "bnd_x1", "bnd_x2", "bnd_y1", "bnd_y2",
        "mmm", "mm", "nnn", "nn", "periodicity_x", "periodicity_y")]


class OraGrid(ctypes.Structure):
    _fields_ = ([("b", OraBounds), ("time_smooth", ctypes.c_double),
                 ("free_fall_acc", ctypes.c_double), ("ref_den", ctypes.c_double),
                 ("full_free_surface", ctypes.c_int)]
                + [(k, FP) for k in MASKS] + [(k, DP) for k in METRICS]
                + [("rlh_s", DP), ("hhq_rest", DP)] + [(k, DP) for k in DEPTHS])


_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is None:
        src = Path(__file__).with_name("oracle.c")
        if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.ora_guard.restype = ctypes.c_long
    return _lib


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.f_contiguous
    return a.ctypes.data_as(DP)


def _f(a):
    assert a.dtype == np.float32 and a.flags.f_contiguous
    return a.ctypes.data_as(FP)


def bounds_struct(b) -> OraBounds:
    return OraBounds(*b.astuple())


def grid_struct(basin) -> OraGrid:
    """ora_grid pointing at the basin's arrays (keep the basin alive)."""
    c = basin.consts
    g = OraGrid()
    g.b = bounds_struct(basin.bounds)
    g.time_smooth, g.free_fall_acc, g.ref_den = c.time_smooth, c.free_fall_acc, c.ref_den
    g.full_free_surface = c.full_free_surface
    for k in MASKS:
        setattr(g, k, _f(basin.masks[k]))
    for k in METRICS:
        setattr(g, k, _d(basin.metrics[k]))
    g.rlh_s, g.hhq_rest = _d(basin.rlh_s), _d(basin.hhq_rest)
    for k in DEPTHS:
        setattr(g, k, _d(basin.depths[k]))
    return g


def set_threads(n: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(n)


# ---------------------------------------------------------------------------
def gridcon(bounds, lu):
    out = {k: bounds.zeros(np.float32) for k in ("luu", "luh", "llu", "llv", "lcu", "lcv")}
    b = bounds_struct(bounds)
    load().ora_gridcon(ctypes.byref(b), _f(lu), _f(out["luu"]), _f(out["luh"]), _f(out["llu"]),
                       _f(out["llv"]), _f(out["lcu"]), _f(out["lcv"]))
    return out


def cyclize8_x(bounds, f):
    b = bounds_struct(bounds)
    load().ora_cyclize8_x(ctypes.byref(b), _d(f))


def cyclize8_y(bounds, f):
    b = bounds_struct(bounds)
    load().ora_cyclize8_y(ctypes.byref(b), _d(f))


def wind_forcing(basin, taux=None, tauy=None):
    """surface stress (Function/fluxes.f90:29-37) then the barotropic RHS
    (Control/dyncall.f90:110-130) with all 3-D terms zero."""
    b = basin.bounds
    taux = basin.taux if taux is None else taux
    tauy = basin.tauy if tauy is None else tauy
    g = grid_struct(basin)
    ssx, ssy, rx, ry = b.zeros(), b.zeros(), b.zeros(), b.zeros()
    hhu, hhv = b.zeros(), b.zeros()
    lib = load()
    lib.ora_surface_stress(ctypes.byref(g), _d(taux), _d(tauy), _d(ssx), _d(ssy))
    lib.ora_rhs2d(ctypes.byref(g), _d(rx), _d(ry), None, None, None, None, None, None,
                  _d(ssx), _d(ssy), None, None, None, _d(hhu), _d(hhv))
    return rx, ry


def rhs2d(basin, rhsx, rhsy, diff_disp=(None, None), tran=(None, None), tran_disp=(None, None),
          surf_stress=(None, None), bot_stress=(None, None), slpr=None, hhu=None, hhv=None):
    """Control/dyncall.f90:110-130 on (rhsx, rhsy) in place (ora_rhs2d)."""
    b = basin.bounds
    g = grid_struct(basin)
    hhu = b.zeros() if hhu is None else hhu
    hhv = b.zeros() if hhv is None else hhv
    load().ora_rhs2d(ctypes.byref(g), _d(rhsx), _d(rhsy), _d(diff_disp[0]), _d(diff_disp[1]), _d(tran[0]),
                     _d(tran[1]), _d(tran_disp[0]), _d(tran_disp[1]), _d(surf_stress[0]), _d(surf_stress[1]),
                     _d(bot_stress[0]), _d(bot_stress[1]), _d(slpr), _d(hhu), _d(hhv))
    return rhsx, rhsy


def velocity2d(basin, uu2d, vv2d, pgrx, pgry, ubrtr_i, vbrtr_i, slpr, hhu, hhv):
    """Control/dyncall.f90:188-201 in place on uu2d, vv2d, pgrx, pgry."""
    g = grid_struct(basin)
    load().ora_velocity2d(ctypes.byref(g), _d(uu2d), _d(vv2d), _d(pgrx), _d(pgry), _d(ubrtr_i), _d(vbrtr_i),
                          _d(slpr), _d(hhu), _d(hhv))
    return uu2d, vv2d, pgrx, pgry


BAROCLINIC_FIELDS = ("ww", "nu", "rhsx", "rhsy", "rhsx_tran", "rhsy_tran", "pgrx", "pgry", "rdis",
                     "tx_surf", "ty_surf", "tx_bot", "ty_bot", "hhu", "hhup", "hhun", "hhv", "hhvp", "hhvn",
                     "hhh")


def baroclinic_dynamics(basin, dz, hzt, tau, uu, uup, vv, vvp, **f):
    """Function/vel_ssh.f90:794-1027 in place on uu, uup, vv, vvp: arrays of
    shape (bnd_x, bnd_y, nz) in Fortran order, ww and nu with nz + 1 levels,
    the rest 2-D; f holds the BAROCLINIC_FIELDS by name."""
    g = grid_struct(basin)
    dz = np.ascontiguousarray(dz, dtype=np.float64)
    hzt = np.ascontiguousarray(hzt, dtype=np.float64)
    load().ora_baroclinic_dynamics(ctypes.byref(g), int(len(dz)), dz.ctypes.data_as(DP), hzt.ctypes.data_as(DP),
                                   ctypes.c_double(tau), _d(uu), _d(uup), _d(vv), _d(vvp),
                                   *[_d(f[k]) for k in BAROCLINIC_FIELDS])
    return uu, uup, vv, vvp


def vertical_velocity(basin, dz, u, v, w, hu, hv, wflux):
    """Function/vel_ssh.f90:1030-1076: w (nz + 1 levels) in place."""
    g = grid_struct(basin)
    dz = np.ascontiguousarray(dz, dtype=np.float64)
    load().ora_vertical_velocity(ctypes.byref(g), int(len(dz)), dz.ctypes.data_as(DP), _d(u), _d(v), _d(w),
                                 _d(hu), _d(hv), _d(wflux))
    return w


TRACER_3D = ("uu", "vv", "ww", "mu", "nu", "slrx", "slry", "slzx", "slzy", "src")


def tracer_tran_diff(basin, dz, hzt, tau, ff, ffp, flux_f_x, flux_f_y, f):
    """Function/tem_sal.f90:1-422 in place on ff, ffp (nz levels) and the
    flux diagnostics flux_f_x, flux_f_y (bnd_x, bnd_y, 4); f holds the other
    arguments by name (see ora_tracer_tran_diff)."""
    g = grid_struct(basin)
    dz = np.ascontiguousarray(dz, dtype=np.float64)
    hzt = np.ascontiguousarray(hzt, dtype=np.float64)
    ip = ctypes.POINTER(ctypes.c_int)
    igt = np.asfortranarray(f["ig_top"], dtype=np.int32)
    igb = np.asfortranarray(f["ig_bot"], dtype=np.int32)
    c = ctypes.c_double
    load().ora_tracer_tran_diff(
        ctypes.byref(g), int(len(dz)), dz.ctypes.data_as(DP), hzt.ctypes.data_as(DP), _d(ff), _d(ffp), c(tau),
        _d(f["uu"]), _d(f["vv"]), _d(f["ww"]), _d(f["mu"]), c(f["factor_mu"]), _d(f["nu"]), c(f["factor_nu"]),
        _d(f["slrx"]), _d(f["slry"]), _d(f["slzx"]), _d(f["slzy"]), c(f["az"]), c(f["ar"]), c(f["alpha_gm"]),
        _d(f["ff_top"]), _d(f["ff_bot"]), igt.ctypes.data_as(ip), igb.ctypes.data_as(ip), _d(flux_f_x),
        _d(flux_f_y), _d(f["swbal"]), _d(f["src"]), c(f["src_factor"]), _d(f["hhu"]), _d(f["hhv"]), _d(f["hhqn"]),
        _d(f["hhqp"]))
    return ff, ffp, flux_f_x, flux_f_y


def depth_ave(basin, dz, u, utr, mask, kbcl):
    """Function/depth.f90:223-254 in place on u (nz levels) and utr."""
    g = grid_struct(basin)
    dz = np.ascontiguousarray(dz, dtype=np.float64)
    load().ora_depth_ave(ctypes.byref(g), int(len(dz)), dz.ctypes.data_as(DP), _d(u), _d(utr), _f(mask), int(kbcl))
    return u, utr


def _levels(a):
    return [a] if a.ndim == 2 else [a[:, :, k] for k in range(a.shape[2])]


def stress_components(basin, u, v, str_t, str_s):
    """Function/mixing.f90:115-168 on every level of u, v (the routine's
    level loop is innermost and the levels do not interact), in place."""
    g = grid_struct(basin)
    for uk, vk, tk, sk in zip(*[_levels(a) for a in (u, v, str_t, str_s)]):
        load().ora_stress_components(ctypes.byref(g), _d(uk), _d(vk), _d(tk), _d(sk))
    return str_t, str_s


def smagorinsky_coeff(basin, visc2, dift, str_t, str_s, amts, amuv, vonkarman=0.4, pi=3.141592653589793):
    """Function/mixing.f90:171-219 on every level, in place on amts, amuv
    (vonkarman, Pi: Inc/basinpar.fi:72,89)."""
    g = grid_struct(basin)
    for tk, sk, ak, mk in zip(*[_levels(a) for a in (str_t, str_s, amts, amuv)]):
        load().ora_smagorinsky_coeff(ctypes.byref(g), ctypes.c_double(visc2), ctypes.c_double(dift), _d(tk),
                                     _d(sk), _d(ak), _d(mk), ctypes.c_double(vonkarman), ctypes.c_double(pi))
    return amts, amuv


def shift_barotropic(basin, nz, uu, vv, uu2d, vv2d, sign):
    """Control/dyncall.f90:170-183 (sign -1) / :215-229 (sign +1) in place."""
    g = grid_struct(basin)
    load().ora_shift_barotropic(ctypes.byref(g), int(nz), _d(uu), _d(vv), _d(uu2d), _d(vv2d), int(sign))
    return uu, vv


def hh_init_external(basin):
    g = grid_struct(basin)
    d = basin.depths
    load().ora_hh_init(ctypes.byref(g), *[_d(d[k]) for k in DEPTHS], _d(basin.state["ssh_e"]),
                       _d(basin.state["sshp_e"]), _d(basin.hhq_rest))


def barotropic_dynamics(basin, tau, nstep, ksw4=0, **override):
    g = grid_struct(basin)
    pools = (basin.state, basin.means, basin.forcing, basin.scratch)
    arrs = []
    for k in DYN_ARGS:
        if k in override:
            arrs.append(override[k])
        else:
            arrs.append(next(p[k] for p in pools if k in p))
    load().ora_barotropic_dynamics(ctypes.byref(g), ctypes.c_double(tau), int(nstep), int(ksw4),
                                   *[_d(a) for a in arrs])


def ssh_internal(basin, tau, ssh_i, sshp_i, u, v, wflux, hhqn, hhun, hhvn, hhhn):
    g = grid_struct(basin)
    load().ora_ssh_internal(ctypes.byref(g), ctypes.c_double(tau), _d(ssh_i), _d(sshp_i), _d(u),
                            _d(v), _d(wflux), _d(hhqn), _d(hhun), _d(hhvn), _d(hhhn))


def r_diss(basin, r_fric, out=None):
    out = basin.bounds.zeros() if out is None else out
    g = grid_struct(basin)
    load().ora_r_diss(ctypes.byref(g), ctypes.c_double(r_fric), _d(out))
    return out


def guard(basin, ssh=None, u=None, v=None):
    s = basin.state
    g = grid_struct(basin)
    return int(load().ora_guard(ctypes.byref(g), _d(s["ssh_e"] if ssh is None else ssh),
                                _d(s["ubrtr_e"] if u is None else u),
                                _d(s["vbrtr_e"] if v is None else v)))


def diag(basin):
    """volume/energy of the state, with hu/hv from hh_init of that state."""
    tmp = basin.copy()
    hh_init_external(tmp)
    g = grid_struct(tmp)
    vol, en = ctypes.c_double(), ctypes.c_double()
    s = tmp.state
    load().ora_diag(ctypes.byref(g), _d(s["ssh_e"]), _d(s["ubrtr_e"]), _d(s["vbrtr_e"]),
                    _d(tmp.depths["hhu_e"]), _d(tmp.depths["hhv_e"]), ctypes.byref(vol),
                    ctypes.byref(en))
    return vol.value, en.value


def run_substeps(basin, nsub, dt, rhs_scale=None):
    """The standalone integration: nsub calls of barotropic_dynamics(dt, 1),
    keeping the saved *_e state; RHS multiplied by rhs_scale[k] in call k."""
    rx0, ry0 = basin.forcing["RHSx"], basin.forcing["RHSy"]
    for k in range(nsub):
        if rhs_scale is None:
            barotropic_dynamics(basin, dt, 1, 0)
        else:
            s = float(rhs_scale[k])
            barotropic_dynamics(basin, dt, 1, 0, RHSx=np.asfortranarray(rx0 * s),
                                RHSy=np.asfortranarray(ry0 * s))


class OracleBackend:
    """Basin set-up on the CPU oracle (tests only)."""

    def gridcon(self, bounds, lu):
        return gridcon(bounds, lu)

    def wind_forcing(self, basin):
        return wind_forcing(basin)


EXCHANGE_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)
_exchange_keep = None


def set_exchange(fn):
    """Install fn(field) at every syncborder_real8 point of the oracle
    (Modules/mod_mpi_parallel_tools.f90:179-252), field being a ctypes
    pointer to the local array; None removes it.  For rank tests."""
    global _exchange_keep
    lib = load()
    lib.ora_set_exchange.argtypes = [EXCHANGE_FN, ctypes.c_void_p]
    if fn is None:
        lib.ora_set_exchange(EXCHANGE_FN(), None)
        _exchange_keep = None
        return
    cb = EXCHANGE_FN(lambda ptr, user: fn(ptr))
    _exchange_keep = cb
    lib.ora_set_exchange(cb, None)
