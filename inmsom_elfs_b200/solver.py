"""Host-side mirror of the reference's barotropic interface over the C ABI.

``BarotropicSolver`` owns one library context for one basin.  Its methods
take the reference's arguments in the reference's order
(Function/vel_ssh.f90:379-406 and :682-687) as Fortran-layout numpy arrays,
or default to the arrays held by the Basin.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import InmsomError, cbounds, cconsts, check, dptr, fptr, load
from .grid import DEPTHS, MASKS, MEANS, METRICS, SCRATCH, STATE, Basin, Bounds

# argument order of barotropic_dynamics after (tau, nstep, ksw4)
DYN_ARGS = ("ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e", "ssh_e", "sshp_e",
            "ubrtr_i", "vbrtr_i", "ssh4gradx", "ssh4grady", "RHSx", "RHSy", "wflux",
            "mu", "mu4", "vort", "str_t2d", "str_s2d", "fx", "fy", "rdis",
            "RHSx_adv", "RHSy_adv", "RHSx_dif", "RHSy_dif")


def gridcon(bounds: Bounds, lu: np.ndarray, device: int = 0) -> dict:
    """Derived masks of Service/grid_construction.f90:59-112, on the GPU."""
    lib = load()
    out = {k: bounds.zeros(np.float32) for k in ("luu", "luh", "llu", "llv", "lcu", "lcv")}
    cb = cbounds(bounds)
    check(lib.inmsom_gridcon(ctypes.byref(cb), fptr(lu), fptr(out["luu"]), fptr(out["luh"]),
                             fptr(out["llu"]), fptr(out["llv"]), fptr(out["lcu"]),
                             fptr(out["lcv"]), device))
    return out


class BarotropicSolver:
    def __init__(self, basin: Basin, device: int = 0, resident: bool = True,
                 force_general: bool = False, guard: bool = False,
                 register_depths: bool = True, fp32_velocity: bool = False,
                 static_coeffs: bool = False):
        lib = load()
        self.basin = basin
        self.device = device
        flags = (_lib.RESIDENT if resident else 0) | (_lib.FORCE_GENERAL if force_general else 0) \
            | (_lib.GUARD if guard else 0) | (_lib.FP32_VELOCITY if fp32_velocity else 0) \
            | (_lib.STATIC_COEFFS if static_coeffs else 0)
        self._ctx = ctypes.c_void_p()
        cb, cc = cbounds(basin.bounds), cconsts(basin.consts)
        check(lib.inmsom_gpu_init(ctypes.byref(self._ctx), ctypes.byref(cb), ctypes.byref(cc),
                                  device, flags))
        m, g = basin.masks, basin.metrics
        depths = [dptr(basin.depths[k]) if register_depths else None for k in DEPTHS]
        check(lib.inmsom_gpu_register_grid(self._ctx, *[fptr(m[k]) for k in MASKS],
                                           *[dptr(g[k]) for k in METRICS], dptr(basin.rlh_s),
                                           dptr(basin.hhq_rest), *depths))

    # ------------------------------------------------------------------
    def close(self) -> None:
        if self._ctx:
            _lib.load().inmsom_gpu_finalize(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------
    def _arrays(self, override: dict) -> list:
        b = self.basin
        pools = (b.state, b.means, b.forcing, b.scratch)
        out = []
        for k in DYN_ARGS:
            if k in override:
                out.append(override[k])
                continue
            for p in pools:
                if k in p:
                    out.append(p[k])
                    break
            else:
                raise KeyError(k)
        return out

    def barotropic_dynamics(self, tau: float, nstep: int, ksw4: int = 0, **arrays) -> None:
        """barotropic_dynamics(tau, nstep, ksw4, ubrtr_e, ..., RHSy_dif);
        arrays not given are taken from the Basin."""
        check(load().inmsom_barotropic_dynamics(self._ctx, float(tau), int(nstep), int(ksw4),
                                                *[dptr(a) for a in self._arrays(arrays)]))

    def ssh_internal(self, tau: float, ssh_i, sshp_i, u, v, wflux, hhqn, hhun, hhvn, hhhn) -> None:
        check(load().inmsom_ssh_internal(self._ctx, float(tau), dptr(ssh_i), dptr(sshp_i),
                                         dptr(u), dptr(v), dptr(wflux), dptr(hhqn), dptr(hhun),
                                         dptr(hhvn), dptr(hhhn)))

    def load_state(self) -> None:
        """Upload the Basin's *_e state and forcing (inmsom_load_state)."""
        st, f = self.basin.state, self.basin.forcing
        check(load().inmsom_load_state(self._ctx, *[dptr(st[k]) for k in STATE],
                                       *[dptr(f[k]) for k in ("RHSx", "RHSy", "wflux", "mu", "mu4",
                                                              "rdis")]))

    def run_substeps(self, nsub: int, dt: float, rhs_scale: Optional[Sequence[float]] = None) -> float:
        """Advance the resident state nsub leap-frog substeps; returns the
        device time in ms."""
        ms = ctypes.c_float(0.0)
        sc = None
        if rhs_scale is not None:
            sc = np.ascontiguousarray(rhs_scale, dtype=np.float64)
            if sc.shape != (nsub,):
                raise ValueError("rhs_scale needs one value per substep")
        check(load().inmsom_run_substeps(self._ctx, int(nsub), float(dt),
                                         None if sc is None else sc.ctypes.data_as(_lib.DP),
                                         ctypes.byref(ms)))
        return float(ms.value)

    def closure_features(self, norm, x_ptr: int) -> None:
        """48 BF16 features of every interior cell of the resident state into
        the device buffer at x_ptr (nx * ny * 48 values)."""
        check(load().inmsom_closure_features(self._ctx, ctypes.byref(norm), ctypes.c_void_p(x_ptr)))

    def run_closure(self, nsub: int, dt: float, every: int, params_ptr: int, wbf16_ptr: int, norm) -> float:
        """nsub substeps with the learned closure re-evaluated every `every`
        substeps (inmsom_run_closure); returns the device time in ms."""
        ms = ctypes.c_float(0.0)
        check(load().inmsom_run_closure(self._ctx, int(nsub), float(dt), int(every), ctypes.c_void_p(params_ptr),
                                        ctypes.c_void_p(wbf16_ptr), ctypes.byref(norm), ctypes.byref(ms)))
        return float(ms.value)

    def closure_tendency(self, params_ptr: int, wbf16_ptr: int, norm):
        """(RHSx, RHSy) increments of the closure on the resident state."""
        b = self.basin.bounds
        fx, fy = b.zeros(), b.zeros()
        check(load().inmsom_closure_tendency(self._ctx, ctypes.c_void_p(params_ptr), ctypes.c_void_p(wbf16_ptr),
                                             ctypes.byref(norm), dptr(fx), dptr(fy)))
        return fx, fy

    def wind_forcing(self, taux, tauy, rhsx=None, rhsy=None):
        b = self.basin.bounds
        rhsx = b.zeros() if rhsx is None else rhsx
        rhsy = b.zeros() if rhsy is None else rhsy
        check(load().inmsom_wind_forcing(self._ctx, dptr(taux), dptr(tauy), dptr(rhsx), dptr(rhsy)))
        return rhsx, rhsy

    def rhs2d(self, rhsx, rhsy, diff_disp=(None, None), tran=(None, None), tran_disp=(None, None),
              surf_stress=(None, None), bot_stress=(None, None), slpr=None, hhu=None, hhv=None):
        """Control/dyncall.f90:110-130 on (rhsx, rhsy) in place (inmsom_rhs2d)."""
        check(load().inmsom_rhs2d(self._ctx, dptr(rhsx), dptr(rhsy), dptr(diff_disp[0]), dptr(diff_disp[1]),
                                  dptr(tran[0]), dptr(tran[1]), dptr(tran_disp[0]), dptr(tran_disp[1]),
                                  dptr(surf_stress[0]), dptr(surf_stress[1]), dptr(bot_stress[0]),
                                  dptr(bot_stress[1]), dptr(slpr), dptr(hhu), dptr(hhv)))
        return rhsx, rhsy

    def velocity2d(self, uu2d, vv2d, pgrx, pgry, ubrtr_i, vbrtr_i, slpr, hhu, hhv):
        """Control/dyncall.f90:188-201 in place (inmsom_velocity2d)."""
        check(load().inmsom_velocity2d(self._ctx, dptr(uu2d), dptr(vv2d), dptr(pgrx), dptr(pgry), dptr(ubrtr_i),
                                       dptr(vbrtr_i), dptr(slpr), dptr(hhu), dptr(hhv)))
        return uu2d, vv2d, pgrx, pgry

    BAROCLINIC_FIELDS = ("ww", "nu", "rhsx", "rhsy", "rhsx_tran", "rhsy_tran", "pgrx", "pgry", "rdis",
                         "tx_surf", "ty_surf", "tx_bot", "ty_bot", "hhu", "hhup", "hhun", "hhv", "hhvp",
                         "hhvn", "hhh")

    def baroclinic_dynamics(self, dz, hzt, tau: float, uu, uup, vv, vvp, **fields):
        """Function/vel_ssh.f90:794-1027 in place on uu, uup, vv, vvp
        (inmsom_baroclinic_dynamics).  3-D arrays are (bnd_x, bnd_y, nz) in
        Fortran order, ww and nu with nz + 1 levels; `fields` holds
        BAROCLINIC_FIELDS by name (hh*: the internal-mode depths)."""
        dz = np.ascontiguousarray(dz, dtype=np.float64)
        hzt = np.ascontiguousarray(hzt, dtype=np.float64)
        nz = len(dz)
        if len(hzt) != nz + 1:
            raise ValueError("hzt needs nz + 1 values")
        shp = self.basin.bounds.shape
        for name, a in (("uu", uu), ("uup", uup), ("vv", vv), ("vvp", vvp)):
            if a.shape != (*shp, nz):
                raise ValueError(f"{name}: expected shape {(*shp, nz)}")
        for name in ("ww", "nu"):
            if fields[name].shape != (*shp, nz + 1):
                raise ValueError(f"{name}: expected shape {(*shp, nz + 1)}")
        for name in ("rhsx", "rhsy", "rhsx_tran", "rhsy_tran"):
            if fields[name].shape != (*shp, nz):
                raise ValueError(f"{name}: expected shape {(*shp, nz)}")
        check(load().inmsom_baroclinic_dynamics(self._ctx, nz, dz.ctypes.data_as(_lib.DP), hzt.ctypes.data_as(_lib.DP),
                                                float(tau), dptr(uu), dptr(uup), dptr(vv), dptr(vvp),
                                                *[dptr(fields[k]) for k in self.BAROCLINIC_FIELDS]))
        return uu, uup, vv, vvp

    def vertical_velocity(self, dz, u, v, w, hu, hv, wflux):
        """Function/vel_ssh.f90:1030-1076: w (nz + 1 levels) in place
        (inmsom_vertical_velocity)."""
        dz = np.ascontiguousarray(dz, dtype=np.float64)
        nz = len(dz)
        shp = self.basin.bounds.shape
        if u.shape != (*shp, nz) or v.shape != (*shp, nz) or w.shape != (*shp, nz + 1):
            raise ValueError("u, v need nz levels and w nz + 1")
        check(load().inmsom_vertical_velocity(self._ctx, nz, dz.ctypes.data_as(_lib.DP), dptr(u), dptr(v), dptr(w),
                                              dptr(hu), dptr(hv), dptr(wflux)))
        return w

    def tracer_tran_diff(self, dz, hzt, tau: float, ff, ffp, flux_f_x, flux_f_y, f: dict):
        """Function/tem_sal.f90:1-422 in place on ff, ffp (nz levels) and the
        diagnostics flux_f_x, flux_f_y (bnd_x, bnd_y, 4)
        (inmsom_tracer_tran_diff); f holds the other arguments by the
        reference's names (basins.tracer_fields)."""
        dz = np.ascontiguousarray(dz, dtype=np.float64)
        hzt = np.ascontiguousarray(hzt, dtype=np.float64)
        nz = len(dz)
        shp = self.basin.bounds.shape
        for name, a, lev in (("ff", ff, nz), ("ffp", ffp, nz), ("flux_f_x", flux_f_x, 4), ("flux_f_y", flux_f_y, 4),
                             *[(k, f[k], nz) for k in ("uu", "vv", "mu", "src")],
                             *[(k, f[k], nz + 1) for k in ("ww", "nu", "slrx", "slry", "slzx", "slzy")]):
            if a.shape != (*shp, lev):
                raise ValueError(f"{name}: expected shape {(*shp, lev)}")
        ip = ctypes.POINTER(ctypes.c_int)
        igt = np.asfortranarray(f["ig_top"], dtype=np.int32)
        igb = np.asfortranarray(f["ig_bot"], dtype=np.int32)
        check(load().inmsom_tracer_tran_diff(
            self._ctx, nz, dz.ctypes.data_as(_lib.DP), hzt.ctypes.data_as(_lib.DP), dptr(ff), dptr(ffp), float(tau),
            dptr(f["uu"]), dptr(f["vv"]), dptr(f["ww"]), dptr(f["mu"]), float(f["factor_mu"]), dptr(f["nu"]),
            float(f["factor_nu"]), dptr(f["slrx"]), dptr(f["slry"]), dptr(f["slzx"]), dptr(f["slzy"]),
            float(f["az"]), float(f["ar"]), float(f["alpha_gm"]), dptr(f["ff_top"]), dptr(f["ff_bot"]),
            igt.ctypes.data_as(ip), igb.ctypes.data_as(ip), dptr(flux_f_x), dptr(flux_f_y), dptr(f["swbal"]),
            0, 0, None, None, None, None, dptr(f["src"]), float(f["src_factor"]), dptr(f["hhu"]), dptr(f["hhv"]),
            dptr(f["hhqn"]), dptr(f["hhqp"])))
        return ff, ffp, flux_f_x, flux_f_y

    def depth_ave(self, dz, u, utr, mask, kbcl: int):
        """Function/depth.f90:223-254 in place on u (nz levels) and utr
        (inmsom_depth_ave)."""
        dz = np.ascontiguousarray(dz, dtype=np.float64)
        if u.shape != (*self.basin.bounds.shape, len(dz)):
            raise ValueError("u needs nz levels")
        check(load().inmsom_depth_ave(self._ctx, len(dz), dz.ctypes.data_as(_lib.DP), dptr(u), dptr(utr),
                                      fptr(mask), int(kbcl)))
        return u, utr

    def stress_components(self, u, v, str_t, str_s):
        """Function/mixing.f90:115-168 on the levels of u, v, in place on
        str_t, str_s (inmsom_stress_components)."""
        arrs = (u, v, str_t, str_s)
        if any(a.shape != u.shape or a.shape[:2] != self.basin.bounds.shape for a in arrs):
            raise ValueError("u, v, str_t, str_s need the array shape and the same levels")
        nlev = u.shape[2] if u.ndim == 3 else 1
        check(load().inmsom_stress_components(self._ctx, nlev, *[dptr(a) for a in arrs]))
        return str_t, str_s

    def smagorinsky_coeff(self, visc2: float, dift: float, str_t, str_s, amts, amuv):
        """Function/mixing.f90:171-219 in place on amts, amuv
        (inmsom_smagorinsky_coeff)."""
        arrs = (str_t, str_s, amts, amuv)
        if any(a.shape != str_t.shape or a.shape[:2] != self.basin.bounds.shape for a in arrs):
            raise ValueError("str_t, str_s, amts, amuv need the array shape and the same levels")
        nz = str_t.shape[2] if str_t.ndim == 3 else 1
        check(load().inmsom_smagorinsky_coeff(self._ctx, nz, float(visc2), float(dift),
                                              *[dptr(a) for a in arrs]))
        return amts, amuv

    def shift_barotropic(self, uu, vv, uu2d, vv2d, sign: int):
        """Control/dyncall.f90:170-183 (sign -1) / :215-229 (sign +1) in
        place on uu, vv (inmsom_shift_barotropic)."""
        nz = uu.shape[2]
        if uu.shape != vv.shape or uu.shape[:2] != self.basin.bounds.shape:
            raise ValueError("uu, vv need the array shape and nz levels")
        check(load().inmsom_shift_barotropic(self._ctx, nz, dptr(uu), dptr(vv), dptr(uu2d), dptr(vv2d), int(sign)))
        return uu, vv

    def write_checkpoint(self, path: str, xt, xu, yt, yv, dxst: float, dyst: float, xgr_type: int = 0,
                         ygr_type: int = 0, calendar: int = 1, date=(2000, 1, 1, 0, 0), tstep: float = 86400.0):
        """The barotropic checkpoint of Control/output.f90:1736-1847 from
        the resident state into `path` (inmsom_write_checkpoint); xt, xu,
        yt, yv: the first coordinate (LINEAR axes) or all of them (LEVELS)."""
        keep = [np.ascontiguousarray(np.atleast_1d(v), dtype=np.float64) for v in (xt, xu, yt, yv)]
        ax = _lib.CCtlAxes(xgr_type, ygr_type, *[k.ctypes.data_as(_lib.DP) for k in keep], float(dxst), float(dyst),
                           calendar, *[int(x) for x in date], float(tstep))
        check(load().inmsom_write_checkpoint(self._ctx, path.encode(), ctypes.byref(ax)))

    def read_checkpoint(self, path: str, into_basin: bool = True) -> None:
        """Restart the resident state from cp*8.dat files in `path`
        (inmsom_read_checkpoint); with into_basin, the basin's state arrays
        receive the fields too."""
        st = self.basin.state
        arrs = [st[k] if into_basin else None for k in ("ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e", "ssh_e",
                                                         "sshp_e")]
        check(load().inmsom_read_checkpoint(self._ctx, path.encode(), *[dptr(a) for a in arrs]))

    def r_diss(self, r_fric: float, out=None):
        out = self.basin.bounds.zeros() if out is None else out
        check(load().inmsom_r_diss(self._ctx, float(r_fric), dptr(out)))
        return out

    def hh_init_external(self, ssh_e=None, sshp_e=None) -> None:
        s = self.basin.state
        check(load().inmsom_hh_init_external(self._ctx, dptr(s["ssh_e"] if ssh_e is None else ssh_e),
                                             dptr(s["sshp_e"] if sshp_e is None else sshp_e)))

    def guard(self) -> int:
        n = ctypes.c_long(0)
        check(load().inmsom_guard(self._ctx, ctypes.byref(n)))
        return int(n.value)

    def diag(self):
        v, e = ctypes.c_double(), ctypes.c_double()
        check(load().inmsom_gpu_diag(self._ctx, ctypes.byref(v), ctypes.byref(e)))
        return float(v.value), float(e.value)

    def sync_to_host(self, what: int = _lib.SYNC_STATE) -> None:
        check(load().inmsom_gpu_sync_to_host(self._ctx, what))

    def sync_from_host(self, what: int = _lib.SYNC_STATE) -> None:
        check(load().inmsom_gpu_sync_from_host(self._ctx, what))

    def last_phases(self):
        """(upload, compute, download) device ms of the last
        barotropic_dynamics call."""
        a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        check(load().inmsom_gpu_last_phases(self._ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return float(a.value), float(b.value), float(c.value)

    def path(self):
        p, r = ctypes.c_int(), ctypes.c_char_p()
        check(load().inmsom_gpu_path(self._ctx, ctypes.byref(p), ctypes.byref(r)))
        return int(p.value), (r.value or b"").decode()


class Ensemble:
    """Independent basins advanced together (inmsom_ens_*): each member is a
    BarotropicSolver with its state resident; `group` substeps of all
    members per CUDA-graph launch.  Creation re-cuts each member's work
    items to 16 rows at least (a solver alone cuts down to 4), and the
    members keep that cut, as they keep what tune() chooses."""

    def __init__(self, members: Sequence["BarotropicSolver"], group: int = 10, persistent: bool = False):
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m._ctx.value for m in self.members])
        self._ens = ctypes.c_void_p()
        check(load().inmsom_ens_create(ctypes.byref(self._ens), arr, len(self.members), int(group)))
        if persistent:
            self.set_persistent(True)

    def set_persistent(self, on: bool) -> None:
        """One persistent cooperative launch per group of substeps
        (inmsom_ens_persistent) instead of one launch per member and substep."""
        check(load().inmsom_ens_persistent(self._ens, 1 if on else 0))

    def _dt(self, dt):
        a = np.ascontiguousarray(dt, dtype=np.float64)
        if a.shape != (len(self.members),):
            raise ValueError("one dt per member")
        return a

    def run(self, nsub: int, dt, rhs_scale: Optional[Sequence[float]] = None) -> float:
        """Advance every member nsub substeps of its dt; returns device ms."""
        d = self._dt(dt)
        sc = None
        if rhs_scale is not None:
            sc = np.ascontiguousarray(rhs_scale, dtype=np.float64)
            if sc.shape != (nsub,):
                raise ValueError("rhs_scale needs one value per substep")
        ms = ctypes.c_float(0.0)
        check(load().inmsom_ens_run(self._ens, int(nsub), dptr(d), None if sc is None else dptr(sc),
                                    ctypes.byref(ms)))
        return float(ms.value)

    def tune(self, dt, trial_groups: int = 2):
        """Autotune chunk heights per size class in the ensemble's current
        form (graph or persistent); the cut before tuning stays unless the
        tuned one is faster.  Returns rows per item per member (0 = one wave
        of cost-balanced chunks).  Advances the states."""
        d = self._dt(dt)
        out = (ctypes.c_int * len(self.members))()
        check(load().inmsom_ens_tune(self._ens, dptr(d), int(trial_groups), out))
        return list(out)

    def close(self) -> None:
        if self._ens:
            load().inmsom_ens_destroy(self._ens)
            self._ens = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Strips:
    """Row strips of one basin advanced together (inmsom_strips_*): each
    strip is a BarotropicSolver of a Basin from strips.split_basin, south
    to north, with its state resident."""

    def __init__(self, members: Sequence["BarotropicSolver"]):
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m._ctx.value for m in self.members])
        self._g = ctypes.c_void_p()
        check(load().inmsom_strips_create(ctypes.byref(self._g), arr, len(self.members)))

    def run(self, nsub: int, dt: float, rhs_scale: Optional[Sequence[float]] = None) -> float:
        sc = None
        if rhs_scale is not None:
            sc = np.ascontiguousarray(rhs_scale, dtype=np.float64)
            if sc.shape != (nsub,):
                raise ValueError("rhs_scale needs one value per substep")
        ms = ctypes.c_float(0.0)
        check(load().inmsom_strips_run(self._g, int(nsub), float(dt), None if sc is None else dptr(sc),
                                       ctypes.byref(ms)))
        return float(ms.value)

    def close(self) -> None:
        if self._g:
            load().inmsom_strips_destroy(self._g)
            self._g = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuBackend:
    """Basin set-up on the GPU: gridcon and the wind forcing."""

    def __init__(self, device: int = 0):
        self.device = device

    def gridcon(self, bounds, lu):
        return gridcon(bounds, lu, self.device)

    def wind_forcing(self, basin: Basin):
        with BarotropicSolver(basin, self.device, register_depths=False) as s:
            return s.wind_forcing(basin.taux, basin.tauy)
