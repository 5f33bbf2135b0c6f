"""The reference's on-disk formats through the C ABI.

DIOGIN-standard direct-access files (Service/input_output_data.f90:117-534):
one record per level of a box of a field, x fastest, FP64 (wdstd8/rdstd8)
or FP32 (wdstd/rdstd), land points written as undef = -1.0e32 and read as 0;
their MPI-IO forms pwdstd/prdstd (:535-819), one rank's subdomain of the
same FP32 file.
GrADS descriptors (Service/rw_ctl_file.f90:1-139 ctl_file_write and
:185-566 ctl_file_read).  Arrays are Fortran-ordered numpy arrays (nx, ny[,
nz]); boxes are 1-based inclusive (nxb, nxe, nyb, nye, nzb, nze) as in the
reference's argument lists.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import DP, FP, check, load

UNDEF = np.float32(-1.0e32)


def _dims(field):
    nx, ny = field.shape[:2]
    nz = field.shape[2] if field.ndim == 3 else 1
    return nx, ny, nz


def _box(field, box):
    nx, ny, nz = _dims(field)
    return tuple(box) if box is not None else (1, nx, 1, ny, 1, nz)


def _call(name, ptr, dtype, path, fname, nfield, field, lu, box):
    if field.dtype != dtype or not field.flags.f_contiguous:
        raise TypeError(f"{name}: expected a Fortran-ordered {np.dtype(dtype).name} array")
    lu = np.asfortranarray(lu, dtype=np.float32)
    nx, ny, nz = _dims(field)
    if lu.shape != (nx, ny):
        raise ValueError(f"{name}: lu must have the field's first two dimensions")
    check(getattr(load(), name)(path.encode(), fname.encode(), int(nfield), field.ctypes.data_as(ptr),
                                lu.ctypes.data_as(FP), nx, ny, nz, *_box(field, box)))
    return field


def wdstd8(path, fname, nfield, field, lu, box=None):
    """inmsom_wdstd8; like the reference, leaves the box's land points of
    `field` at 0."""
    return _call("inmsom_wdstd8", DP, np.float64, path, fname, nfield, field, lu, box)


def wdstd(path, fname, nfield, field, lu, box=None):
    return _call("inmsom_wdstd", FP, np.float32, path, fname, nfield, field, lu, box)


def rdstd8(path, fname, nfield, field, lu, box=None):
    return _call("inmsom_rdstd8", DP, np.float64, path, fname, nfield, field, lu, box)


def rdstd(path, fname, nfield, field, lu, box=None):
    return _call("inmsom_rdstd", FP, np.float32, path, fname, nfield, field, lu, box)


def ctl_file_write(fname, undef, nx, ny, nz, nt, xtype, x0, hx, ytype, y0, hy, ztype, z0, hz, yr_type, year0,
                   month0, day0, hour0, minute0, ht, title, varname):
    """inmsom_ctl_file_write: x0, y0, z0 are sequences (one value for a
    LINEAR axis, nx/ny/nz values for LEVELS)."""
    arrs = [np.ascontiguousarray(np.atleast_1d(v), dtype=np.float64) for v in (x0, y0, z0)]
    check(load().inmsom_ctl_file_write(fname.encode(), float(undef), nx, ny, nz, nt, xtype,
                                       arrs[0].ctypes.data_as(DP), float(hx), ytype, arrs[1].ctypes.data_as(DP),
                                       float(hy), ztype, arrs[2].ctypes.data_as(DP), float(hz), yr_type, year0,
                                       month0, day0, hour0, minute0, float(ht), title.encode(), varname.encode()))


def ctl_file_read(ctlname, x_cap=4096, y_cap=4096, z_cap=1024, var_cap=16, name_len=256):
    """inmsom_ctl_file_read (Service/rw_ctl_file.f90:185-566): a dict of the
    reference's output arguments; x0, y0, z0 hold nx, ny, nz values (at
    least one), varname the nvar names.  Arguments the descriptor does not
    set come back as 0 (the reference leaves them as they were)."""
    I, F, D = ctypes.c_int, ctypes.c_float, ctypes.c_double
    ints = {k: I(0) for k in ("nx", "ny", "nz", "nt", "xtype", "ytype", "ztype", "nvar", "yr_type", "year0",
                              "month0", "day0", "hour0", "minute0", "inform")}
    undef, ht, hx, hy, hz = F(0), F(0), D(0), D(0), D(0)
    x0, y0, z0 = (np.zeros(max(n, 1)) for n in (x_cap, y_cap, z_cap))
    datname, title = ctypes.create_string_buffer(name_len), ctypes.create_string_buffer(name_len)
    names = ctypes.create_string_buffer(var_cap * name_len)
    r = ctypes.byref
    check(load().inmsom_ctl_file_read(
        str(ctlname).encode(), datname, name_len, r(undef), r(ints["nx"]), r(ints["ny"]), r(ints["nz"]),
        r(ints["nt"]), r(ints["xtype"]), x0.ctypes.data_as(DP), len(x0), r(hx), r(ints["ytype"]),
        y0.ctypes.data_as(DP), len(y0), r(hy), r(ints["ztype"]), z0.ctypes.data_as(DP), len(z0), r(hz),
        r(ints["nvar"]), r(ints["yr_type"]), r(ints["year0"]), r(ints["month0"]), r(ints["day0"]),
        r(ints["hour0"]), r(ints["minute0"]), r(ht), title, name_len, names, name_len, var_cap, r(ints["inform"])))
    out = {k: v.value for k, v in ints.items()}
    nvar = max(out["nvar"], 0)
    out.update(datname=datname.value.decode(), title=title.value.decode(), undef=np.float32(undef.value),
               ht=np.float32(ht.value), hx=hx.value, hy=hy.value, hz=hz.value,
               x0=x0[:max(out["nx"], 1)].copy(), y0=y0[:max(out["ny"], 1)].copy(), z0=z0[:max(out["nz"], 1)].copy(),
               varname=[names.raw[k * name_len:(k + 1) * name_len].split(b"\0", 1)[0].decode()
                        for k in range(min(nvar, var_cap))])
    return out


def _pcall(name, bounds, path, fname, nfild, fild, lu, nx, ny, nz, box):
    from ._lib import cbounds
    if fild.dtype != np.float32 or not fild.flags.f_contiguous:
        raise TypeError(f"{name}: expected a Fortran-ordered float32 array")
    if fild.shape[:2] != bounds.shape:
        raise ValueError(f"{name}: the local array must have the bounds' shape {bounds.shape}")
    lu = np.asfortranarray(lu, dtype=np.float32)
    if lu.shape != bounds.shape:
        raise ValueError(f"{name}: lu must have the bounds' shape {bounds.shape}")
    cb = cbounds(bounds)
    check(getattr(load(), name)(ctypes.byref(cb), path.encode(), fname.encode(), int(nfild), fild.ctypes.data_as(FP),
                                lu.ctypes.data_as(FP), int(nx), int(ny), int(nz), *box))
    return fild


def pwdstd(bounds, path, fname, nfild, fild, lu, nx, ny, nz, box):
    """inmsom_pwdstd (Service/input_output_data.f90:657-819): this rank's
    interior of the local float32 array fild (bounds.shape[+ (nz,)]) into
    the file every rank shares; nx, ny, nz and the 1-based box are global.
    Like the reference, sets the interior's land points of fild to undef."""
    return _pcall("inmsom_pwdstd", bounds, path, fname, nfild, fild, lu, nx, ny, nz, box)


def prdstd(bounds, path, fname, nfild, fild, lu, nx, ny, nz, box):
    """inmsom_prdstd (Service/input_output_data.f90:535-652): this rank's
    interior of fild from the shared file (every point; values past the
    end of the file are left as they were)."""
    return _pcall("inmsom_prdstd", bounds, path, fname, nfild, fild, lu, nx, ny, nz, box)


def _ocean_state(state, bounds, nz):
    """COceanState over the arrays of `state` (a dict by field name; pairs
    left out are skipped), each checked for its shape."""
    from ._lib import OCEAN_STATE_FIELDS, COceanState
    cs = COceanState()
    for name in OCEAN_STATE_FIELDS:
        a = state.get(name)
        if a is None:
            continue
        lev = (nz if name in ("tt", "ttp", "ss", "ssp", "uu", "uup", "vv", "vvp")
               else nz + 1 if name in ("q2", "q2p", "q2l", "q2lp") else 1)
        want = bounds.shape + ((lev,) if lev > 1 else ())
        if a.dtype != np.float64 or not a.flags.f_contiguous or a.shape[:len(want)] != want or a.size != np.prod(want):
            raise ValueError(f"{name}: expected a Fortran-ordered float64 array of shape {want}")
        setattr(cs, name, a.ctypes.data_as(DP))
    return cs


def ocpwrite(path, bounds, nz, lu, llu, llv, z, zw, axes, state):
    """inmsom_ocpwrite (Control/output.f90:1454-1847): the checkpoint files
    of every pair in `state` (a dict: tt, ttp, ..., vbrtrp_e); `axes` is a
    dict of xt, xu, yt, yv (first values for LINEAR axes), dxst, dyst and
    optionally xgr_type, ygr_type, calendar, date=(y, mo, d, h, mn), tstep.
    Like the reference, zeroes the written land points of the arrays."""
    from ._lib import CCtlAxes, cbounds
    keep = [np.ascontiguousarray(np.atleast_1d(axes[k]), dtype=np.float64) for k in ("xt", "xu", "yt", "yv")]
    ax = CCtlAxes(axes.get("xgr_type", 0), axes.get("ygr_type", 0), *[k.ctypes.data_as(DP) for k in keep],
                  float(axes["dxst"]), float(axes["dyst"]), axes.get("calendar", 1),
                  *[int(x) for x in axes.get("date", (2000, 1, 1, 0, 0))], float(axes.get("tstep", 86400.0)))
    zs = [np.ascontiguousarray(v, dtype=np.float64) for v in (z, zw)]
    if zs[0].size < nz or zs[1].size < nz + 1:
        raise ValueError("z needs nz values and zw nz+1")
    masks = [np.asfortranarray(m, dtype=np.float32) for m in (lu, llu, llv)]
    cb = cbounds(bounds)
    cs = _ocean_state(state, bounds, nz)
    check(load().inmsom_ocpwrite(str(path).encode(), ctypes.byref(cb), int(nz), *[m.ctypes.data_as(FP) for m in masks],
                                 zs[0].ctypes.data_as(DP), zs[1].ctypes.data_as(DP), ctypes.byref(ax),
                                 ctypes.byref(cs)))


def ocpread(path, bounds, nz, lu, llu, llv, state, tur_var_min=1.0e-8):
    """inmsom_ocpread: the restart of every pair in `state` (arrays filled in
    place) from the checkpoint files in `path`."""
    from ._lib import cbounds
    masks = [np.asfortranarray(m, dtype=np.float32) for m in (lu, llu, llv)]
    cb = cbounds(bounds)
    cs = _ocean_state(state, bounds, nz)
    check(load().inmsom_ocpread(str(path).encode(), ctypes.byref(cb), int(nz),
                                *[m.ctypes.data_as(FP) for m in masks], float(tur_var_min), ctypes.byref(cs)))
    return state


def compare_grids(a, b, maxgridlen=4096):
    """inmsom_compare_grids (Service/rw_ctl_file.f90:628-714) on two
    ctl_file_read results: 0 same grids, 1 too long or different counts,
    2 different coordinates."""
    ierr = ctypes.c_int(-1)

    def args(g):
        arrs = [np.ascontiguousarray(np.resize(np.asarray(g[k], dtype=np.float64), max(len(g[k]), 1)))
                for k in ("x0", "y0", "z0")]
        return arrs, [float(g["undef"]), g["nx"], g["ny"], g["nz"], g["nt"], arrs[0].ctypes.data_as(DP), g["hx"],
                      arrs[1].ctypes.data_as(DP), g["hy"], 0.0, float(g["ht"]), arrs[2].ctypes.data_as(DP), g["hz"]]

    keep_a, la = args(a)
    keep_b, lb = args(b)
    check(load().inmsom_compare_grids(int(maxgridlen), ctypes.byref(ierr), *la, *lb))
    return ierr.value
