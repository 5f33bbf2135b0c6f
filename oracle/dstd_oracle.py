"""Test infrastructure (the checker, never the product): a numpy/Python
restatement of the reference's on-disk formats.

* wdstd / wdstd8 / rdstd8 (Service/input_output_data.f90:117-534): the
  records of a box, x fastest, one per level, record number
  (nfield-1)*(nze-nzb+1) + (k-nzb+1), land (|lu| < 0.5) as undef = -1.0e32
  (Inc/reclen.fi:6), FP32 or FP64.
* ctl_file_write (Service/rw_ctl_file.f90:1-139) with the Fortran 2008
  rules for the Ew.d, Gw.d, Iw and Iw.m edit descriptors it uses
  (10.7.2.3.3, 10.7.5.2.2, 10.7.2.2), and sec_to_yr_mo_hr_mn (:161-183).

Parity unpinned: no Fortran compiler exists here, so no file written by the
reference itself is available; these restate the reference's statements.
"""
from __future__ import annotations

import numpy as np

UNDEF = np.float32(-1.0e32)
MONTHS = ["JAN", "FEB", "MAR", "APR", "MAY", "JUN", "JUL", "AUG", "SEP", "OCT", "NOV", "DEC"]


def _as3(a):
    return a if a.ndim == 3 else a[:, :, None]


def records(field, lu, box, dtype):
    """The bytes of each level record wdstd (float32) / wdstd8 (float64)
    writes for the 1-based box (nxb, nxe, nyb, nye, nzb, nze)."""
    nxb, nxe, nyb, nye, nzb, nze = box
    f = _as3(field)
    land = np.abs(lu[nxb - 1:nxe, nyb - 1:nye]) < 0.5
    out = []
    for k in range(nzb, nze + 1):
        sub = np.where(land, dtype(UNDEF), f[nxb - 1:nxe, nyb - 1:nye, k - 1].astype(dtype))
        out.append(np.asarray(sub, dtype=dtype).tobytes(order="F"))
    return out


def record_offset(nfield, box, kr, itemsize):
    """Byte offset of record kr (1-based) of field nfield."""
    nxb, nxe, nyb, nye, nzb, nze = box
    recl = (nxe - nxb + 1) * (nye - nyb + 1) * itemsize
    return ((nfield - 1) * (nze - nzb + 1) + kr - 1) * recl


def read_field(data: bytes, nfield, box, dtype, lu, field):
    """rdstd/rdstd8 on the bytes of a file: the box of `field` (in place),
    land points 0."""
    nxb, nxe, nyb, nye, nzb, nze = box
    f = _as3(field)
    bx, by = nxe - nxb + 1, nye - nyb + 1
    isz = np.dtype(dtype).itemsize
    land = np.abs(lu[nxb - 1:nxe, nyb - 1:nye]) < 0.5
    for kr, k in enumerate(range(nzb, nze + 1), start=1):
        off = record_offset(nfield, box, kr, isz)
        rec = np.frombuffer(data[off:off + bx * by * isz], dtype=dtype).reshape((bx, by), order="F")
        f[nxb - 1:nxe, nyb - 1:nye, k - 1] = np.where(land, 0.0, rec)
    return field


# ---- Fortran editing --------------------------------------------------------

def _right(s, w):
    return "*" * w if len(s) > w else " " * (w - len(s)) + s


def _digits(x, d):
    """d significant decimal digits of |x| (correctly rounded) and N with
    |x| ~ 0.d1..dd x 10**N."""
    m, e = f"{abs(x):.{d - 1}e}".split("e")
    return m.replace(".", ""), int(e) + 1


def edit_e(x, w, d):
    sign = "-" if x < 0 else ""
    if x == 0:
        s = "0." + "0" * d + "E+00"
    else:
        dig, n = _digits(x, d)
        ex = f"E{'-' if n < 0 else '+'}{abs(n):02d}" if abs(n) <= 99 else f"{'-' if n < 0 else '+'}{abs(n):03d}"
        s = "0." + dig + ex
    s = sign + s
    if len(s) > w:                       # the optional zero before the point
        s = s.replace("0.", ".", 1)
    return _right(s, w)


def edit_f(x, w, d):
    s = f"{x:.{d}f}" + ("." if d == 0 else "")     # Fw.0 still writes the point
    if s.startswith("-") and float(s) == 0.0:
        s = s[1:]
    if len(s) > w:
        s = s.replace("0.", ".", 1)
    return _right(s, w)


def edit_g(x, w, d):
    if x == 0:
        return edit_f(0.0, w - 4, d - 1) + " " * 4
    _, n = _digits(x, d)
    if 0 <= n <= d:
        return edit_f(x, w - 4, d - n) + " " * 4
    return edit_e(x, w, d)


def edit_i(v, w, m=0):
    s = str(abs(int(v))).rjust(m, "0")
    return _right(("-" if v < 0 else "") + s, w)


def sec_to_yr_mo_hr_mn(sec):
    f = np.float32
    yr, mo = f(360.0) * f(86400.0), f(30.0) * f(86400.0)
    s1 = f(sec) + f(0.10)
    nyr = int(s1 / yr); s1 = f(s1 - f(nyr) * yr)
    nmo = int(s1 / mo); s1 = f(s1 - f(nmo) * mo)
    ndy = int(s1 / f(86400.0)); s1 = f(s1 - f(ndy) * f(86400.0))
    nhr = int(s1 / f(3600.0)); s1 = f(s1 - f(nhr) * f(3600.0))
    nmn = int(s1 / f(60.0))
    return nyr, nmo, ndy, nhr, nmn


def _axis(tag, n, typ, v, h):
    """The trailing 5x / 1x of each record skip positions that no character
    follows, so they write nothing (Fortran 2008 10.8.1.1)."""
    s = tag + edit_i(n, 6)
    if typ == 0:
        return s + "  LINEAR   " + edit_g(v[0], 15, 8) + " " * 5 + edit_g(h, 15, 8) + "\n"
    s += "  LEVELS  "
    fields = [edit_g(x, 15, 8) for x in v[:n]]
    rows = [" ".join(fields[i:i + 7]) for i in range(0, n, 7)]
    return s + ("\n" + " " * 22).join(rows) + "\n"


def extname(name, ext):
    s = name[:128].ljust(128)
    n = next((p for p in range(125, 1, -1) if s[p - 1] == "."), 2)
    s = s[:n - 1] + ext.ljust(5) + s[n + 4:]
    return s.rstrip()


def ctl_text(fname, undef, nx, ny, nz, nt, xtype, x0, hx, ytype, y0, hy, ztype, z0, hz, yr_type, year0, month0,
             day0, hour0, minute0, ht, title, varname):
    """(name of the .ctl file, its text) as ctl_file_write writes them."""
    namectl, namedat = extname(fname, ".ctl"), extname(fname, ".dat")
    namedat2 = namedat.rsplit("/", 1)[-1].ljust(128)
    t = f"DSET    ^{namedat2}\n"
    t += f"TITLE    {title}\n"
    t += "UNDEF   " + edit_e(float(np.float32(undef)), 12, 5) + "  ! gap value\n"
    t += _axis("XDEF  ", nx, xtype, x0, hx) + _axis("YDEF  ", ny, ytype, y0, hy) + _axis("ZDEF  ", nz, ztype, z0, hz)
    nyr, nmo, ndy, nhr, nmn = sec_to_yr_mo_hr_mn(ht)
    k, tf = namedat.rfind("/") + 1, "  "          # unset unit; k from the DSET name search
    for val, tag in ((nyr, "yr"), (nmo, "mo"), (ndy, "dy"), (nhr, "hr"), (nmn, "mn")):
        if val != 0:
            k, tf = val, tag
            break
    t += ("TDEF  " + edit_i(nt, 6) + "  LINEAR  " + edit_i(hour0, 2, 2) + ":" + edit_i(minute0, 2, 2) + "Z"
          + edit_i(day0, 2, 2) + MONTHS[month0 - 1] + edit_i(year0, 4, 4) + " " * 5 + edit_i(k, 4) + tf + "\n")
    if yr_type == 0:
        t += "OPTIONS  365_DAY_CALENDAR\n"
    t += "VARS 1  ! Number of variables\n"
    t += varname + " " * 8 + edit_i(nz, 5) + "  1 VARIABLES \n"
    t += "ENDVARS\n\n"
    return namectl, t
