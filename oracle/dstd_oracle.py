"""Test infrastructure (the checker, never the product): a numpy/Python
restatement of the reference's on-disk formats.

* wdstd / wdstd8 / rdstd8 (Service/input_output_data.f90:117-534): the
  records of a box, x fastest, one per level, record number
  (nfield-1)*(nze-nzb+1) + (k-nzb+1), land (|lu| < 0.5) as undef = -1.0e32
  (Inc/reclen.fi:6), FP32 or FP64.
* ctl_file_write (Service/rw_ctl_file.f90:1-139) with the Fortran 2008
  rules for the Ew.d, Gw.d, Iw and Iw.m edit descriptors it uses
  (10.7.2.3.3, 10.7.5.2.2, 10.7.2.2), and sec_to_yr_mo_hr_mn (:161-183).
* ctl_file_read (Service/rw_ctl_file.f90:185-566) and nonblank (:568-596),
  with the list-directed input rules its READ statements use
  (Fortran 2008 10.10.3).

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


# ---- ctl_file_read (Service/rw_ctl_file.f90:185-566, nonblank :568-596) ------

class CtlError(ValueError):
    """The reference prints an error message and returns, or stops on an
    end of file."""


def _f32(x):
    return float(np.float32(x))


def _values(rec):
    """The values of one list-directed record (blanks/commas separate,
    quotes delimit, r*c repeats) and whether a slash ended it.  Null values
    raise."""
    vals, i, n = [], 0, len(rec)
    while i < n:
        commas = 0
        while i < n and rec[i] in " \t,":
            commas += rec[i] == ","
            i += 1
        if commas > 1:
            raise CtlError("null value")
        if i >= n:
            return vals, False
        if rec[i] == "/":
            return vals, True
        if rec[i] in "'\"":
            q, j, tok = rec[i], i + 1, ""
            while j < n:
                if rec[j] == q and j + 1 < n and rec[j + 1] == q:
                    tok, j = tok + q, j + 2
                elif rec[j] == q:
                    j += 1
                    break
                else:
                    tok, j = tok + rec[j], j + 1
            vals.append(tok)
            i = j
            continue
        j = i
        while j < n and rec[j] not in " \t,/":
            j += 1
        tok, i = rec[i:j], j
        head, star, tail = tok.partition("*")
        if star and head.isdigit():
            if not tail:
                raise CtlError("null value")
            vals += [tail] * int(head)
        else:
            vals.append(tok)
    return vals, False


def _int(t):
    try:
        return int(t.strip())
    except ValueError:
        raise CtlError(f"not an integer: {t!r}") from None


def _real(t):
    u = t.strip().upper().replace("D", "E").replace("Q", "E")
    if "E" not in u:
        for k in range(1, len(u)):
            if u[k] in "+-" and (u[k - 1].isdigit() or u[k - 1] == "."):
                u = u[:k] + "E" + u[k:]
                break
    try:
        return float(u)
    except ValueError:
        raise CtlError(f"not a real: {t!r}") from None


def _spelled(s, word):
    w = s[:len(word)]
    return w in (word, word.lower(), word.capitalize())


def ctl_read(text, datname_len=255, title_len=255):
    """The output arguments of ctl_file_read on a descriptor's text, as a
    dict (arguments it does not set are absent).  Raises CtlError where the
    reference prints an error or stops."""
    recs = [ln.rstrip("\r")[:256].ljust(256) for ln in text.split("\n")]
    if text.endswith("\n"):
        recs.pop()
    out = {"inform": 0, "datname": "", "yr_type": 1}
    nxt = 0

    def ext_read(need):
        """READ(40, *) from the next record on."""
        nonlocal nxt
        vals = []
        while len(vals) < need:
            if nxt >= len(recs):
                raise CtlError("end of file")
            v, slash = _values(recs[nxt])
            nxt += 1
            vals += v
            if slash:
                break
        return vals

    for _line in range(512):
        if nxt >= len(recs):
            raise CtlError("exit by eof, not by endvars")
        s = recs[nxt]
        nxt += 1
        stripped = s.lstrip(" ")
        nb = len(s) - len(stripped) + 1            # nonblank(string, 1)
        if not stripped or nb > len(s) - 5:
            continue
        key = s[nb - 1:]
        # READ(string, *) of the record happens only in the branches of the
        # keywords that read values (VARS, UNDEF, OPTIONS, XDEF/YDEF/ZDEF,
        # TDEF); a TITLE or DSET record is never read that way
        if _spelled(key, "ENDVARS"):
            return out
        if _spelled(key, "VARS"):
            vals, _ = _values(s)
            if len(vals) < 2:
                raise CtlError("in definition vars or variable name")
            out["nvar"] = _int(vals[1])
            out["varname"] = []
            for _ in range(out["nvar"]):
                v = ext_read(2)
                if len(v) < 2:
                    raise CtlError("in definition vars or variable name")
                _int(v[1])
                out["varname"].append(v[0])
            out["inform"] += 1
        if _spelled(key, "DSET"):
            l1 = nb + 4                           # 1-based positions, as the reference
            while l1 <= 256 and s[l1 - 1] in " ^":
                l1 += 1
            l2 = min(256, datname_len + l1 - 1)
            while l2 >= nb + 4 and s[l2 - 1] == " ":
                l2 -= 1
            if l2 < nb + 4:
                l2 -= 1
            if l1 > l2:
                raise CtlError("in definition name of file with data")
            out["datname"] = s[l1 - 1:l2]
            out["inform"] += 1
        if _spelled(key, "TITLE"):
            out["title"] = s[nb + 4:][:title_len].rstrip(" ")
            out["inform"] += 1
        if _spelled(key, "UNDEF"):
            vals, _ = _values(s)
            if len(vals) < 2:
                raise CtlError("in definition undefinit value")
            out["undef"] = _f32(_real(vals[1]))
            out["inform"] += 1
        if _spelled(key, "OPTIONS"):
            vals, _ = _values(s)
            if len(vals) < 2:
                raise CtlError("in definition Options")
            out["inform"] += 1
            if vals[1][:32][:3] == "365":
                out["yr_type"] = 0
        for tag, a in (("XDEF", "x"), ("YDEF", "y"), ("ZDEF", "z")):
            if not _spelled(key, tag):
                continue
            vals, _ = _values(s)
            if len(vals) < 3:
                raise CtlError(f"in definition {a}-grid")
            n = out["n" + a] = _int(vals[1])
            gt = vals[2][:32]
            if gt in ("linear", "LINEAR", "Linear"):
                out[a + "type"] = 0
                if len(vals) < 5:
                    raise CtlError(f"in definition {a}-grid")
                v0, h = _real(vals[3]), _real(vals[4])
                # x0(i) = x0(1) + hx*dfloat(i-1); the z axis: z0(1) + hz*dfloat(i)
                step = (lambda i: i - 1) if a != "z" else (lambda i: i)
                out[a + "0"] = [v0] + [v0 + h * float(step(i)) for i in range(2, n + 1)]
                out["h" + a] = h
                out["inform"] += 1
            elif gt in ("levels", "LEVELS", "Levels"):
                out[a + "type"] = 1
                nxt -= 1                          # BACKSPACE (40)
                v = ext_read(3 + max(n, 0))
                _int(v[1])
                out[a + "0"] = [_real(t) for t in v[3:3 + n]]
                out["h" + a] = 0.0
                out["inform"] += 1
        if _spelled(key, "TDEF"):
            vals, _ = _values(s)
            if len(vals) < 5:
                raise CtlError("in definition t-grid")
            out["nt"] = _int(vals[1])
            if vals[2][:32] in ("linear", "LINEAR", "Linear"):
                ti, st = vals[3][:32].ljust(32), vals[4][:32].ljust(32)
                l2 = len(st.rstrip(" ")) or 1
                out["hour0"], out["minute0"] = _int(ti[0:2]), _int(ti[3:5])
                out["day0"], out["year0"] = _int(ti[6:8]), _int(ti[11:15])
                for k, m in enumerate(MONTHS):
                    if ti[8:11] in (m, m.lower(), m.capitalize()):
                        out["month0"] = k + 1
                if l2 < 3:
                    raise CtlError("in definition t-grid")
                f = np.float32
                ht = f(_real(st[:l2 - 2]))
                unit = st[l2 - 2:l2]
                mult = {"yr": (365.0, 24.0, 3600.0), "mo": (30.0, 24.0, 3600.0), "dy": (24.0, 3600.0),
                        "hr": (3600.0,), "mn": (60.0,)}
                if unit not in mult:
                    out["ht"] = ht
                    raise CtlError("in definition time step for t-grid")
                for m in mult[unit]:
                    ht = f(ht * f(m))
                out["ht"] = ht
    raise CtlError("in definition undefinit value")


# ---- the ocean checkpoint (Control/output.f90:1454-1847) and its restart ------
# (Control/init_pars.f90:312-417)

# the groups of ocpwrite in its order: FP64 file, FP32 file, the name the
# descriptor is made from, mask, box start offsets (dx, dy), levels
# ("1", "nz", "nz+1"), title, variable, the pair of fields
CP_GROUPS = [
    ("cptt8.dat", "cptt.dat", "cptt.dat", "lu", 0, 0, "nz", "Potential temperature, C", "tt", ("tt", "ttp")),
    ("cpss8.dat", "cpss.dat", "cpss.dat", "lu", 0, 0, "nz", "Salinity, PSU", "ss", ("ss", "ssp")),
    ("cpuu8.dat", "cpuu.dat", "cpuu.dat", "llu", 1, 0, "nz", "Zonal velocity, m/s", "u", ("uu", "uup")),
    ("cpvv8.dat", "cpvv.dat", "cpvv.dat", "llv", 0, 1, "nz", "Meridional velocity, m/s", "v", ("vv", "vvp")),
    ("cpq28.dat", "cpq2.dat", "cpq2.dat", "lu", 0, 0, "nz+1", "turbulent kunetic energy, (m/s)^2", "q2",
     ("q2", "q2p")),
    ("cpq2l8.dat", "cpq2l.dat", "cpq2l.dat", "lu", 0, 0, "nz+1",
     "turbulent kunetic energy by length scale, (m/s)^2*m", "q2l", ("q2l", "q2lp")),
    ("cpsshi8.dat", "cpsshi.dat", "cpsshi.dat", "lu", 0, 0, "1", "Internal SSH, m", "ssh", ("ssh_i", "sshp_i")),
    ("cpsshe8.dat", "cpsshe.dat", "cpsshe.dat", "lu", 0, 0, "1", "External SSH, m", "ssh", ("ssh_e", "sshp_e")),
    ("cpube8.dat", "cpubi.dat", "cpube.dat", "llu", 1, 0, "1", "External UB, m/s", "ub", ("ubrtr_e", "ubrtrp_e")),
    ("cpvbe8.dat", "cpvbe.dat", "cpvbe.dat", "llv", 0, 1, "1", "External VB, m/s", "vb", ("vbrtr_e", "vbrtrp_e")),
]


def file_bytes(fields, lu, box, dtype):
    """The bytes of a file holding fields [(nfield, field), ...] of one box,
    written by wdstd / wdstd8 in that order."""
    chunks, size = [], 0
    for nfield, f in fields:
        for kr, rec in enumerate(records(f, lu, box, dtype), start=1):
            off = record_offset(nfield, box, kr, np.dtype(dtype).itemsize)
            chunks.append((off, rec))
            size = max(size, off + len(rec))
    buf = bytearray(size)
    for off, rec in chunks:
        buf[off:off + len(rec)] = rec
    return bytes(buf)


def _cp_box(b, dx, dy, levels):
    i0, i1 = b.mmm - b.bnd_x1 + 1, b.mm - b.bnd_x1 + 1
    j0, j1 = b.nnn - b.bnd_y1 + 1, b.nn - b.bnd_y1 + 1
    return (i0 - dx, i1, j0 - dy, j1, 1, levels)


def ocpwrite_files(path, b, nz, masks, z, zw, axes, state):
    """{file name: bytes or text} of everything ocpwrite writes for the
    pairs present in `state` (masks: dict lu/llu/llv; axes as the library's
    ocpwrite takes them)."""
    out = {}
    nx_glob, ny_glob = b.mm - b.mmm + 1, b.nn - b.nnn + 1
    date = axes.get("date", (2000, 1, 1, 0, 0))
    for f8, f4, ctl, mk, dx, dy, lev, title, var, (a, ap) in CP_GROUPS:
        if a not in state:
            continue
        L = {"1": 1, "nz": nz, "nz+1": nz + 1}[lev]
        box = _cp_box(b, dx, dy, L)
        lu = masks[mk]
        f, fp = state[a], state[ap]
        out[f8] = file_bytes([(1, f), (2, fp)], lu, box, np.float64)
        out[f4] = file_bytes([(1, f.astype(np.float32)), (2, fp.astype(np.float32))], lu, box, np.float32)
        zv = [0.0] if L == 1 else [float(v) * 1000.0 for v in (z if lev == "nz" else zw)[:L]]
        name, text = ctl_text(f"{path}/{ctl}", -1.0e32, nx_glob + dx, ny_glob + dy, L, 2, axes.get("xgr_type", 0),
                              axes["xu"] if dx else axes["xt"], axes["dxst"], axes.get("ygr_type", 0),
                              axes["yv"] if dy else axes["yt"], axes["dyst"], 0 if L == 1 else 1, zv, 1.0,
                              axes.get("calendar", 1), *date, axes.get("tstep", 86400.0), title, var)
        out[name.rsplit("/", 1)[-1]] = text
    return out


def ocpread_state(files, b, nz, masks, state, tur_var_min=1.0e-8):
    """The arrays of `state` (in place) after the restart reads of
    Control/init_pars.f90:312-417 from files {name: bytes}: rdstd8 (land of
    the box 0), the wraps (cyclize8_y of q2/q2l over nz levels), the
    tur_var_min floor of q2, q2p, q2l, q2lp."""
    for f8, _, _, mk, dx, dy, lev, _, _, pair in CP_GROUPS:
        if pair[0] not in state:
            continue
        L = {"1": 1, "nz": nz, "nz+1": nz + 1}[lev]
        box = _cp_box(b, dx, dy, L)
        for nfield, name in enumerate(pair, start=1):
            f = state[name]
            read_field(files[f8], nfield, box, np.float64, masks[mk], f)
            g = f if f.ndim == 3 else f[:, :, None]
            i0, i1 = b.mmm - b.bnd_x1, b.mm - b.bnd_x1
            j0, j1 = b.nnn - b.bnd_y1, b.nn - b.bnd_y1
            ly = nz if lev == "nz+1" else L
            if b.periodicity_x:
                g[i0 - 1, :, :L], g[i1 + 1, :, :L] = g[i1, :, :L].copy(), g[i0, :, :L].copy()
            if b.periodicity_y:
                g[:, j0 - 1, :ly], g[:, j1 + 1, :ly] = g[:, j1, :ly].copy(), g[:, j0, :ly].copy()
    for name in ("q2", "q2p", "q2l", "q2lp"):
        if name in state:
            np.maximum(state[name], tur_var_min, out=state[name])
    return state
