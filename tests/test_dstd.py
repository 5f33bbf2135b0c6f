"""On-disk formats: the DIOGIN-standard direct-access files and GrADS
descriptors of the reference (Service/input_output_data.f90:117-534,
Service/rw_ctl_file.f90:1-596) through the C ABI, against the oracle's
restatements (oracle/dstd_oracle.py): the files byte for byte (the MPI-IO
forms prdstd/pwdstd through several ranks, gloo processes included), the
descriptor reader's outputs value for value; the barotropic
checkpoint and restart (Control/output.f90:1736-1847,
Control/init_pars.f90:384-411) on the GPU.
"""
import numpy as np
import pytest

from inmsom_elfs_b200 import dstd
from inmsom_elfs_b200._lib import InmsomError
from oracle import dstd_oracle as od


def _case(seed=0, nx=13, ny=9, nz=4):
    rng = np.random.default_rng(seed)
    field = np.asfortranarray(rng.standard_normal((nx, ny, nz)))
    lu = np.asfortranarray((rng.random((nx, ny)) > 0.3).astype(np.float32))
    lu[0, 0] = -1.0                       # |lu| >= 0.5 is ocean
    return field, lu


def _expected_file(fields, lu, box, dtype):
    size = 0
    chunks = []
    for nfield, f in fields:
        for kr, rec in enumerate(od.records(f, lu, box, dtype), start=1):
            off = od.record_offset(nfield, box, kr, np.dtype(dtype).itemsize)
            chunks.append((off, rec))
            size = max(size, off + len(rec))
    buf = bytearray(size)
    for off, rec in chunks:
        buf[off:off + len(rec)] = rec
    return bytes(buf)


@pytest.mark.parametrize("kind", ["8", "4"])
def test_write_records_match_oracle(tmp_path, kind):
    dtype = np.float64 if kind == "8" else np.float32
    write = dstd.wdstd8 if kind == "8" else dstd.wdstd
    f1, lu = _case(1)
    f2, _ = _case(2)
    f1, f2 = f1.astype(dtype, order="F"), f2.astype(dtype, order="F")
    box = (2, 12, 3, 8, 2, 4)
    want = _expected_file([(1, f1), (2, f2)], lu, box, dtype)
    g1, g2 = f1.copy(order="F"), f2.copy(order="F")
    write(str(tmp_path), "cpx.dat", 1, g1, lu, box)
    write(str(tmp_path), "cpx.dat", 2, g2, lu, box)
    assert (tmp_path / "cpx.dat").read_bytes() == want
    # the reference leaves the written land points of the field at zero
    land = np.zeros(f1.shape, bool)
    land[1:12, 2:8, 1:4] = (np.abs(lu[1:12, 2:8]) < 0.5)[..., None]
    assert np.all(g1[land] == 0) and np.array_equal(g1[~land], f1[~land])


def test_undef_value_and_record_length(tmp_path):
    f, lu = _case(3, nx=6, ny=5, nz=1)
    lu[:] = 0.0
    dstd.wdstd8(str(tmp_path), "u8.dat", 1, f.copy(order="F"), lu)
    data = np.frombuffer((tmp_path / "u8.dat").read_bytes(), dtype=np.float64)
    assert data.size == 30 and np.all(data == np.float64(np.float32(-1.0e32)))
    dstd.wdstd(str(tmp_path), "u4.dat", 1, f.astype(np.float32, order="F"), lu)
    data = np.frombuffer((tmp_path / "u4.dat").read_bytes(), dtype=np.float32)
    assert data.size == 30 and np.all(data == np.float32(-1.0e32))


@pytest.mark.parametrize("kind", ["8", "4"])
def test_read_matches_oracle(tmp_path, kind):
    dtype = np.float64 if kind == "8" else np.float32
    write, read = (dstd.wdstd8, dstd.rdstd8) if kind == "8" else (dstd.wdstd, dstd.rdstd)
    f, lu = _case(4)
    f = f.astype(dtype, order="F")
    box = (1, 13, 2, 9, 1, 3)
    write(str(tmp_path), "r.dat", 2, f.copy(order="F"), lu, box)
    got = np.full(f.shape, np.nan, dtype=dtype, order="F")
    read(str(tmp_path), "r.dat", 2, got, lu, box)
    want = od.read_field((tmp_path / "r.dat").read_bytes(), 2, box, dtype, lu,
                         np.full(f.shape, np.nan, dtype=dtype, order="F"))
    assert np.array_equal(got, want, equal_nan=True)
    inbox = np.zeros(f.shape, bool)
    inbox[:, 1:9, 0:3] = True
    ocean = (np.abs(lu) >= 0.5)[..., None] & inbox
    assert np.array_equal(got[ocean], f[ocean])
    assert np.all(got[inbox & ~ocean] == 0) and np.all(np.isnan(got[~inbox]))


def test_existing_file_is_not_truncated(tmp_path):
    p = tmp_path / "keep.dat"
    p.write_bytes(b"\xab" * 4096)
    f, lu = _case(5, nx=4, ny=3, nz=1)
    dstd.wdstd8(str(tmp_path), "keep.dat", 1, f.copy(order="F"), lu)
    data = p.read_bytes()
    assert len(data) == 4096 and data[96:] == b"\xab" * (4096 - 96)


def test_path_joining_and_errors(tmp_path):
    f, lu = _case(6, nx=4, ny=3, nz=1)
    dstd.wdstd8(f"  {tmp_path}/  ", "  j.dat  ", 1, f.copy(order="F"), lu)     # blanks around, one '/'
    assert (tmp_path / "j.dat").exists()
    with pytest.raises(InmsomError) as e:
        dstd.wdstd8(str(tmp_path), "j.dat", 1, f.copy(order="F"), lu, (0, 4, 1, 3, 1, 1))
    assert e.value.code == 2
    with pytest.raises(InmsomError) as e:
        dstd.rdstd8(str(tmp_path), "missing.dat", 1, f.copy(order="F"), lu)
    assert e.value.code == 6


CTL_CASES = [
    dict(nx=256, ny=256, nz=1, nt=2, xtype=0, x0=[27.5], hx=0.5, ytype=0, y0=[40.9], hy=0.25, ztype=0, z0=[0.0],
         hz=1.0, yr_type=1, date=(2000, 1, 1, 0, 0), ht=86400.0, title="External SSH, m", var="ssh"),
    dict(nx=9, ny=3, nz=20, nt=12, xtype=1, x0=list(np.linspace(-1500.0, 1.0e9, 9)), hx=0.0, ytype=1,
         y0=[0.001, 0.05, 123456789.0], hy=0.0, ztype=1, z0=list(np.linspace(2.5, 997.5, 20)), hz=1.0,
         yr_type=0, date=(1957, 12, 31, 23, 59), ht=6 * 3600.0, title="Potential temperature, C", var="tt"),
    dict(nx=2049, ny=1537, nz=1, nt=1, xtype=0, x0=[-0.5], hx=1000.0, ytype=0, y0=[0.0], hy=1.0e-9, ztype=0,
         z0=[0.0], hz=1.0, yr_type=1, date=(2024, 6, 15, 12, 30), ht=30.0 * 86400.0, title="External UB, m/s",
         var="ub"),
    dict(nx=4, ny=4, nz=1, nt=3, xtype=0, x0=[1.0], hx=1.0, ytype=0, y0=[1.0], hy=1.0, ztype=0, z0=[0.0], hz=1.0,
         yr_type=1, date=(1, 2, 3, 4, 5), ht=90.0, title="t", var="v"),
    # a step under a minute: no unit, k left from the file-name search
    dict(nx=4, ny=4, nz=1, nt=3, xtype=0, x0=[1.0], hx=1.0, ytype=0, y0=[1.0], hy=1.0, ztype=0, z0=[0.0], hz=1.0,
         yr_type=1, date=(1, 2, 3, 4, 5), ht=30.0, title="t", var="v"),
]


@pytest.mark.parametrize("case", range(len(CTL_CASES)))
def test_ctl_file_matches_oracle(tmp_path, case):
    c = CTL_CASES[case]
    fname = str(tmp_path / "cpsshe.dat")
    args = (fname, -1.0e32, c["nx"], c["ny"], c["nz"], c["nt"], c["xtype"], c["x0"], c["hx"], c["ytype"], c["y0"],
            c["hy"], c["ztype"], c["z0"], c["hz"], c["yr_type"], *c["date"][:1], c["date"][1], c["date"][2],
            c["date"][3], c["date"][4], c["ht"], c["title"], c["var"])
    dstd.ctl_file_write(*args)
    name, text = od.ctl_text(*args)
    assert name == str(tmp_path / "cpsshe.ctl")
    assert (tmp_path / "cpsshe.ctl").read_text() == text


def test_ctl_lines_by_hand(tmp_path):
    """A few lines worked out from the edit descriptors by hand."""
    c = CTL_CASES[0]
    dstd.ctl_file_write(str(tmp_path / "a.dat"), -1.0e32, 256, 256, 1, 2, 0, [27.5], 0.5, 0, [40.9], 0.25, 0, [0.0],
                        1.0, 1, 2000, 1, 1, 0, 0, 86400.0, c["title"], "ssh")
    lines = (tmp_path / "a.ctl").read_text().split("\n")
    assert lines[0] == "DSET    ^a.dat" + " " * 123
    assert lines[1] == "TITLE    External SSH, m"
    assert lines[2] == "UNDEF   -0.10000E+33  ! gap value"
    # a6 i6 a11, g15.8 (F11.6 + 4 blanks), 5x, g15.8 (F11.8 + 4 blanks); the
    # final 5x writes nothing
    assert lines[3] == "XDEF  " + "   256" + "  LINEAR   " + "  27.500000" + " " * 9 + " 0.50000000" + " " * 4
    # g15.8 of zero: F11.7 + 4 blanks
    assert lines[5] == "ZDEF  " + "     1" + "  LINEAR   " + "  0.0000000" + " " * 9 + "  1.0000000" + " " * 4
    assert lines[6] == "TDEF       2  LINEAR  00:00Z01JAN2000        1dy"
    assert lines[7:11] == ["VARS 1  ! Number of variables", "ssh" + " " * 8 + "    1" + "  1 VARIABLES ", "ENDVARS", ""]


# ---- the barotropic checkpoint on the GPU -----------------------------------

@pytest.mark.gpu
def test_checkpoint_restart_continues_bit_for_bit(gpu, tmp_path):
    from inmsom_elfs_b200 import basins
    from oracle import oracle as ora
    b = basins.regional_basin(nx=150, ny=110, seed=12)
    basins.finalize(b, ora.OracleBackend())
    fresh = b.copy()
    ax = dict(xt=[0.5], xu=[0.0], yt=[0.5], yv=[0.0], dxst=1.0, dyst=1.0)
    with gpu.BarotropicSolver(b, resident=True) as s:
        s.load_state()
        s.run_substeps(40, b.dt)
        s.write_checkpoint(str(tmp_path), **ax)
        s.sync_to_host(0x1)
        saved = {k: v.copy(order="F") for k, v in b.state.items()}
        s.run_substeps(30, b.dt)
        s.sync_to_host(0x1)
        cont = {k: v.copy(order="F") for k, v in b.state.items()}
    B = b.bounds
    box = (B.mmm - B.bnd_x1 + 1, B.mm - B.bnd_x1 + 1, B.nnn - B.bnd_y1 + 1, B.nn - B.bnd_y1 + 1, 1, 1)
    for name, k0, k1, mask, dx, dy in (("cpsshe8.dat", "ssh_e", "sshp_e", "lu", 0, 0),
                                       ("cpube8.dat", "ubrtr_e", "ubrtrp_e", "llu", 1, 0),
                                       ("cpvbe8.dat", "vbrtr_e", "vbrtrp_e", "llv", 0, 1)):
        bx = (box[0] - dx, box[1], box[2] - dy, box[3], 1, 1)
        want = _expected_file([(1, saved[k0]), (2, saved[k1])], b.masks[mask], bx, np.float64)
        assert (tmp_path / name).read_bytes() == want, name
    for name in ("cpsshe.dat", "cpubi.dat", "cpvbe.dat", "cpsshe.ctl", "cpube.ctl", "cpvbe.ctl"):
        assert (tmp_path / name).exists(), name
    with gpu.BarotropicSolver(fresh, resident=True) as s:
        s.load_state()
        s.read_checkpoint(str(tmp_path))
        for k in saved:
            assert np.array_equal(fresh.state[k], saved[k]), k
        s.run_substeps(30, b.dt)
        s.sync_to_host(0x1)
    for k in cont:
        assert np.array_equal(fresh.state[k], cont[k]), k


def test_format_error_codes(tmp_path):
    c = CTL_CASES[0]
    with pytest.raises(InmsomError) as e:
        dstd.ctl_file_write(str(tmp_path / "a.dat"), -1.0e32, 4, 4, 1, 1, 0, [0.0], 1.0, 0, [0.0], 1.0, 0, [0.0], 1.0,
                            1, 2000, 13, 1, 0, 0, 86400.0, c["title"], "ssh")
    assert e.value.code == 2
    f, lu = _case(7, nx=4, ny=3, nz=2)
    (tmp_path / "short.dat").write_bytes(b"\0" * 40)          # less than one 96-byte record
    with pytest.raises(InmsomError) as e:
        dstd.rdstd8(str(tmp_path), "short.dat", 1, f.copy(order="F"), lu)
    assert e.value.code == 6
    with pytest.raises(InmsomError) as e:
        dstd.wdstd8(str(tmp_path / "no" / "such" / "dir"), "x.dat", 1, f.copy(order="F"), lu)
    assert e.value.code == 6


def test_ctl_number_editing_edge_cases(tmp_path):
    """G15.8 editing of values at the F/E boundaries (rounding that changes
    the decade, tiny and huge exponents, negative zero) and random values,
    through a LEVELS axis: the library's text equals the restatement's."""
    rng = np.random.default_rng(3)
    edge = [0.0, -0.0, 1.0, -1.0, 0.1, 0.099999999, 0.0999999999, 9.999999994, 9.999999995, 99999999.4,
            99999999.5, 1.0e8, 123456789.0, 1.0e-100, -1.0e-100, 1.0e100, 3.0e-5, 0.5, 27.5, -1500.0,
            np.nextafter(0.1, 0.0), np.nextafter(1.0e8, 0.0)]
    vals = edge + list(10.0 ** rng.uniform(-12, 12, 60) * rng.choice([-1.0, 1.0], 60))
    n = len(vals)
    args = (str(tmp_path / "g.dat"), -1.0e32, n, 1, 1, 1, 1, vals, 0.0, 0, [0.0], 1.0, 0, [0.0], 1.0, 1, 2000, 1, 1,
            0, 0, 86400.0, "t", "v")
    dstd.ctl_file_write(*args)
    _, text = od.ctl_text(*args)
    assert (tmp_path / "g.ctl").read_text() == text
    # worked out by hand: G15.8 of 99999999.4 is F11.0 (the point kept) and 4 blanks
    assert od.edit_g(99999999.4, 15, 8) == "  99999999.    "
    assert od.edit_g(9.999999995, 15, 8) == "  10.000000    "
    assert od.edit_g(1.0e100, 15, 8) == " 0.10000000+101"


# ---- the descriptor reader (Service/rw_ctl_file.f90:185-566) -----------------

def _read_both(tmp_path, text, name="d.ctl", **kw):
    """The library's ctl_file_read and the oracle's on the same text: both
    fail or both give the same outputs (exactly).  Returns the library's."""
    p = tmp_path / name
    p.write_text(text)
    try:
        want = od.ctl_read(text)
    except od.CtlError:
        with pytest.raises(InmsomError) as e:
            dstd.ctl_file_read(p, **kw)
        assert e.value.code == 2
        return None
    got = dstd.ctl_file_read(p, **kw)
    for k, v in want.items():
        if k in ("x0", "y0", "z0"):
            assert np.array_equal(got[k][:len(v)], np.asarray(v, dtype=np.float64)), k
        elif k == "undef":
            assert np.float32(got[k]) == np.float32(v), k
        else:
            assert got[k] == v, (k, got[k], v)
    return got


@pytest.mark.parametrize("case", range(len(CTL_CASES)))
def test_ctl_read_round_trip(tmp_path, case):
    """What ctl_file_write writes, ctl_file_read reads back: the axes to the
    eight significant digits of G15.8, the calendar, the step in the unit
    the writer chose."""
    c = CTL_CASES[case]
    fname = str(tmp_path / "cpsshe.dat")
    y, mo, d, h, mn = c["date"]
    dstd.ctl_file_write(fname, -1.0e32, c["nx"], c["ny"], c["nz"], c["nt"], c["xtype"], c["x0"], c["hx"],
                        c["ytype"], c["y0"], c["hy"], c["ztype"], c["z0"], c["hz"], c["yr_type"], y, mo, d, h, mn,
                        c["ht"], c["title"], c["var"])
    text = (tmp_path / "cpsshe.ctl").read_text()
    got = _read_both(tmp_path, text, name="cpsshe.ctl")
    if c["ht"] < 60.0:
        assert got is None       # a step under a minute has no unit to read back
        return
    assert got["inform"] == 8 - (c["yr_type"] == 1)
    assert got["datname"] == "cpsshe.dat" and got["title"] == "    " + c["title"]
    assert got["undef"] == np.float32(-1.0e32)
    for a, n in (("x", c["nx"]), ("y", c["ny"]), ("z", c["nz"])):
        assert got["n" + a] == n and got[a + "type"] == c[a + "type"]
        if c[a + "type"] == 1:
            np.testing.assert_allclose(got[a + "0"], c[a + "0"], rtol=5e-8, atol=1e-300)
        else:
            np.testing.assert_allclose(got[a + "0"][0], c[a + "0"][0], rtol=5e-8)
            np.testing.assert_allclose(got["h" + a], c["h" + a], rtol=5e-8)
    assert got["nt"] == c["nt"] and got["yr_type"] == c["yr_type"]
    assert (got["year0"], got["month0"], got["day0"], got["hour0"], got["minute0"]) == c["date"]
    assert got["nvar"] == 1 and got["varname"] == [c["var"]]
    want_ht = {86400.0: 86400.0, 6 * 3600.0: 21600.0, 30 * 86400.0: 2592000.0, 90.0: 60.0}[c["ht"]]
    assert got["ht"] == np.float32(want_ht)


HAND_CTL = """dset ^../data/run 1/temp.dat
title   Model   output
undef -9.99e8
options 365_day_calendar
xdef 10 linear 0 1.5
Ydef 3 levels
  -10.0, 0.0 10.0
zdef 4 LINEAR 1.0 2.0
tdef 24 linear 12:30z15jul1999 3hr
VARS 2
t  4  99 temperature
'sal inity'  4  99 salinity
ENDVARS
"""


def test_ctl_read_by_hand(tmp_path):
    """A descriptor in lower and capitalised keywords, worked out by hand:
    the DSET name after '^' with its inner blank, TITLE from the fifth
    character after the keyword, the LEVELS values on the next line, the
    z axis filled as z0(1) + hz*i, the month in lower case."""
    got = _read_both(tmp_path, HAND_CTL)
    assert got["datname"] == "../data/run 1/temp.dat"
    assert got["title"] == "   Model   output"
    assert got["undef"] == np.float32(-9.99e8) and got["yr_type"] == 0
    assert got["nx"] == 10 and got["xtype"] == 0 and np.array_equal(got["x0"], 1.5 * np.arange(10))
    assert got["ytype"] == 1 and np.array_equal(got["y0"], [-10.0, 0.0, 10.0]) and got["hy"] == 0.0
    assert got["ztype"] == 0 and np.array_equal(got["z0"], [1.0, 5.0, 7.0, 9.0])
    assert (got["nt"], got["hour0"], got["minute0"], got["day0"], got["month0"], got["year0"]) == \
        (24, 12, 30, 15, 7, 1999)
    assert got["ht"] == np.float32(10800.0)
    assert got["nvar"] == 2 and got["varname"] == ["t", "sal inity"] and got["inform"] == 8


@pytest.mark.parametrize("text, check", [
    # the step units in single precision
    ("TDEF 1 LINEAR 00:00Z01JAN2000 2yr\nENDVARS\n", lambda g: g["ht"] == np.float32(2 * 365 * 86400.0)),
    ("TDEF 1 LINEAR 00:00Z01Feb2000 1mo\nENDVARS\n", lambda g: g["ht"] == np.float32(2592000.0) and g["month0"] == 2),
    ("TDEF 1 LINEAR 00:00Z01DEC2000 0.1dy\nENDVARS\n",
     lambda g: g["ht"] == np.float32(np.float32(np.float32(0.1) * np.float32(24.0)) * np.float32(3600.0))),
    ("TDEF 1 LINEAR 00:00Z01DEC2000 45mn\nENDVARS\n", lambda g: g["ht"] == np.float32(2700.0)),
    # TDEF is not counted in inform; a non-linear time axis leaves the calendar unread
    ("TDEF 5 levels 1 2\nENDVARS\n", lambda g: g["nt"] == 5 and g["inform"] == 0 and g["ht"] == 0),
    # Fortran real forms: a D exponent, a signed exponent with no letter, r*c repeats
    ("UNDEF -1.0D+30\nXDEF 3 LEVELS 0.1+101 1.5-3 2*7\nENDVARS\n",
     lambda g: g["undef"] == np.float32(-1.0e30) and list(g["x0"]) == [1.0e100, 1.5e-3, 7.0]),
    ("ZDEF 4 LEVELS 4*2.5\nENDVARS\n", lambda g: list(g["z0"]) == [2.5] * 4),
    # a slash ends the LEVELS read: the values it did not reach stay as they were
    ("XDEF 5 LEVELS 1 2 3 /\nENDVARS\n", lambda g: list(g["x0"]) == [1.0, 2.0, 3.0, 0.0, 0.0]),
    # keywords in other spellings are not keywords
    ("xDef 4 LINEAR 0 1\nENDVARS\n", lambda g: g["nx"] == 0 and g["inform"] == 0),
    # nonblank: a first non-blank past column 251 makes the record blank
    (" " * 251 + "UNDEF\nENDVARS\n", lambda g: g["inform"] == 0),
    # blank lines and '^' runs before the name
    ("\n\n   DSET  ^^ ^a.dat   \nENDVARS\n", lambda g: g["datname"] == "a.dat" and g["inform"] == 1),
    # OPTIONS other than 365... keep the leap-year calendar but count
    ("OPTIONS template\nENDVARS\n", lambda g: g["yr_type"] == 1 and g["inform"] == 1),
    # ENDVARS in its three spellings ends the read; later lines are not read
    ("Endvars\nUNDEF 5\n", lambda g: g["inform"] == 0 and g["undef"] == 0),
])
def test_ctl_read_rules(tmp_path, text, check):
    got = _read_both(tmp_path, text)
    assert got is not None and check(got)


@pytest.mark.parametrize("text", [
    "UNDEF 5\n",                                          # end of file before ENDVARS
    " " * 250 + "UNDEF\nENDVARS\n",                       # column 251 is read: no value
    "TDEF 1 LINEAR 00:00Z01JAN2000 3wk\nENDVARS\n",       # no such unit
    "TDEF 1 LINEAR 00:00Z01JAN2000 hr\nENDVARS\n",        # no count before the unit
    "XDEF 3 LEVELS 1 2\n",                                # LEVELS runs into the end of file
    "VARS 2\nt 1\nENDVARS\n",                             # the second name takes ENDVARS; the file ends before its integer
    "DSET ^^^\nENDVARS\n",                                # no name
    "XDEF 3 LINEAR 1,,2\nENDVARS\n",                      # a null value
    "\n" * 512 + "ENDVARS\n",                             # 512 records without ENDVARS
])
def test_ctl_read_errors(tmp_path, text):
    assert _read_both(tmp_path, text) is None


def test_ctl_read_limits(tmp_path):
    # 511 blank records and ENDVARS are within the 512 the reference reads
    assert _read_both(tmp_path, "\n" * 511 + "ENDVARS\n")["inform"] == 0
    # the unit's value is kept when the unit is unknown (the reference sets
    # ht before it checks the unit); a name is cut to its variable's length
    (tmp_path / "n.ctl").write_text("DSET abcdefghij\nENDVARS\n")
    assert dstd.ctl_file_read(tmp_path / "n.ctl", name_len=8)["datname"] == "abcdefg"
    (tmp_path / "n.ctl").write_text("XDEF 9 LEVELS 1 2 3 4 5 6 7 8 9\nENDVARS\n")
    with pytest.raises(InmsomError) as e:
        dstd.ctl_file_read(tmp_path / "n.ctl", x_cap=8)
    assert e.value.code == 2
    with pytest.raises(InmsomError) as e:
        dstd.ctl_file_read(tmp_path / "missing.ctl")
    assert e.value.code == 6


# ---- the MPI-IO forms (Service/input_output_data.f90:535-819) ----------------

def _rank_grid(g, xs, ys):
    """Local bounds of a process grid: interior x ranges xs, y ranges ys
    (global indices), arrays with the two-point halo."""
    from dataclasses import replace
    return [replace(g, nx_start=a, nx_end=b, ny_start=c, ny_end=d, bnd_x1=a - 2, bnd_x2=b + 2, bnd_y1=c - 2,
                    bnd_y2=d + 2) for (c, d) in ys for (a, b) in xs]


def _local(a, g, lb):
    return np.asfortranarray(a[lb.bnd_x1 - g.bnd_x1:lb.bnd_x2 - g.bnd_x1 + 1,
                               lb.bnd_y1 - g.bnd_y1:lb.bnd_y2 - g.bnd_y1 + 1].copy())


def _pglobal(seed=11, nz=3):
    from inmsom_elfs_b200.grid import Bounds
    g = Bounds.serial(11, 9)
    f, lu = _case(seed, nx=g.shape[0], ny=g.shape[1], nz=nz)
    return g, np.asfortranarray(f.astype(np.float32)), lu


def test_pwdstd_ranks_write_the_wdstd_file(tmp_path):
    """Four ranks of a 2 x 2 process grid (uneven parts) write fields 1 and
    2, levels 2..3, of the global interior: the file is byte for byte the
    one wdstd writes for the global field, the ranks' land points are undef
    in their arrays and nothing outside their interiors changes."""
    g, f1, lu = _pglobal(11)
    _, f2, _ = _pglobal(12)
    nx, ny, nz = f1.shape
    box = (g.mmm, g.mm, g.nnn, g.nn, 2, 3)
    ranks = _rank_grid(g, [(3, 7), (8, 13)], [(3, 6), (7, 11)])
    for nfild, f in ((2, f2), (1, f1)):             # the ranks and fields in any order
        for lb in reversed(ranks):
            loc = _local(f, g, lb)
            before = loc.copy()
            dstd.pwdstd(lb, str(tmp_path), "p.dat", nfild, loc, _local(lu, g, lb), nx, ny, nz, box)
            inner = np.zeros(loc.shape, bool)
            inner[2:-2, 2:-2, 1:3] = True
            land = inner & (np.abs(_local(lu, g, lb)) < 0.5)[..., None]
            assert np.all(loc[land] == od.UNDEF) and np.array_equal(loc[~land], before[~land])
    assert (tmp_path / "p.dat").read_bytes() == _expected_file([(1, f1), (2, f2)], lu, box, np.float32)


def test_prdstd_reads_each_rank_part(tmp_path):
    """prdstd of each rank gives its interior of the wdstd file (undef at
    land, not 0 as rdstd gives) and leaves the rest of its array alone;
    values past the end of a short file stay as they were."""
    g, f, lu = _pglobal(13)
    nx, ny, nz = f.shape
    box = (g.mmm, g.mm, g.nnn, g.nn, 1, 3)
    dstd.wdstd(str(tmp_path), "w.dat", 1, f.copy(order="F"), lu, box)
    want = f.copy(order="F")
    want[np.broadcast_to((np.abs(lu) < 0.5)[..., None], want.shape)] = od.UNDEF
    for lb in _rank_grid(g, [(3, 13)], [(3, 4), (5, 11)]) + _rank_grid(g, [(3, 9), (10, 13)], [(3, 11)]):
        loc = np.full(lb.shape + (nz,), 7.0, np.float32, order="F")
        dstd.prdstd(lb, str(tmp_path), "w.dat", 1, loc, _local(lu, g, lb), nx, ny, nz, box)
        exp = np.full_like(loc, 7.0)
        exp[2:-2, 2:-2, :] = _local(want, g, lb)[2:-2, 2:-2, :]
        assert np.array_equal(loc, exp)
    # a file that ends inside level 2 of the top strip
    data = (tmp_path / "w.dat").read_bytes()
    bx, by = g.mm - g.mmm + 1, g.nn - g.nnn + 1
    cut = 4 * (bx * by + bx * 7 + 3)                  # level 2, row 8 of the box, three values in
    (tmp_path / "s.dat").write_bytes(data[:cut])
    lb = _rank_grid(g, [(3, 13)], [(5, 11)])[0]
    loc = np.full(lb.shape + (nz,), 7.0, np.float32, order="F")
    dstd.prdstd(lb, str(tmp_path), "s.dat", 1, loc, _local(lu, g, lb), nx, ny, nz, box)
    w = _local(want, g, lb)
    assert np.array_equal(loc[2:-2, 2:-2, 0], w[2:-2, 2:-2, 0])
    lvl2 = loc[2:-2, 2:-2, 1]                          # box rows 3..9 of this strip; row 8 is local row 5
    assert np.array_equal(lvl2[:, :5], w[2:-2, 2:7, 1])
    assert np.array_equal(lvl2[:3, 5], w[2:5, 7, 1]) and np.all(lvl2[3:, 5] == 7.0) and np.all(lvl2[:, 6:] == 7.0)
    assert np.all(loc[2:-2, 2:-2, 2] == 7.0)


def test_parallel_forms_errors(tmp_path):
    g, f, lu = _pglobal(14)
    nx, ny, nz = f.shape
    lb = _rank_grid(g, [(3, 13)], [(3, 11)])[0]
    loc = _local(f, g, lb)
    for box in [(4, 13, 3, 11, 1, 1),                 # the interior starts before the box
                (3, 12, 3, 11, 1, 1),                 # ... and ends after it
                (3, nx + 1, 3, 11, 1, 1),             # the box leaves the global field
                (3, 13, 3, 11, 2, 1)]:
        with pytest.raises(InmsomError) as e:
            dstd.pwdstd(lb, str(tmp_path), "e.dat", 1, loc.copy(order="F"), _local(lu, g, lb), nx, ny, nz, box)
        assert e.value.code == 2
    with pytest.raises(InmsomError) as e:
        dstd.pwdstd(lb, str(tmp_path), "  ", 1, loc.copy(order="F"), _local(lu, g, lb), nx, ny, nz,
                    (3, 13, 3, 11, 1, 1))
    assert e.value.code == 2
    with pytest.raises(InmsomError) as e:
        dstd.prdstd(lb, str(tmp_path), "none.dat", 1, loc, _local(lu, g, lb), nx, ny, nz, (3, 13, 3, 11, 1, 1))
    assert e.value.code == 6
    assert not (tmp_path / "e.dat").exists()


def _pw_rank(rank, world, port, path, q):
    import os
    import torch.distributed as dist
    from inmsom_elfs_b200.strips import strip_bounds
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, f, lu = _pglobal(15)
        nx, ny, nz = f.shape
        lb = strip_bounds(g, world)[rank]
        box = (g.mmm, g.mm, g.nnn, g.nn, 1, nz)
        dstd.pwdstd(lb, path, "cp.dat", 3, _local(f, g, lb), _local(lu, g, lb), nx, ny, nz, box)
        dist.barrier()
        loc = np.zeros(lb.shape + (nz,), np.float32, order="F")
        dstd.prdstd(lb, path, "cp.dat", 3, loc, _local(lu, g, lb), nx, ny, nz, box)
        q.put((rank, loc[2:-2, 2:-2].copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_pwdstd_gloo_ranks(tmp_path, world):
    """One process per strip (gloo ranks): each writes its strip of field 3
    with no collective on the data, then reads it back; the file is the
    wdstd file of the global field."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_pw_rank, args=(r, world, port, str(tmp_path), q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g, f, lu = _pglobal(15)
    box = (g.mmm, g.mm, g.nnn, g.nn, 1, f.shape[2])
    want = _expected_file([(3, f)], lu, box, np.float32)
    assert (tmp_path / "cp.dat").read_bytes() == want
    from inmsom_elfs_b200.strips import strip_bounds
    full = f.copy(order="F")
    full[np.broadcast_to((np.abs(lu) < 0.5)[..., None], full.shape)] = od.UNDEF
    for r, lb in enumerate(strip_bounds(g, world)):
        assert np.array_equal(got[r], _local(full, g, lb)[2:-2, 2:-2])


# ---- the whole checkpoint from host arrays (Control/output.f90:1454-1847) ----

def _ocean(seed, b, nz):
    rng = np.random.default_rng(seed)
    sh = b.shape
    st = {}
    for name in ("tt", "ttp", "ss", "ssp", "uu", "uup", "vv", "vvp"):
        st[name] = np.asfortranarray(rng.standard_normal(sh + (nz,)))
    for name in ("q2", "q2p", "q2l", "q2lp"):
        st[name] = np.asfortranarray(rng.standard_normal(sh + (nz + 1,)) * 1e-6)   # some below tur_var_min
    for name in ("ssh_i", "sshp_i", "ssh_e", "sshp_e", "ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e"):
        st[name] = np.asfortranarray(rng.standard_normal(sh))
    masks = {k: np.asfortranarray((rng.random(sh) > 0.35).astype(np.float32)) for k in ("lu", "llu", "llv")}
    return st, masks


AXES = dict(xt=[27.5], xu=[27.25], yt=[40.9], yv=[40.775], dxst=0.5, dyst=0.25, calendar=0,
            date=(2001, 7, 15, 6, 0), tstep=21600.0)


@pytest.mark.parametrize("px, py", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_ocean_checkpoint_files_and_restart(tmp_path, px, py):
    """ocpwrite from host arrays writes the reference's 30 files (FP64, FP32
    and descriptor of ten pairs) byte for byte as the restatement does, and
    zeroes the written land points of its arrays; ocpread brings back what
    the restart reads give (land 0, the wraps, the q2 floor)."""
    from inmsom_elfs_b200.grid import Bounds
    b = Bounds.serial(10, 7, px, py)
    nz = 4
    st, masks = _ocean(21 + 2 * px + py, b, nz)
    z = np.linspace(0.005, 0.9, nz)
    zw = np.linspace(0.0, 1.0, nz + 1)
    mine = {k: v.copy(order="F") for k, v in st.items()}
    dstd.ocpwrite(str(tmp_path), b, nz, masks["lu"], masks["llu"], masks["llv"], z, zw, AXES, mine)
    want = od.ocpwrite_files(str(tmp_path), b, nz, masks, z, zw, AXES, st)
    assert len(want) == 30 and sorted(p.name for p in tmp_path.iterdir()) == sorted(want)
    for name, content in want.items():
        got = (tmp_path / name).read_bytes()
        assert got == (content.encode() if isinstance(content, str) else content), name
    # the written boxes' land points are 0 in the caller's arrays, the rest untouched
    for f8, _, _, mk, dx, dy, lev, _, _, pair in od.CP_GROUPS:
        box = od._cp_box(b, dx, dy, 1)
        land = np.zeros(b.shape, bool)
        land[box[0] - 1:box[1], box[2] - 1:box[3]] = np.abs(masks[mk][box[0] - 1:box[1], box[2] - 1:box[3]]) < 0.5
        for name in pair:
            m = land if mine[name].ndim == 2 else land[..., None] & np.ones(mine[name].shape, bool)
            assert np.all(mine[name][m] == 0) and np.array_equal(mine[name][~m], st[name][~m]), name
    # the restart, into arrays that hold something else
    rng = np.random.default_rng(99)
    old = {k: np.asfortranarray(rng.standard_normal(v.shape)) for k, v in st.items()}
    got = {k: v.copy(order="F") for k, v in old.items()}
    dstd.ocpread(str(tmp_path), b, nz, masks["lu"], masks["llu"], masks["llv"], got)
    files = {f8: (tmp_path / f8).read_bytes() for f8, *_ in od.CP_GROUPS}
    exp = od.ocpread_state(files, b, nz, masks, {k: v.copy(order="F") for k, v in old.items()})
    for k in st:
        assert np.array_equal(got[k], exp[k]), k
    # the interior ocean values come back exactly
    i, j = b.interior
    ocean = np.abs(masks["lu"][i, j]) >= 0.5
    assert np.array_equal(got["tt"][i, j][ocean], st["tt"][i, j][ocean])
    assert np.all(got["q2"] >= 1.0e-8)


def test_ocean_checkpoint_pairs_and_errors(tmp_path):
    """Only the pairs given are written (a barotropic-only state writes the
    same three groups as the context's checkpoint); half a pair, a missing
    z or an unreadable file is an error."""
    from inmsom_elfs_b200.grid import Bounds
    b = Bounds.serial(6, 5)
    st, masks = _ocean(5, b, 2)
    baro = {k: st[k] for k in ("ssh_e", "sshp_e", "ubrtr_e", "ubrtrp_e", "vbrtr_e", "vbrtrp_e")}
    dstd.ocpwrite(str(tmp_path), b, 2, masks["lu"], masks["llu"], masks["llv"], [0.1, 0.6], [0, 0.5, 1], AXES, baro)
    assert sorted(p.name for p in tmp_path.iterdir()) == sorted(
        ["cpsshe8.dat", "cpsshe.dat", "cpsshe.ctl", "cpube8.dat", "cpubi.dat", "cpube.ctl", "cpvbe8.dat",
         "cpvbe.dat", "cpvbe.ctl"])
    with pytest.raises(InmsomError) as e:
        dstd.ocpwrite(str(tmp_path), b, 2, masks["lu"], masks["llu"], masks["llv"], [0.1, 0.6], [0, 0.5, 1], AXES,
                      {"tt": st["tt"]})
    assert e.value.code == 2
    with pytest.raises(InmsomError) as e:
        dstd.ocpread(str(tmp_path), b, 2, masks["lu"], masks["llu"], masks["llv"],
                     {"tt": st["tt"].copy(order="F"), "ttp": st["ttp"].copy(order="F")})
    assert e.value.code == 6


def test_compare_grids(tmp_path):
    """compare_grids on descriptors read back: 0 for the same grids, 1 for
    different counts or a grid past maxgridlen, 2 for a coordinate that
    differs; the undefined value and time step are not compared."""
    c = CTL_CASES[1]

    def write(name, **over):
        a = dict(c, **over)
        y, mo, d, h, mn = a["date"]
        dstd.ctl_file_write(str(tmp_path / f"{name}.dat"), a.get("undef", -1.0e32), a["nx"], a["ny"], a["nz"],
                            a["nt"], a["xtype"], a["x0"], a["hx"], a["ytype"], a["y0"], a["hy"], a["ztype"], a["z0"],
                            a["hz"], a["yr_type"], y, mo, d, h, mn, a["ht"], a["title"], a["var"])
        return dstd.ctl_file_read(tmp_path / f"{name}.ctl")

    base = write("a")
    assert dstd.compare_grids(base, write("b", undef=-9.0, ht=3600.0)) == 0
    assert dstd.compare_grids(base, write("c", nt=13)) == 1
    z = list(c["z0"])
    assert dstd.compare_grids(base, write("d", nz=19, z0=z[:19])) == 1
    assert dstd.compare_grids(base, base, maxgridlen=8) == 1
    z[4] += 1.0
    assert dstd.compare_grids(base, write("e", z0=z)) == 2


def test_ctl_write_read_random(tmp_path):
    """Random descriptors: the library's text equals the restatement's, and
    the library's reader and the restatement's reader agree on it."""
    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as st

    real = st.floats(min_value=-1e12, max_value=1e12, allow_nan=False, allow_infinity=False)
    axis = st.tuples(st.integers(1, 30), st.sampled_from([0, 1]), st.lists(real, min_size=30, max_size=30), real)
    word = st.text(alphabet="abcdefghijklmnopqrstuvwxyz_0123456789", min_size=1, max_size=12)
    title = st.text(alphabet="abcdefghijklmnopqrstuvwxyz ,.()^*/0123456789", min_size=0, max_size=60)

    @settings(max_examples=150, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(ax=axis, ay=axis, az=axis, nt=st.integers(1, 9999), yr=st.sampled_from([0, 1]),
           date=st.tuples(st.integers(1, 9999), st.integers(1, 12), st.integers(1, 31), st.integers(0, 23),
                          st.integers(0, 59)),
           ht=st.floats(min_value=60.0, max_value=5.0e8), title=title, var=word)
    def run(ax, ay, az, nt, yr, date, ht, title, var):
        fname = str(tmp_path / "r.dat")
        args = [fname, -1.0e32]
        dims = [ax[0], ay[0], az[0], nt]
        axes = []
        for n, typ, vals, h in (ax, ay, az):
            axes += [typ, vals[:n] if typ else vals[:1], h]
        args += dims + axes + [yr, *date, ht, title, var]
        dstd.ctl_file_write(*args)
        _, text = od.ctl_text(*args)
        assert (tmp_path / "r.ctl").read_text() == text
        got = _read_both(tmp_path, text, name="r2.ctl")
        assert got is not None and got["nx"] == ax[0] and got["nt"] == nt and got["varname"] == [var]

    run()


def test_field_files_random_boxes(tmp_path):
    """Random fields, masks, boxes and process grids: wdstd/wdstd8 give the
    restatement's bytes, rdstd8 reads back the ocean values, and the ranks
    of a random process grid tiling the box write wdstd's FP32 file with
    pwdstd and read their parts back with prdstd."""
    from dataclasses import replace

    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as st

    from inmsom_elfs_b200.grid import Bounds

    @settings(max_examples=60, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(nx=st.integers(6, 20), ny=st.integers(6, 16), nz=st.integers(1, 4), seed=st.integers(0, 10**6),
           data=st.data())
    def run(nx, ny, nz, seed, data):
        rng = np.random.default_rng(seed)
        g = Bounds.serial(nx - 4, ny - 4)           # arrays 1..nx x 1..ny, interior 3..nx-2 x 3..ny-2
        f = np.asfortranarray(rng.standard_normal((nx, ny, nz)))
        lu = np.asfortranarray((rng.random((nx, ny)) > 0.3).astype(np.float32))
        nzb = data.draw(st.integers(1, nz))
        nze = data.draw(st.integers(nzb, nz))
        nfield = data.draw(st.integers(1, 3))
        box = (data.draw(st.integers(1, 3)), data.draw(st.integers(nx - 2, nx)),
               data.draw(st.integers(1, 3)), data.draw(st.integers(ny - 2, ny)), nzb, nze)
        for name, dtype, write in (("a8.dat", np.float64, dstd.wdstd8), ("a4.dat", np.float32, dstd.wdstd)):
            fx = f.astype(dtype, order="F")
            p = tmp_path / name
            if p.exists():
                p.unlink()
            write(str(tmp_path), name, nfield, fx.copy(order="F"), lu, box)
            assert p.read_bytes() == od.file_bytes([(nfield, fx)], lu, box, dtype)   # earlier fields: zeros
        back = np.zeros_like(f)
        dstd.rdstd8(str(tmp_path), "a8.dat", nfield, back, lu, box)
        nxb, nxe, nyb, nye = box[:4]
        sub = (slice(nxb - 1, nxe), slice(nyb - 1, nye), slice(nzb - 1, nze))
        ocean = np.broadcast_to((np.abs(lu) >= 0.5)[..., None], f.shape)[sub]
        assert np.array_equal(back[sub][ocean], f[sub][ocean]) and np.all(back[sub][~ocean] == 0)
        # a process grid over the interior, with the box equal to the interior
        xs = sorted(set(data.draw(st.lists(st.integers(g.mmm + 1, g.mm), max_size=2))))
        ys = sorted(set(data.draw(st.lists(st.integers(g.nnn + 1, g.nn), max_size=2))))
        xr = list(zip([g.mmm] + xs, [x - 1 for x in xs] + [g.mm]))
        yr = list(zip([g.nnn] + ys, [y - 1 for y in ys] + [g.nn]))
        ibox = (g.mmm, g.mm, g.nnn, g.nn, nzb, nze)
        f4 = f.astype(np.float32, order="F")
        for p in ("w.dat", "p.dat"):
            if (tmp_path / p).exists():
                (tmp_path / p).unlink()
        dstd.wdstd(str(tmp_path), "w.dat", nfield, f4.copy(order="F"), lu, ibox)
        ranks = [replace(g, nx_start=a, nx_end=b_, ny_start=c, ny_end=d, bnd_x1=a - 2, bnd_x2=b_ + 2,
                         bnd_y1=c - 2, bnd_y2=d + 2) for (c, d) in yr for (a, b_) in xr]
        order = data.draw(st.permutations(range(len(ranks))))
        for r in order:
            lb = ranks[r]
            dstd.pwdstd(lb, str(tmp_path), "p.dat", nfield, _local(f4, g, lb), _local(lu, g, lb), nx, ny, nz, ibox)
        assert (tmp_path / "p.dat").read_bytes() == (tmp_path / "w.dat").read_bytes()
        for lb in ranks:
            loc = np.zeros(lb.shape + (nz,), np.float32, order="F")
            dstd.prdstd(lb, str(tmp_path), "w.dat", nfield, loc, _local(lu, g, lb), nx, ny, nz, ibox)
            want = _local(np.where((np.abs(lu) < 0.5)[..., None], od.UNDEF, f4), g, lb)
            assert np.array_equal(loc[2:-2, 2:-2, nzb - 1:nze], want[2:-2, 2:-2, nzb - 1:nze])

    run()


def test_checkpoint_golden_fixture(tmp_path):
    """The library writes the committed golden bytes of a seeded checkpoint
    (tests/golden/make_formats.py) and reads its descriptors as stored."""
    import importlib.util
    from pathlib import Path
    gdir = Path(__file__).resolve().parent / "golden"
    spec = importlib.util.spec_from_file_location("make_formats", gdir / "make_formats.py")
    mf = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mf)
    fix = np.load(gdir / "formats_checkpoint.npz")
    b, masks, z, zw, st = mf.case()
    dstd.ocpwrite(str(tmp_path), b, mf.NZ, masks["lu"], masks["llu"], masks["llv"], z, zw, mf.AXES, st)
    names = sorted(k[5:] for k in fix.files if k.startswith("file:"))
    assert names == sorted(p.name for p in tmp_path.iterdir()) and len(names) == 30
    for name in names:
        assert (tmp_path / name).read_bytes() == fix["file:" + name].tobytes(), name
    for ctl in ("cptt.ctl", "cpube.ctl"):
        got = dstd.ctl_file_read(tmp_path / ctl)
        for key in (k for k in fix.files if k.startswith(f"read:{ctl}:")):
            name, want = key.split(":")[2], fix[key]
            g = got[name]
            if name == "varname":
                assert "\n".join(g) == str(want)
            elif name in ("x0", "y0", "z0"):
                assert np.array_equal(g, want)
            elif want.dtype.kind in "US":
                assert g == str(want)
            else:
                assert g == want.item(), name


def test_ctl_title_is_not_read_list_directed(tmp_path):
    """A TITLE record is taken as text (Service/rw_ctl_file.f90: the title
    is a substring of the record; only VARS, UNDEF, OPTIONS, the axis and
    TDEF records are read list-directed), so separators or slashes in a
    title are no error."""
    for title in (",,", "a, b / c", "/", "1*,2"):
        fname = str(tmp_path / "t.dat")
        dstd.ctl_file_write(fname, -1.0e32, 1, 1, 1, 1, 0, [0.0], 0.0, 0, [0.0], 0.0, 0, [0.0], 0.0,
                            0, 1, 1, 1, 0, 0, 60.0, title, "v")
        text = (tmp_path / "t.ctl").read_text()
        got = _read_both(tmp_path, text, name="t2.ctl")
        assert got is not None and got["title"].strip() == title
