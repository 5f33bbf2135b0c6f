// The reference's on-disk formats (host code; no kernels):
//  * DIOGIN-standard direct-access files: one record per level of a
//    (nxb:nxe, nyb:nye) box of a field, x fastest, FP32 (wdstd/rdstd) or
//    FP64 (wdstd8/rdstd8), record (nfield-1)*(nze-nzb+1) + k-nzb+1, land
//    points (|lu| < 0.5) written as undef = -1.0e32 and read back as 0
//    (Service/input_output_data.f90:117-534; Inc/reclen.fi);
//  * prdstd / pwdstd, the MPI-IO forms (Service/input_output_data.f90:535-819):
//    each rank reads or writes its own interior of the same FP32 file, by
//    positioned I/O on disjoint byte ranges instead of a collective;
//  * the GrADS descriptor ctl_file_write (Service/rw_ctl_file.f90:1-183)
//    with the Fortran edit descriptors of its WRITE statements;
//  * the checkpoint of the barotropic state and its restart
//    (Control/output.f90:1736-1847, Control/init_pars.f90:384-411).
#include "inmsom_gpu.h"

#include <fcntl.h>
#include <unistd.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace inmsom {
int record_error(int code, const char *msg);
}

namespace {

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return inmsom::record_error(code, buf);
}

constexpr float UNDEF = -1.0e32f;   // Inc/reclen.fi:6

// Service/input_output_data.f90:4-115 fulfname: the first blank-free word
// of path and of the file name, joined by one '/'
bool fulfname(std::string &out, const char *path, const char *fname)
{
    auto word = [](const char *s) {
        std::string w;
        if (!s) return w;
        const char *p = s;
        while (*p == ' ') p++;
        while (*p && *p != ' ') w.push_back(*p++);
        return w;
    };
    std::string p = word(path), f = word(fname);
    if (f.empty()) return false;
    if (p.empty()) {
        out = f;
        return true;
    }
    if (p.back() == '/' && f.front() == '/') p.pop_back();
    if (p.back() != '/' && f.front() != '/') p.push_back('/');
    out = p + f;
    return true;
}

bool box_ok(int nx, int ny, int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze)
{
    return !(nxe > nx || nxb < 1 || nxb > nxe || nye > ny || nyb < 1 || nyb > nye || nze > nz || nzb < 1 ||
             nzb > nze);
}

// the shared body of wdstd / wdstd8 (T = float / double)
template <typename T>
int write_std(const char *path, const char *fname, int nfield, T *field, const float *lu, int nx, int ny, int nz,
              int nxb, int nxe, int nyb, int nye, int nzb, int nze, const char *who)
{
    std::string name;
    if (!fulfname(name, path, fname)) return fail(INMSOM_EARG, "%s: no file name", who);
    if (!field || !lu || nfield < 1) return fail(INMSOM_EARG, "%s: bad argument", who);
    if (!box_ok(nx, ny, nz, nxb, nxe, nyb, nye, nzb, nze))
        return fail(INMSOM_EARG, "%s: box outside the field", who);
    const int fd = open(name.c_str(), O_WRONLY | O_CREAT, 0644);    // status='unknown': no truncation
    if (fd < 0) return fail(INMSOM_EIO, "%s: cannot open %s", who, name.c_str());
    const long long bx = nxe - nxb + 1, by = nye - nyb + 1;
    const long long recl = bx * by * (long long)sizeof(T);
    const long long nrecf = (long long)(nfield - 1) * (nze - nzb + 1);
    std::vector<T> rec((size_t)(bx * by));
    auto at = [&](int i, int j, int k) -> T & {
        return field[(size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1))];
    };
    int rc = INMSOM_OK;
    for (int k = nzb, kr = 1; k <= nze; k++, kr++) {
        size_t q = 0;
        for (int j = nyb; j <= nye; j++)
            for (int i = nxb; i <= nxe; i++) {
                if (std::fabs(lu[(size_t)(i - 1) + (size_t)nx * (size_t)(j - 1)]) < 0.5f) at(i, j, k) = (T)UNDEF;
                rec[q++] = at(i, j, k);
            }
        const long long off = (nrecf + kr - 1) * recl;
        if (pwrite(fd, rec.data(), (size_t)recl, (off_t)off) != (ssize_t)recl) {
            rc = fail(INMSOM_EIO, "%s: error writing level %d of %s", who, k, name.c_str());
            break;
        }
        // the reference leaves the written land points at zero in the caller's field
        for (int j = nyb; j <= nye; j++)
            for (int i = nxb; i <= nxe; i++)
                if (std::fabs(lu[(size_t)(i - 1) + (size_t)nx * (size_t)(j - 1)]) < 0.5f) at(i, j, k) = (T)0.0;
    }
    if (close(fd) != 0 && rc == INMSOM_OK) rc = fail(INMSOM_EIO, "%s: error closing %s", who, name.c_str());
    return rc;
}

template <typename T>
int read_std(const char *path, const char *fname, int nfield, T *field, const float *lu, int nx, int ny, int nz,
             int nxb, int nxe, int nyb, int nye, int nzb, int nze, const char *who)
{
    std::string name;
    if (!fulfname(name, path, fname)) return fail(INMSOM_EARG, "%s: no file name", who);
    if (!field || !lu || nfield < 1) return fail(INMSOM_EARG, "%s: bad argument", who);
    if (!box_ok(nx, ny, nz, nxb, nxe, nyb, nye, nzb, nze))
        return fail(INMSOM_EARG, "%s: box outside the field", who);
    const int fd = open(name.c_str(), O_RDONLY);                    // status='old'
    if (fd < 0) return fail(INMSOM_EIO, "%s: cannot open %s", who, name.c_str());
    const long long bx = nxe - nxb + 1, by = nye - nyb + 1;
    const long long recl = bx * by * (long long)sizeof(T);
    const long long nrecf = (long long)(nfield - 1) * (nze - nzb + 1);
    std::vector<T> rec((size_t)(bx * by));
    int rc = INMSOM_OK;
    for (int k = nzb, kr = 1; k <= nze; k++, kr++) {
        const long long off = (nrecf + kr - 1) * recl;
        if (pread(fd, rec.data(), (size_t)recl, (off_t)off) != (ssize_t)recl) {
            rc = fail(INMSOM_EIO, "%s: error reading level %d of %s", who, k, name.c_str());
            break;
        }
        size_t q = 0;
        for (int j = nyb; j <= nye; j++)
            for (int i = nxb; i <= nxe; i++) {
                const size_t ij = (size_t)(i - 1) + (size_t)nx * (size_t)(j - 1);
                field[ij + (size_t)nx * ny * (size_t)(k - 1)] = std::fabs(lu[ij]) < 0.5f ? (T)0.0 : rec[q];
                q++;
            }
    }
    close(fd);
    return rc;
}

// ---- prdstd / pwdstd: one rank's subdomain of the file ---------------------

// Where one rank's interior (nx_start..nx_end, ny_start..ny_end) of levels
// nzb..nze sits in the file: the MPI subarray view of
// Service/input_output_data.f90:583-611 / 706-772 (global sizes = the box,
// local sizes = the interior, offsets = interior start - box start) after
// the displacement bx*by*4*(nfild-1)*bz bytes.
struct SubView {
    long long bx, by, bz;       // the box
    long long lx, ly, ox, oy;   // the rank's part of it
    long long disp;             // bytes before field nfild
    long long nxa, nya;         // the rank's local arrays (bnd_x1:bnd_x2, bnd_y1:bnd_y2)
};

int sub_view(const inmsom_bounds *b, int nfild, int nx, int ny, int nz, int nxb, int nxe, int nyb, int nye, int nzb,
             int nze, SubView &v, const char *who)
{
    if (!b || nfild < 1) return fail(INMSOM_EARG, "%s: bad argument", who);
    if (b->nx_start > b->nx_end || b->ny_start > b->ny_end || b->bnd_x1 > b->nx_start || b->bnd_x2 < b->nx_end ||
        b->bnd_y1 > b->ny_start || b->bnd_y2 < b->ny_end)
        return fail(INMSOM_EARG, "%s: interior %d..%d x %d..%d outside the arrays %d..%d x %d..%d", who, b->nx_start,
                    b->nx_end, b->ny_start, b->ny_end, b->bnd_x1, b->bnd_x2, b->bnd_y1, b->bnd_y2);
    // ierr = 1, 2, 3 of the reference (then mpi_abort)
    if (nxe > nx || nxb < 1 || nxb > nxe) return fail(INMSOM_EARG, "%s: error in grid diapason of 1 - coordinate", who);
    if (nye > ny || nyb < 1 || nyb > nye) return fail(INMSOM_EARG, "%s: error in grid diapason of 2 - coordinate", who);
    if (nze > nz || nzb < 1 || nzb > nze) return fail(INMSOM_EARG, "%s: error in grid diapason of 3 - coordinate", who);
    v.bx = nxe - nxb + 1;
    v.by = nye - nyb + 1;
    v.bz = nze - nzb + 1;
    v.lx = b->nx_end - b->nx_start + 1;
    v.ly = b->ny_end - b->ny_start + 1;
    v.ox = b->nx_start - nxb;
    v.oy = b->ny_start - nyb;
    // MPI_Type_create_subarray refuses a part that leaves the box
    if (v.ox < 0 || v.oy < 0 || v.ox + v.lx > v.bx || v.oy + v.ly > v.by)
        return fail(INMSOM_EARG, "%s: the interior %d..%d x %d..%d is not inside the box %d..%d x %d..%d", who,
                    b->nx_start, b->nx_end, b->ny_start, b->ny_end, nxb, nxe, nyb, nye);
    // 64-bit: the reference forms this product in default integers
    v.disp = v.bx * v.by * 4LL * (long long)(nfild - 1) * v.bz;
    v.nxa = b->bnd_x2 - b->bnd_x1 + 1;
    v.nya = b->bnd_y2 - b->bnd_y1 + 1;
    return INMSOM_OK;
}

// the rank's part of level kr (0-based in the box) as runs of contiguous
// bytes: one run when the part spans whole rows of the box, else one per row
template <typename F>
int for_runs(const SubView &v, long long kr, F &&run)
{
    const long long lvl = v.disp + 4LL * kr * v.bx * v.by;
    if (v.lx == v.bx) return run(lvl + 4LL * v.oy * v.bx, 0LL, v.lx * v.ly);
    for (long long j = 0; j < v.ly; j++) {
        const int rc = run(lvl + 4LL * ((v.oy + j) * v.bx + v.ox), j * v.lx, v.lx);
        if (rc != INMSOM_OK) return rc;
    }
    return INMSOM_OK;
}

// ---- Fortran edit descriptors of ctl_file_write ----------------------------

// d significant digits of |x| and the exponent N with |x| = 0.d1d2..dd x 10^N
void sig_digits(double x, int d, std::string &digits, int &n)
{
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(x));
    digits.clear();
    const char *p = buf;
    for (; *p && *p != 'e'; p++)
        if (*p >= '0' && *p <= '9') digits.push_back(*p);
    n = std::atoi(p + 1) + 1;
}

std::string right(const std::string &s, int w)
{
    if ((int)s.size() > w) return std::string((size_t)w, '*');
    return std::string((size_t)(w - (int)s.size()), ' ') + s;
}

// Ew.d: [-]0.d1..ddE+NN (E omitted for |N| > 99)
std::string fmt_e(double x, int w, int d)
{
    std::string s = std::signbit(x) && x != 0.0 ? "-" : "";
    if (x == 0.0) {
        s += "0." + std::string((size_t)d, '0') + "E+00";
        return right(s, w);
    }
    std::string dig;
    int n;
    sig_digits(x, d, dig, n);
    char ex[16];
    if (std::abs(n) <= 99) std::snprintf(ex, sizeof ex, "E%c%02d", n < 0 ? '-' : '+', std::abs(n));
    else std::snprintf(ex, sizeof ex, "%c%03d", n < 0 ? '-' : '+', std::abs(n));
    s += "0." + dig + ex;
    if ((int)s.size() > w && s.compare(0, 2, "0.") == 0) s.erase(0, 1);      // optional leading zero
    if ((int)s.size() > w && s.compare(0, 3, "-0.") == 0) s.erase(1, 1);
    return right(s, w);
}

// Fw.d (the decimal point is always written, also for d = 0)
std::string fmt_f(double x, int w, int d)
{
    char buf[512];
    std::snprintf(buf, sizeof buf, "%#.*f", d, x);
    std::string s = buf;
    if (s[0] == '-' && s.find_first_not_of("-0.") == std::string::npos) s.erase(0, 1);   // no minus zero
    if ((int)s.size() > w && s.compare(0, 2, "0.") == 0) s.erase(0, 1);
    if ((int)s.size() > w && s.compare(0, 3, "-0.") == 0) s.erase(1, 1);
    return right(s, w);
}

// Gw.d for a real value (Fortran 2008 10.7.5.2.2, no Ee part: n = 4 blanks)
std::string fmt_g(double x, int w, int d)
{
    if (x == 0.0) return fmt_f(0.0, w - 4, d - 1) + "    ";
    std::string dig;
    int n;
    sig_digits(x, d, dig, n);
    if (n >= 0 && n <= d) return fmt_f(x, w - 4, d - n) + "    ";
    return fmt_e(x, w, d);
}

std::string fmt_i(long long v, int w, int m = 0)
{
    std::string s = std::to_string(v < 0 ? -v : v);
    if ((int)s.size() < m) s = std::string((size_t)(m - (int)s.size()), '0') + s;
    if (v < 0) s = "-" + s;
    return right(s, w);
}

// '(a,i6,a,2(g15.8,5x))' or '(a,i6,a,7(g15.8,1x)/(22x,7(g15.8,1x)))'.  An X
// edit descriptor only moves the position: the blanks it skips are written
// when characters follow in the record, so none ends a line.
std::string axis_lines(const char *tag, int n, int type, const double *v0, double h)
{
    std::string s = std::string(tag) + fmt_i(n, 6);
    if (type == 0) {
        s += "  LINEAR   " + fmt_g(v0[0], 15, 8) + "     " + fmt_g(h, 15, 8);
        return s + "\n";
    }
    s += "  LEVELS  ";
    for (int i = 0; i < n; i++) {
        if (i > 0) s += i % 7 == 0 ? "\n" + std::string(22, ' ') : std::string(" ");
        s += fmt_g(v0[i], 15, 8);
    }
    return s + "\n";
}

// Service/rw_ctl_file.f90:161-183 (single-precision arithmetic as there)
void sec_to_yr_mo_hr_mn(float sec, int &nyr, int &nmo, int &ndy, int &nhr, int &nmn)
{
    const float yr_sec = 360.0f * 86400.0f, mo_sec = 30.0f * 86400.0f;
    float sec1 = sec + 0.10f;
    nyr = (int)(sec1 / yr_sec);
    sec1 = sec1 - (float)nyr * yr_sec;
    nmo = (int)(sec1 / mo_sec);
    sec1 = sec1 - (float)nmo * mo_sec;
    ndy = (int)(sec1 / 86400.0f);
    sec1 = sec1 - (float)ndy * 86400.0f;
    nhr = (int)(sec1 / 3600.0f);
    sec1 = sec1 - (float)nhr * 3600.0f;
    nmn = (int)(sec1 / 60.0f);
}

// Service/rw_ctl_file.f90:140-158 extname on a character(128) name: the
// last '.' in positions 2..125 and the four characters after it become
// `ext` and a blank (without a '.', positions 2..6, as the loop leaves n)
std::string extname(const std::string &name, const char *ext)
{
    std::string s = name.substr(0, 128);
    s.resize(128, ' ');
    int n = 125;
    for (; n >= 2; n--)
        if (s[(size_t)n - 1] == '.') break;
    if (n < 2) n = 2;
    std::string e(ext);
    e.resize(5, ' ');
    s.replace((size_t)n - 1, 5, e);
    while (!s.empty() && s.back() == ' ') s.pop_back();
    return s;
}

}  // namespace

namespace inmsom {
// fulfname for callers elsewhere in the library (empty on a missing file name)
std::string full_file_name(const char *path, const char *fname)
{
    std::string out;
    return fulfname(out, path, fname) ? out : std::string();
}
}  // namespace inmsom

extern "C" {

int inmsom_wdstd8(const char *path, const char *fname, int nfield, double *field, const float *lu, int nx, int ny,
                  int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze)
{
    return write_std<double>(path, fname, nfield, field, lu, nx, ny, nz, nxb, nxe, nyb, nye, nzb, nze,
                             "inmsom_wdstd8");
}

int inmsom_wdstd(const char *path, const char *fname, int nfield, float *field, const float *lu, int nx, int ny,
                 int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze)
{
    return write_std<float>(path, fname, nfield, field, lu, nx, ny, nz, nxb, nxe, nyb, nye, nzb, nze,
                            "inmsom_wdstd");
}

int inmsom_rdstd8(const char *path, const char *fname, int nfield, double *field, const float *lu, int nx, int ny,
                  int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze)
{
    return read_std<double>(path, fname, nfield, field, lu, nx, ny, nz, nxb, nxe, nyb, nye, nzb, nze,
                            "inmsom_rdstd8");
}

int inmsom_rdstd(const char *path, const char *fname, int nfield, float *field, const float *lu, int nx, int ny,
                 int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze)
{
    return read_std<float>(path, fname, nfield, field, lu, nx, ny, nz, nxb, nxe, nyb, nye, nzb, nze,
                           "inmsom_rdstd");
}

int inmsom_pwdstd(const inmsom_bounds *b, const char *path, const char *fname, int nfild, float *fild,
                  const float *lu, int nx, int ny, int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze)
{
    const char *who = "inmsom_pwdstd";
    std::string name;
    if (!fulfname(name, path, fname)) return fail(INMSOM_EARG, "%s: error in full name of file for writing", who);
    if (!fild || !lu) return fail(INMSOM_EARG, "%s: NULL array", who);
    SubView v;
    const int rc0 = sub_view(b, nfild, nx, ny, nz, nxb, nxe, nyb, nye, nzb, nze, v, who);
    if (rc0 != INMSOM_OK) return rc0;
    auto at = [&](int i, int j, int k) -> float & {
        return fild[(size_t)(i - b->bnd_x1) + (size_t)v.nxa * ((size_t)(j - b->bnd_y1) + (size_t)v.nya * (k - 1))];
    };
    // the land points of the interior become undef in the caller's array
    for (int j = b->ny_start; j <= b->ny_end; j++)
        for (int i = b->nx_start; i <= b->nx_end; i++)
            if (std::fabs(lu[(size_t)(i - b->bnd_x1) + (size_t)v.nxa * (size_t)(j - b->bnd_y1)]) < 0.5f)
                for (int k = nzb; k <= nze; k++) at(i, j, k) = UNDEF;
    const int fd = open(name.c_str(), O_WRONLY | O_CREAT, 0644);    // mpi_mode_wronly + mpi_mode_create
    if (fd < 0) return fail(INMSOM_EIO, "%s: error in open file for writing: %s", who, name.c_str());
    std::vector<float> part((size_t)(v.lx * v.ly));
    int rc = INMSOM_OK;
    for (int k = nzb; k <= nze && rc == INMSOM_OK; k++) {
        size_t q = 0;
        for (int j = b->ny_start; j <= b->ny_end; j++)
            for (int i = b->nx_start; i <= b->nx_end; i++) part[q++] = at(i, j, k);
        rc = for_runs(v, k - nzb, [&](long long off, long long first, long long n) {
            const ssize_t want = (ssize_t)(4 * n);
            if (pwrite(fd, part.data() + first, (size_t)want, (off_t)off) != want)
                return fail(INMSOM_EIO, "%s: error in writing level %d of %s", who, k, name.c_str());
            return (int)INMSOM_OK;
        });
    }
    if (close(fd) != 0 && rc == INMSOM_OK) rc = fail(INMSOM_EIO, "%s: error closing %s", who, name.c_str());
    return rc;
}

int inmsom_prdstd(const inmsom_bounds *b, const char *path, const char *fname, int nfild, float *fild,
                  const float *lu, int nx, int ny, int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze)
{
    (void)lu;   // prdstd takes the mask but reads every point
    const char *who = "inmsom_prdstd";
    std::string name;
    if (!fulfname(name, path, fname)) return fail(INMSOM_EARG, "%s: error in full name of file for reading", who);
    if (!fild) return fail(INMSOM_EARG, "%s: NULL array", who);
    SubView v;
    const int rc0 = sub_view(b, nfild, nx, ny, nz, nxb, nxe, nyb, nye, nzb, nze, v, who);
    if (rc0 != INMSOM_OK) return rc0;
    const int fd = open(name.c_str(), O_RDONLY);                    // mpi_mode_rdonly
    if (fd < 0) return fail(INMSOM_EIO, "%s: error in open file for reading: %s", who, name.c_str());
    std::vector<float> part((size_t)(v.lx * v.ly));
    int rc = INMSOM_OK;
    for (int k = nzb; k <= nze && rc == INMSOM_OK; k++) {
        // what lies past the end of the file is not read, as MPI-IO reads
        // (the reference does not look at the count read): keep those values
        size_t q = 0;
        for (int j = b->ny_start; j <= b->ny_end; j++)
            for (int i = b->nx_start; i <= b->nx_end; i++)
                part[q++] = fild[(size_t)(i - b->bnd_x1) +
                                 (size_t)v.nxa * ((size_t)(j - b->bnd_y1) + (size_t)v.nya * (k - 1))];
        rc = for_runs(v, k - nzb, [&](long long off, long long first, long long n) {
            char *dst = reinterpret_cast<char *>(part.data() + first);
            long long got = 0;
            while (got < 4 * n) {
                const ssize_t r = pread(fd, dst + got, (size_t)(4 * n - got), (off_t)(off + got));
                if (r < 0) return fail(INMSOM_EIO, "%s: error in reading level %d of %s", who, k, name.c_str());
                if (r == 0) break;
                got += r;
            }
            return (int)INMSOM_OK;
        });
        q = 0;
        for (int j = b->ny_start; j <= b->ny_end; j++)
            for (int i = b->nx_start; i <= b->nx_end; i++)
                fild[(size_t)(i - b->bnd_x1) + (size_t)v.nxa * ((size_t)(j - b->bnd_y1) + (size_t)v.nya * (k - 1))] =
                    part[q++];
    }
    close(fd);
    return rc;
}

int inmsom_ctl_file_write(const char *fname, float undef, int nx, int ny, int nz, int nt, int xtype, const double *x0,
                          double hx, int ytype, const double *y0, double hy, int ztype, const double *z0, double hz,
                          int yr_type, int year0, int month0, int day0, int hour0, int minute0, float ht,
                          const char *title, const char *varname)
{
    static const char *month[12] = {"JAN", "FEB", "MAR", "APR", "MAY", "JUN",
                                    "JUL", "AUG", "SEP", "OCT", "NOV", "DEC"};
    if (!fname || !x0 || !y0 || !z0 || !title || !varname || month0 < 1 || month0 > 12)
        return fail(INMSOM_EARG, "inmsom_ctl_file_write: bad argument");
    // the names are character(128) variables: truncated there, padded with blanks
    const std::string base(fname);
    const std::string namectl = extname(base, ".ctl"), namedat = extname(base, ".dat");
    std::string namedat2 = namedat.substr(namedat.find_last_of('/') == std::string::npos ? 0
                                                                                          : namedat.find_last_of('/') + 1);
    namedat2.resize(128, ' ');
    std::string s;
    s += "DSET    ^" + namedat2 + "\n";
    s += std::string("TITLE    ") + title + "\n";
    s += "UNDEF   " + fmt_e(undef, 12, 5) + "  ! gap value\n";
    s += axis_lines("XDEF  ", nx, xtype, x0, hx);
    s += axis_lines("YDEF  ", ny, ytype, y0, hy);
    s += axis_lines("ZDEF  ", nz, ztype, z0, hz);
    // for a step under a minute the reference leaves the unit unset and k at
    // the position of the last '/' in the data file's name (its earlier use)
    const size_t sl = namedat.find_last_of('/');
    int nyr, nmo, ndy, nhr, nmn, k = sl == std::string::npos ? 0 : (int)sl + 1;
    sec_to_yr_mo_hr_mn(ht, nyr, nmo, ndy, nhr, nmn);
    std::string tf = "  ";
    if (nyr != 0) tf = "yr", k = nyr;
    else if (nmo != 0) tf = "mo", k = nmo;
    else if (ndy != 0) tf = "dy", k = ndy;
    else if (nhr != 0) tf = "hr", k = nhr;
    else if (nmn != 0) tf = "mn", k = nmn;
    s += "TDEF  " + fmt_i(nt, 6) + "  LINEAR  " + fmt_i(hour0, 2, 2) + ":" + fmt_i(minute0, 2, 2) + "Z" +
         fmt_i(day0, 2, 2) + month[month0 - 1] + fmt_i(year0, 4, 4) + "     " + fmt_i(k, 4) + tf + "\n";
    if (yr_type == 0) s += "OPTIONS  365_DAY_CALENDAR\n";
    s += "VARS 1  ! Number of variables\n";
    s += std::string(varname) + "        " + fmt_i(nz, 5) + "  1 VARIABLES \n";
    s += "ENDVARS\n";
    s += "\n";
    FILE *f = std::fopen(namectl.c_str(), "w");
    if (!f) return fail(INMSOM_EIO, "inmsom_ctl_file_write: cannot open %s", namectl.c_str());
    const bool ok = std::fwrite(s.data(), 1, s.size(), f) == s.size();
    if (std::fclose(f) != 0 || !ok)
        return fail(INMSOM_EIO, "inmsom_ctl_file_write: error writing %s", namectl.c_str());
    return INMSOM_OK;
}

}  // extern "C"
