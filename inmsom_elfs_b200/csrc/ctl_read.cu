// The GrADS descriptor reader ctl_file_read (Service/rw_ctl_file.f90:185-566),
// its helper nonblank (:568-596), and compare_grids (:628-714), which
// compares the grids two descriptors state; host code, no kernels.
//
// The reference reads the descriptor record by record (character(256),
// at most 512 iterations) and dispatches on the keyword at the first
// non-blank position in three spellings (UPPER, lower, Capitalised).  Its
// list-directed READs are restated here: values separated by blanks or
// commas, quoted character values, r*c repeat counts, a slash ending the
// read; an external read (VARS names, LEVELS values after BACKSPACE)
// continues over the following records until it has its values and the
// loop goes on after the last record consumed.  Where the reference stops
// on an end-of-file or a malformed value (a runtime error in Fortran, or a
// printed message and RETURN at its labels 8-22), this returns INMSOM_EARG
// with the message and leaves what it had read so far in the outputs,
// inform included.  A slash ends a LEVELS read and leaves the values it
// did not reach as they were; a slash or a null value ("r*", ",,") before
// any other value the reference reads makes the call fail.  The summary
// the reference prints on standard output when inform is non-zero on entry
// is not written.
#include "inmsom_gpu.h"

#include <algorithm>
#include <cctype>
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

constexpr size_t kRecLen = 256;   // character(256) string
constexpr int kMaxIter = 512;     // do line = 1, 512

constexpr size_t kNone = (size_t)-1;

// one list-directed record: its values, whether a slash ended it, and how
// many values precede the first null value (kNone: there is none)
struct Items {
    std::vector<std::string> v;
    bool slash = false;
    size_t null_at = kNone;
};

Items list_items(const std::string &rec)
{
    Items out;
    size_t i = 0;
    while (i < rec.size()) {
        bool comma = false;
        while (i < rec.size() && (rec[i] == ' ' || rec[i] == '\t' || rec[i] == ',')) {
            if (rec[i] == ',') {
                if (comma && out.null_at == kNone) out.null_at = out.v.size();   // ",,"
                comma = true;
            }
            i++;
        }
        if (i >= rec.size()) break;
        if (rec[i] == '/') {
            out.slash = true;
            break;
        }
        std::string tok;
        if (rec[i] == '\'' || rec[i] == '"') {
            const char q = rec[i++];
            while (i < rec.size()) {
                if (rec[i] == q) {
                    if (i + 1 < rec.size() && rec[i + 1] == q) {   // a doubled quote is one quote
                        tok.push_back(q);
                        i += 2;
                        continue;
                    }
                    i++;
                    break;
                }
                tok.push_back(rec[i++]);
            }
            out.v.push_back(tok);
            continue;
        }
        while (i < rec.size() && rec[i] != ' ' && rec[i] != '\t' && rec[i] != ',' && rec[i] != '/')
            tok.push_back(rec[i++]);
        const size_t star = tok.find('*');
        size_t d = 0;
        while (d < tok.size() && std::isdigit((unsigned char)tok[d])) d++;
        if (star != std::string::npos && star == d && d > 0) {   // r*c
            const long r = std::strtol(tok.substr(0, d).c_str(), nullptr, 10);
            const std::string c = tok.substr(d + 1);
            if (c.empty()) {   // r* : r null values
                if (out.null_at == kNone) out.null_at = out.v.size();
                continue;
            }
            for (long k = 0; k < r; k++) out.v.push_back(c);
        } else {
            out.v.push_back(tok);
        }
    }
    return out;
}

std::string trim(const std::string &t)
{
    const size_t a = t.find_first_not_of(' ');
    if (a == std::string::npos) return "";
    return t.substr(a, t.find_last_not_of(' ') - a + 1);
}

bool read_int(const std::string &tok, int &v)
{
    const std::string t = trim(tok);
    if (t.empty()) return false;
    char *end = nullptr;
    const long x = std::strtol(t.c_str(), &end, 10);
    if (*end) return false;
    v = (int)x;
    return true;
}

// a real constant in Fortran's input forms: a D or Q exponent letter, or a
// signed exponent with no letter ("1.5-3")
std::string c_real(const std::string &tok)
{
    std::string u = trim(tok);
    for (char &ch : u)
        if (ch == 'd' || ch == 'D' || ch == 'q' || ch == 'Q') ch = 'E';
    if (u.find_first_of("eE") == std::string::npos)
        for (size_t k = 1; k < u.size(); k++)
            if ((u[k] == '+' || u[k] == '-') && (std::isdigit((unsigned char)u[k - 1]) || u[k - 1] == '.')) {
                u.insert(k, 1, 'E');
                break;
            }
    return u;
}

bool read_double(const std::string &tok, double &v)
{
    const std::string u = c_real(tok);
    if (u.empty()) return false;
    char *end = nullptr;
    v = std::strtod(u.c_str(), &end);
    return !*end;
}

// a REAL (kind 4) value: the decimal string rounded once to single precision
bool read_float(const std::string &tok, float &v)
{
    const std::string u = c_real(tok);
    if (u.empty()) return false;
    char *end = nullptr;
    v = std::strtof(u.c_str(), &end);
    return !*end;
}

// a Fortran character variable of length cap gets tok: truncated or padded
std::string as_char(const std::string &tok, size_t cap)
{
    std::string s = tok.substr(0, std::min(tok.size(), cap));
    s.resize(cap, ' ');
    return s;
}

// s(n0:n0+len(w)-1) equals w in one of its three spellings
bool spelled(const std::string &s, size_t n0, const char *upper)
{
    const size_t n = std::strlen(upper);
    if (n0 + n > s.size()) return false;
    const std::string w = s.substr(n0, n);
    std::string lo(upper), cap(upper);
    for (char &ch : lo) ch = (char)std::tolower((unsigned char)ch);
    for (size_t k = 1; k < n; k++) cap[k] = lo[k];
    return w == upper || w == lo || w == cap;
}

// a grid or calendar word compared as the character(32) variable holding it
bool word_is(const std::string &tok, const char *upper)
{
    return spelled(as_char(tok, 32), 0, upper) && trim(as_char(tok, 32)).size() == std::strlen(upper);
}

// a character variable of len-1 characters takes v (truncated, blank
// padded); it is returned without its trailing blanks, NUL-terminated
void put(char *dst, int len, const std::string &v)
{
    if (!dst || len <= 0) return;
    size_t n = std::min(v.size(), (size_t)len - 1);
    while (n > 0 && v[n - 1] == ' ') n--;
    std::memcpy(dst, v.data(), n);
    dst[n] = '\0';
}

struct Reader {
    std::vector<std::string> rec;   // the file's records as character(256)
    size_t next = 0;                // the record the next READ takes

    // an external list-directed READ of `need` values from the next record
    // on; returns false at the end of the file before a slash or the values
    bool read(size_t need, Items &out)
    {
        out = Items{};
        while (out.v.size() < need) {
            if (next >= rec.size()) return false;
            Items r = list_items(rec[next++]);
            if (out.null_at == kNone && r.null_at != kNone) out.null_at = out.v.size() + r.null_at;
            out.v.insert(out.v.end(), r.v.begin(), r.v.end());
            if (r.slash) {
                out.slash = true;
                break;
            }
        }
        return true;
    }
};

}  // namespace

extern "C" {

int inmsom_ctl_file_read(const char *ctlname, char *datname, int datname_len, float *undef, int *nx, int *ny,
                         int *nz, int *nt, int *xtype, double *x0, int x0_cap, double *hx, int *ytype, double *y0,
                         int y0_cap, double *hy, int *ztype, double *z0, int z0_cap, double *hz, int *nvar,
                         int *yr_type, int *year0, int *month0, int *day0, int *hour0, int *minute0, float *ht,
                         char *title, int title_len, char *varname, int varname_len, int varname_cap, int *inform)
{
    static const char *const kMonth[12] = {"JAN", "FEB", "MAR", "APR", "MAY", "JUN",
                                           "JUL", "AUG", "SEP", "OCT", "NOV", "DEC"};
    if (!ctlname || !undef || !nx || !ny || !nz || !nt || !xtype || !x0 || !hx || !ytype || !y0 || !hy || !ztype ||
        !z0 || !hz || !nvar || !yr_type || !year0 || !month0 || !day0 || !hour0 || !minute0 || !ht || !inform)
        return fail(INMSOM_EARG, "inmsom_ctl_file_read: NULL argument");
    if (datname_len < 1 || (title && title_len < 1) || (varname && (varname_len < 1 || varname_cap < 1)))
        return fail(INMSOM_EARG, "inmsom_ctl_file_read: a character argument has no room");
    *inform = 0;
    FILE *f = std::fopen(ctlname, "r");
    if (!f) return fail(INMSOM_EIO, "inmsom_ctl_file_read: cannot open %s", ctlname);
    Reader in;
    {
        std::string cur;
        int ch;
        bool any = false;
        while ((ch = std::fgetc(f)) != EOF) {
            any = true;
            if (ch == '\n') {
                if (!cur.empty() && cur.back() == '\r') cur.pop_back();
                in.rec.push_back(as_char(cur, kRecLen));
                cur.clear();
                any = false;
            } else {
                cur.push_back((char)ch);
            }
        }
        if (any) in.rec.push_back(as_char(cur, kRecLen));
    }
    std::fclose(f);

    put(datname, datname_len, "");
    *yr_type = 1;
    const auto err = [&](const char *what) {
        return fail(INMSOM_EARG, "inmsom_ctl_file_read: error in %s: %s", ctlname, what);
    };

    for (int line = 1; line <= kMaxIter; line++) {
        if (in.next >= in.rec.size()) return err("exit by eof, not by endvars");
        const std::string s = in.rec[in.next++];
        // nonblank(string, 1): 0 for a blank record and for a first
        // non-blank past len(string)-5
        const size_t p = s.find_first_not_of(' ');
        if (p == std::string::npos || p + 1 > kRecLen - 5) continue;
        const Items it = list_items(s);   // READ(string, *)
        const auto have = [&](size_t n) { return it.v.size() >= n && (it.null_at == kNone || it.null_at >= n); };

        if (spelled(s, p, "ENDVARS")) return INMSOM_OK;

        if (spelled(s, p, "VARS")) {
            if (!have(2) || !read_int(it.v[1], *nvar)) return err("in definition vars or variable name");
            for (int l = 0; l < *nvar; l++) {
                Items v;
                int i;
                if (!in.read(2, v) || v.v.size() < 2 || (v.null_at != kNone && v.null_at < 2) ||
                    !read_int(v.v[1], i))
                    return err("in definition vars or variable name");
                if (varname) {
                    if (l >= varname_cap) return err("more variables than the varname array holds");
                    put(varname + (size_t)l * (size_t)varname_len, varname_len, v.v[0]);
                }
            }
            (*inform)++;
        }

        if (spelled(s, p, "DSET")) {
            size_t l1 = p + 4;
            while (l1 < kRecLen && (s[l1] == ' ' || s[l1] == '^')) l1++;
            // the last non-blank within len(datname) characters from l1
            const size_t cap = (size_t)datname_len - 1;
            long l2 = (long)std::min(kRecLen, l1 + cap) - 1;
            while (l2 >= (long)(p + 4) && s[(size_t)l2] == ' ') l2--;
            if (l1 >= kRecLen || (long)l1 > l2) return err("in definition name of file with data");
            put(datname, datname_len, s.substr(l1, (size_t)l2 - l1 + 1));
            (*inform)++;
        }

        if (spelled(s, p, "TITLE")) {
            // READ(string(nb+5:256), '(A)') title: its first len(title) characters
            put(title, title_len, s.substr(p + 5));
            (*inform)++;
        }

        if (spelled(s, p, "UNDEF")) {
            if (!have(2) || !read_float(it.v[1], *undef)) return err("in definition undefinit value");
            (*inform)++;
        }

        if (spelled(s, p, "OPTIONS")) {
            if (!have(2)) return err("in definition Options");
            (*inform)++;
            if (as_char(it.v[1], 32).compare(0, 3, "365") == 0) *yr_type = 0;
        }

        struct Axis {
            const char *tag, *what;
            int *n, *type, cap;
            double *v, *h;
            int off;   // v(i) = v(1) + h*dfloat(i - off): x and y use i-1, z uses i
        };
        const Axis axes[3] = {{"XDEF", "in definition x-grid", nx, xtype, x0_cap, x0, hx, 1},
                              {"YDEF", "in definition y-grid", ny, ytype, y0_cap, y0, hy, 1},
                              {"ZDEF", "in definition z-grid", nz, ztype, z0_cap, z0, hz, 0}};
        for (const Axis &ax : axes) {
            if (!spelled(s, p, ax.tag)) continue;
            if (!have(3) || !read_int(it.v[1], *ax.n)) return err(ax.what);
            if (word_is(it.v[2], "LINEAR")) {
                *ax.type = 0;
                if (std::max(*ax.n, 1) > ax.cap) return err("more grid values than the array holds");
                if (!have(5) || !read_int(it.v[1], *ax.n) || !read_double(it.v[3], ax.v[0]) ||
                    !read_double(it.v[4], *ax.h))
                    return err(ax.what);
                for (int i = 2; i <= *ax.n; i++) ax.v[i - 1] = ax.v[0] + *ax.h * (double)(i - ax.off);
                (*inform)++;
            } else if (word_is(it.v[2], "LEVELS")) {
                *ax.type = 1;
                if (*ax.n > ax.cap) return err("more grid values than the array holds");
                in.next--;   // BACKSPACE
                Items all;
                const size_t need = 3 + (size_t)std::max(*ax.n, 0);
                if (!in.read(need, all) || all.v.size() < 3) return err(ax.what);
                const size_t got = std::min({need, all.v.size(), all.null_at});
                int l;
                if (!read_int(all.v[1], l)) return err(ax.what);
                // a slash leaves the values it did not reach as they were
                if (got < 3 || (got < need && all.null_at != kNone)) return err(ax.what);
                for (size_t i = 3; i < got; i++)
                    if (!read_double(all.v[i], ax.v[i - 3])) return err(ax.what);
                *ax.h = 0.0;
                (*inform)++;
            }
        }

        if (spelled(s, p, "TDEF")) {
            if (!have(5) || !read_int(it.v[1], *nt)) return err("in definition t-grid");
            if (word_is(it.v[2], "LINEAR")) {
                const std::string ti = as_char(it.v[3], 32), st = as_char(it.v[4], 32);
                size_t l2 = 32;   // last non-blank of timestep (1-based), 1 when none after position 1
                while (l2 >= 2 && st[l2 - 1] == ' ') l2--;
                if (l2 < 2) l2 = 1;
                if (!read_int(ti.substr(0, 2), *hour0) || !read_int(ti.substr(3, 2), *minute0) ||
                    !read_int(ti.substr(6, 2), *day0) || !read_int(ti.substr(11, 4), *year0))
                    return err("in definition t-grid");
                const std::string mo = ti.substr(8, 3);
                for (int k = 0; k < 12; k++)
                    if (spelled(mo, 0, kMonth[k])) *month0 = k + 1;
                float h;
                if (l2 < 3 || !read_float(st.substr(0, l2 - 2), h)) return err("in definition t-grid");
                const std::string unit = st.substr(l2 - 2, 2);
                if (unit == "yr") h = h * 365.0f * 24.0f * 3600.0f;
                else if (unit == "mo") h = h * 30.0f * 24.0f * 3600.0f;
                else if (unit == "dy") h = h * 24.0f * 3600.0f;
                else if (unit == "hr") h = h * 3600.0f;
                else if (unit == "mn") h = h * 60.0f;
                else {
                    *ht = h;
                    return err("in definition time step for t-grid");
                }
                *ht = h;
            }
        }
    }
    // the loop ends without ENDVARS: the reference falls through to its
    // first error label (the undefined-value message)
    return err("in definition undefinit value");
}

int inmsom_compare_grids(int maxgridlen, int *ierr, float undefa, int nxa, int nya, int nza, int nta,
                         const double *xa, double hxa, const double *ya, double hya, float ta, float hta,
                         const double *za, double hza, float undefb, int nxb, int nyb, int nzb, int ntb,
                         const double *xb, double hxb, const double *yb, double hyb, float tb, float htb,
                         const double *zb, double hzb)
{
    (void)undefa, (void)hxa, (void)hya, (void)ta, (void)hta, (void)hza;
    (void)undefb, (void)hxb, (void)hyb, (void)tb, (void)htb, (void)hzb;
    if (!ierr || !xa || !ya || !za || !xb || !yb || !zb)
        return fail(INMSOM_EARG, "inmsom_compare_grids: NULL argument");
    *ierr = 0;
    // ierr = 1: a grid longer than maxgridlen, or different point counts
    // (the checks of Service/rw_ctl_file.f90:653-692, in their order)
    if (nxa > maxgridlen || nya > maxgridlen || nza > maxgridlen || nxa != nxb || nya != nyb || nza != nzb ||
        nta != ntb) {
        *ierr = 1;
        return INMSOM_OK;
    }
    // ierr = 2: a coordinate that differs (:694-712)
    for (int i = 0; i < nxa; i++)
        if (xa[i] != xb[i]) *ierr = 2;
    for (int i = 0; i < nya; i++)
        if (ya[i] != yb[i]) *ierr = 2;
    for (int i = 0; i < nza; i++)
        if (za[i] != zb[i]) *ierr = 2;
    return INMSOM_OK;
}

}  // extern "C"
