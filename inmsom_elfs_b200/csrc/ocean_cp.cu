// The whole checkpoint of the ocean state from host arrays (host code, no
// kernels): ocpwrite (Control/output.f90:1454-1847) and the restart reads
// that Control/init_pars.f90:312-417 lists after its "not done yet" stop.
// The file formats are the ones of dstd.cu (wdstd8/wdstd/rdstd8 and
// ctl_file_write); inmsom_write_checkpoint / inmsom_read_checkpoint cover
// the barotropic part of the same files from a context's resident state.
#include "inmsom_gpu.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

namespace inmsom {
int record_error(int code, const char *msg);
std::string full_file_name(const char *path, const char *fname);
}  // namespace inmsom

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

#define CKR(expr)                       \
    do {                                \
        const int r_ = (expr);          \
        if (r_ != INMSOM_OK) return r_; \
    } while (0)

enum Mask { LU, LLU, LLV };
enum Levels { ONE, NZ, NZ1 };   // 1, nz or nz+1 levels

// one checkpoint group of ocpwrite, in its order: the FP64 file, the FP32
// file, the name the descriptor is made from, the mask, the box start
// (mmm-dx, nnn-dy), the levels, the descriptor's title and variable
struct Group {
    const char *f8, *f4, *ctl;
    Mask mask;
    int dx, dy;
    Levels lev;
    const char *title, *var;
};
const Group GROUPS[10] = {
    {"cptt8.dat", "cptt.dat", "cptt.dat", LU, 0, 0, NZ, "Potential temperature, C", "tt"},
    {"cpss8.dat", "cpss.dat", "cpss.dat", LU, 0, 0, NZ, "Salinity, PSU", "ss"},
    {"cpuu8.dat", "cpuu.dat", "cpuu.dat", LLU, 1, 0, NZ, "Zonal velocity, m/s", "u"},
    {"cpvv8.dat", "cpvv.dat", "cpvv.dat", LLV, 0, 1, NZ, "Meridional velocity, m/s", "v"},
    {"cpq28.dat", "cpq2.dat", "cpq2.dat", LU, 0, 0, NZ1, "turbulent kunetic energy, (m/s)^2", "q2"},
    {"cpq2l8.dat", "cpq2l.dat", "cpq2l.dat", LU, 0, 0, NZ1, "turbulent kunetic energy by length scale, (m/s)^2*m",
     "q2l"},
    {"cpsshi8.dat", "cpsshi.dat", "cpsshi.dat", LU, 0, 0, ONE, "Internal SSH, m", "ssh"},
    {"cpsshe8.dat", "cpsshe.dat", "cpsshe.dat", LU, 0, 0, ONE, "External SSH, m", "ssh"},
    // the FP32 file of the u transport is cpubi.dat, its descriptor names cpube.dat
    {"cpube8.dat", "cpubi.dat", "cpube.dat", LLU, 1, 0, ONE, "External UB, m/s", "ub"},
    {"cpvbe8.dat", "cpvbe.dat", "cpvbe.dat", LLV, 0, 1, ONE, "External VB, m/s", "vb"},
};

// the pair of arrays of group g (present, previous)
void pair(inmsom_ocean_state *s, int g, double **a, double **b)
{
    double **p[10][2] = {{&s->tt, &s->ttp},     {&s->ss, &s->ssp},         {&s->uu, &s->uup},
                         {&s->vv, &s->vvp},     {&s->q2, &s->q2p},         {&s->q2l, &s->q2lp},
                         {&s->ssh_i, &s->sshp_i}, {&s->ssh_e, &s->sshp_e}, {&s->ubrtr_e, &s->ubrtrp_e},
                         {&s->vbrtr_e, &s->vbrtrp_e}};
    *a = *p[g][0];
    *b = *p[g][1];
}

struct Dims {
    int nx, ny;             // the local arrays (bnd_x1:bnd_x2, bnd_y1:bnd_y2)
    int i0, i1, j0, j1;     // mmm..mm, nnn..nn as 1-based positions in them
    int nx_glob, ny_glob;
};

int dims(const inmsom_bounds *b, int nz, Dims &d, const char *who)
{
    if (!b || nz < 1) return fail(INMSOM_EARG, "%s: bad bounds or nz", who);
    if (b->mmm - 1 < b->bnd_x1 || b->mm + 1 > b->bnd_x2 || b->nnn - 1 < b->bnd_y1 || b->nn + 1 > b->bnd_y2 ||
        b->mmm > b->mm || b->nnn > b->nn)
        return fail(INMSOM_EARG, "%s: mmm-1..mm+1 x nnn-1..nn+1 must lie inside the arrays", who);
    d.nx = b->bnd_x2 - b->bnd_x1 + 1;
    d.ny = b->bnd_y2 - b->bnd_y1 + 1;
    d.i0 = b->mmm - b->bnd_x1 + 1;
    d.i1 = b->mm - b->bnd_x1 + 1;
    d.j0 = b->nnn - b->bnd_y1 + 1;
    d.j1 = b->nn - b->bnd_y1 + 1;
    d.nx_glob = b->mm - b->mmm + 1;
    d.ny_glob = b->nn - b->nnn + 1;
    return INMSOM_OK;
}

int nlev(Levels l, int nz) { return l == ONE ? 1 : l == NZ ? nz : nz + 1; }

}  // namespace

extern "C" {

int inmsom_ocpwrite(const char *path, const inmsom_bounds *b, int nz, const float *lu, const float *llu,
                    const float *llv, const double *z, const double *zw, const inmsom_ctl_axes *ax,
                    inmsom_ocean_state *s)
{
    const char *who = "inmsom_ocpwrite";
    Dims d;
    CKR(dims(b, nz, d, who));
    if (!path || !lu || !llu || !llv || !ax || !s || !ax->xt || !ax->xu || !ax->yt || !ax->yv)
        return fail(INMSOM_EARG, "%s: NULL argument", who);
    const float *masks[3] = {lu, llu, llv};
    std::vector<double> zk(nz), zwk(nz + 1);
    for (int g = 0; g < 10; g++) {
        const Group &G = GROUPS[g];
        double *a, *ap;
        pair(s, g, &a, &ap);
        if (!a && !ap) continue;                     // a group the caller does not hold
        if (!a || !ap) return fail(INMSOM_EARG, "%s: %s needs both time levels", who, G.f8);
        if (G.lev == NZ && !z) return fail(INMSOM_EARG, "%s: %s needs z", who, G.f8);
        if (G.lev == NZ1 && !zw) return fail(INMSOM_EARG, "%s: %s needs zw", who, G.f8);
        const int L = nlev(G.lev, nz);
        const size_t n = (size_t)d.nx * d.ny * L;
        const int xb = d.i0 - G.dx, yb = d.j0 - G.dy;
        CKR(inmsom_wdstd8(path, G.f8, 1, a, masks[G.mask], d.nx, d.ny, L, xb, d.i1, yb, d.j1, 1, L));
        CKR(inmsom_wdstd8(path, G.f8, 2, ap, masks[G.mask], d.nx, d.ny, L, xb, d.i1, yb, d.j1, 1, L));
        // array4 = sngl(field) after wdstd8 has put the land points to 0
        std::vector<float> f4(n);
        double *t[2] = {a, ap};
        for (int k = 0; k < 2; k++) {
            for (size_t q = 0; q < n; q++) f4[q] = (float)t[k][q];
            CKR(inmsom_wdstd(path, G.f4, k + 1, f4.data(), masks[G.mask], d.nx, d.ny, L, xb, d.i1, yb, d.j1, 1,
                             L));
        }
        // z*1000.0d0 / zw*1000.0d0 as LEVELS, or a LINEAR 0.0 for one level
        const double zero = 0.0;
        const double *z0 = &zero;
        int ztype = 0;
        if (G.lev != ONE) {
            std::vector<double> &v = G.lev == NZ ? zk : zwk;
            const double *src = G.lev == NZ ? z : zw;
            for (int k = 0; k < L; k++) v[k] = src[k] * 1000.0;
            z0 = v.data();
            ztype = 1;
        }
        const std::string name = inmsom::full_file_name(path, G.ctl);
        CKR(inmsom_ctl_file_write(name.c_str(), -1.0e32f, d.nx_glob + G.dx, d.ny_glob + G.dy, L, 2, ax->xgr_type,
                                  G.dx ? ax->xu : ax->xt, ax->dxst, ax->ygr_type, G.dy ? ax->yv : ax->yt, ax->dyst,
                                  ztype, z0, 1.0, ax->calendar, ax->year, ax->month, ax->day, ax->hour, ax->minute,
                                  ax->tstep, G.title, G.var));
    }
    return INMSOM_OK;
}

int inmsom_ocpread(const char *path, const inmsom_bounds *b, int nz, const float *lu, const float *llu,
                   const float *llv, double tur_var_min, inmsom_ocean_state *s)
{
    const char *who = "inmsom_ocpread";
    Dims d;
    CKR(dims(b, nz, d, who));
    if (!path || !lu || !llu || !llv || !s) return fail(INMSOM_EARG, "%s: NULL argument", who);
    const float *masks[3] = {lu, llu, llv};
    const size_t plane = (size_t)d.nx * d.ny;
    // cyclize8_x / cyclize8_y (Service/oc_algorithms.f90:50-95, 118-135) on
    // levels 1..L of one array: the column mm into mmm-1 and mmm into mm+1
    // over all rows (the wrap cyclize8_x performs with two or more process
    // columns; on one it copies mmm into mmm-1), the row nn into nnn-1 and
    // nnn into nn+1 over all columns
    auto wrap = [&](double *f, int Lx, int Ly) {
        for (int k = 0; k < Lx && b->periodicity_x; k++)
            for (int j = 1; j <= d.ny; j++) {
                double *row = f + (size_t)k * plane + (size_t)(j - 1) * d.nx;
                const double left = row[d.i1 - 1], right = row[d.i0 - 1];
                row[d.i0 - 2] = left;
                row[d.i1] = right;
            }
        for (int k = 0; k < Ly && b->periodicity_y; k++)
            for (int i = 1; i <= d.nx; i++) {
                double *lvl = f + (size_t)k * plane + (size_t)(i - 1);
                lvl[(size_t)(d.j0 - 2) * d.nx] = lvl[(size_t)(d.j1 - 1) * d.nx];
                lvl[(size_t)d.j1 * d.nx] = lvl[(size_t)(d.j0 - 1) * d.nx];
            }
    };
    for (int g = 0; g < 10; g++) {
        const Group &G = GROUPS[g];
        double *a, *ap;
        pair(s, g, &a, &ap);
        if (!a && !ap) continue;
        if (!a || !ap) return fail(INMSOM_EARG, "%s: %s needs both time levels", who, G.f8);
        const int L = nlev(G.lev, nz);
        const int xb = d.i0 - G.dx, yb = d.j0 - G.dy;
        CKR(inmsom_rdstd8(path, G.f8, 1, a, masks[G.mask], d.nx, d.ny, L, xb, d.i1, yb, d.j1, 1, L));
        CKR(inmsom_rdstd8(path, G.f8, 2, ap, masks[G.mask], d.nx, d.ny, L, xb, d.i1, yb, d.j1, 1, L));
        // the q2 and q2l wraps: cyclize8_x over nz+1 levels, cyclize8_y
        // over nz (Control/init_pars.f90:356-367 pass nz to the y wrap)
        const int Ly = G.lev == NZ1 ? nz : L;
        wrap(a, L, Ly);
        wrap(ap, L, Ly);
    }
    // q2 = max(q2, tur_var_min) and the like, over the whole arrays
    double *tke[4] = {s->q2, s->q2p, s->q2l, s->q2lp};
    const size_t n1 = plane * (size_t)(nz + 1);
    for (double *f : tke)
        if (f)
            for (size_t q = 0; q < n1; q++) f[q] = std::max(f[q], tur_var_min);
    return INMSOM_OK;
}

}  // extern "C"
