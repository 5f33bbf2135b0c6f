/*
 * CPU oracle for the INMSOM barotropic step -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h for what this file is, how it is built and why parity with
 * the Fortran build is unpinned.  Every function cites the reference lines
 * it restates; comments mark the places where the Fortran expression order
 * decides the rounding.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LD(b) ((b)->bnd_x2 - (b)->bnd_x1 + 1)
#define NTOT(b) ((size_t)LD(b) * (size_t)((b)->bnd_y2 - (b)->bnd_y1 + 1))
/* Fortran element (m,n) of an array with the bounds in *B. */
#define I(m, n) ((size_t)((n) - B->bnd_y1) * (size_t)LDX + (size_t)((m) - B->bnd_x1))

#define SETUP(bptr)                  \
    const ora_bounds *B = (bptr);    \
    const int LDX = LD(B);           \
    (void)LDX

/* ------------------------------------------------------------------ */
/* Service/grid_construction.f90:59-112 */
void ora_gridcon(const ora_bounds *b, const float *lu, float *luu, float *luh,
                 float *llu, float *llv, float *lcu, float *lcv)
{
    SETUP(b);
    /* :59-65 luh: any of the 4 surrounding T points is ocean */
    for (int n = B->ny_start - 1; n <= B->ny_end; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end; m++)
            if (lu[I(m, n)] + lu[I(m + 1, n)] + lu[I(m, n + 1)] + lu[I(m + 1, n + 1)] > 0.5f)
                luh[I(m, n)] = 1.0f;
    /* :67-73 luu: all 4 are ocean */
    for (int n = B->ny_start - 1; n <= B->ny_end; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end; m++)
            if (lu[I(m, n)] * lu[I(m + 1, n)] * lu[I(m, n + 1)] * lu[I(m + 1, n + 1)] > 0.5f)
                luu[I(m, n)] = 1.0f;
    /* :92-112 llu/llv (either side ocean), lcu/lcv (both sides ocean) */
    for (int n = B->ny_start - 1; n <= B->ny_end; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end; m++) {
            if (lu[I(m, n)] + lu[I(m + 1, n)] > 0.5f) llu[I(m, n)] = 1.0f;
            if (lu[I(m, n)] + lu[I(m, n + 1)] > 0.5f) llv[I(m, n)] = 1.0f;
            if (lu[I(m, n)] * lu[I(m + 1, n)] > 0.5f) lcu[I(m, n)] = 1.0f;
            if (lu[I(m, n)] * lu[I(m, n + 1)] > 0.5f) lcv[I(m, n)] = 1.0f;
        }
}

/* ------------------------------------------------------------------ */
/* Service/oc_algorithms.f90:50-95.  With two or more process columns the
 * first column receives ff(mm) into ff(mmm-1) and the last receives ff(mmm)
 * into ff(mm+1): a periodic wrap of one column over the full y extent.
 * (On a single process column the routine sends to itself and copies
 * ff(mmm) into ff(mmm-1) instead; the oracle follows the wrap.) */
void ora_cyclize8_x(const ora_bounds *b, double *f)
{
    SETUP(b);
    for (int n = B->bnd_y1; n <= B->bnd_y2; n++) {
        double left = f[I(B->mm, n)], right = f[I(B->mmm, n)];
        f[I(B->mmm - 1, n)] = left;
        f[I(B->mm + 1, n)] = right;
    }
}

/* Service/oc_algorithms.f90:118-135 */
void ora_cyclize8_y(const ora_bounds *b, double *f)
{
    SETUP(b);
    for (int m = B->bnd_x1; m <= B->bnd_x2; m++) {
        f[I(m, B->nnn - 1)] = f[I(m, B->nn)];
        f[I(m, B->nn + 1)] = f[I(m, B->nnn)];
    }
}

/* syncborder_real8 (Modules/mod_mpi_parallel_tools.f90:179-252): on one
 * domain it exchanges nothing (check_p_coord, :102-113, skips neighbours
 * outside the process grid); for a strip of a 1 x P process grid the
 * caller's hook does the exchanges (rank tests only). */
static ora_exchange_fn g_exchange = 0;
static void *g_exchange_user = 0;

void ora_set_exchange(ora_exchange_fn fn, void *user)
{
    g_exchange = fn;
    g_exchange_user = user;
}

/* the "syncborder + cyclize" pair that follows every field update */
static void halo(const ora_bounds *b, double *f)
{
    if (g_exchange) g_exchange(f, g_exchange_user);
    if (b->periodicity_x) ora_cyclize8_x(b, f);
    if (b->periodicity_y) ora_cyclize8_y(b, f);
}

/* ------------------------------------------------------------------ */
/* interpolations of depth from T points, Function/depth.f90:29-66 */
static inline double h_on_u(const ora_grid *g, const double *hq, int m, int n)
{
    SETUP(&g->b);
    const float *lu = g->lu;
    double slu = (double)(lu[I(m, n)] + lu[I(m + 1, n)]);
    return (hq[I(m, n)] * g->dx[I(m, n)] * g->dy[I(m, n)] * (double)lu[I(m, n)]
            + hq[I(m + 1, n)] * g->dx[I(m + 1, n)] * g->dy[I(m + 1, n)] * (double)lu[I(m + 1, n)])
           / slu / g->dxt[I(m, n)] / g->dyh[I(m, n)];
}

static inline double h_on_v(const ora_grid *g, const double *hq, int m, int n)
{
    SETUP(&g->b);
    const float *lu = g->lu;
    double slu = (double)(lu[I(m, n)] + lu[I(m, n + 1)]);
    return (hq[I(m, n)] * g->dx[I(m, n)] * g->dy[I(m, n)] * (double)lu[I(m, n)]
            + hq[I(m, n + 1)] * g->dx[I(m, n + 1)] * g->dy[I(m, n + 1)] * (double)lu[I(m, n + 1)])
           / slu / g->dxh[I(m, n)] / g->dyt[I(m, n)];
}

static inline double h_on_h(const ora_grid *g, const double *hq, int m, int n)
{
    SETUP(&g->b);
    const float *lu = g->lu;
    /* real(4) sum of the four masks, then dble */
    double slu = (double)(lu[I(m, n)] + lu[I(m + 1, n)] + lu[I(m, n + 1)] + lu[I(m + 1, n + 1)]);
    return (hq[I(m, n)] * g->dx[I(m, n)] * g->dy[I(m, n)] * (double)lu[I(m, n)]
            + hq[I(m + 1, n)] * g->dx[I(m + 1, n)] * g->dy[I(m + 1, n)] * (double)lu[I(m + 1, n)]
            + hq[I(m, n + 1)] * g->dx[I(m, n + 1)] * g->dy[I(m, n + 1)] * (double)lu[I(m, n + 1)]
            + hq[I(m + 1, n + 1)] * g->dx[I(m + 1, n + 1)] * g->dy[I(m + 1, n + 1)] * (double)lu[I(m + 1, n + 1)])
           / slu / g->dxb[I(m, n)] / g->dyb[I(m, n)];
}

/* Function/depth.f90:2-105 */
void ora_hh_init(const ora_grid *g,
                 double *hq, double *hqp, double *hqn,
                 double *hu, double *hup, double *hun,
                 double *hv, double *hvp, double *hvn,
                 double *hh, double *hhp, double *hhn,
                 const double *sh, const double *shp, const double *h_r)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
    const double ffs = (double)g->full_free_surface;
    /* :21-23 whole-array assignments */
    for (size_t i = 0; i < nt; i++) {
        hq[i] = h_r[i] + sh[i] * ffs;
        hqp[i] = h_r[i] + shp[i] * ffs;
        hqn[i] = h_r[i];
    }
    /* :25-70 */
#pragma omp parallel for
    for (int n = B->ny_start - 1; n <= B->ny_end; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end; m++) {
            if (g->llu[I(m, n)] > 0.5f) {
                hu[I(m, n)] = h_on_u(g, hq, m, n);
                hup[I(m, n)] = h_on_u(g, hqp, m, n);
                hun[I(m, n)] = h_on_u(g, hqn, m, n);
            }
            if (g->llv[I(m, n)] > 0.5f) {
                hv[I(m, n)] = h_on_v(g, hq, m, n);
                hvp[I(m, n)] = h_on_v(g, hqp, m, n);
                hvn[I(m, n)] = h_on_v(g, hqn, m, n);
            }
            if (g->luh[I(m, n)] > 0.5f) {
                hh[I(m, n)] = h_on_h(g, hq, m, n);
                hhp[I(m, n)] = h_on_h(g, hqp, m, n);
                hhn[I(m, n)] = h_on_h(g, hqn, m, n);
            }
        }
    /* :72-104 */
    double *fs[9] = {hu, hup, hun, hv, hvp, hvn, hh, hhp, hhn};
    for (int k = 0; k < 9; k++) halo(B, fs[k]);
}

/* Function/depth.f90:108-170 */
void ora_hh_update(const ora_grid *g, double *hqn, double *hun, double *hvn,
                   double *hhn, const double *sh, const double *h_r)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
    for (size_t i = 0; i < nt; i++) hqn[i] = h_r[i] + sh[i]; /* :121 */
#pragma omp parallel for
    for (int n = B->ny_start - 1; n <= B->ny_end; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end; m++) {
            if (g->llu[I(m, n)] > 0.5f) hun[I(m, n)] = h_on_u(g, hqn, m, n);
            if (g->llv[I(m, n)] > 0.5f) hvn[I(m, n)] = h_on_v(g, hqn, m, n);
            if (g->luh[I(m, n)] > 0.5f) hhn[I(m, n)] = h_on_h(g, hqn, m, n);
        }
    halo(B, hun);
    halo(B, hvn);
    halo(B, hhn);
}

/* Robert-Asselin step shared by Function/depth.f90:196-211 and
 * Function/vel_ssh.f90:594-606: f + ts*(fn - 2f + fp)/2/nstep, evaluated as
 * f + (((ts*((fn - 2f) + fp))/2)/nstep). */
static inline double asselin(double ts, double f, double fn, double fp, double nstep)
{
    return f + ts * (fn - 2.0 * f + fp) / 2.0 / nstep;
}

/* Function/depth.f90:174-220 */
void ora_hh_shift(const ora_grid *g,
                  double *hq, double *hqp, double *hqn,
                  double *hu, double *hup, double *hun,
                  double *hv, double *hvp, double *hvn,
                  double *hh, double *hhp, double *hhn, int nstep)
{
    SETUP(&g->b);
    const double ts = g->time_smooth, ns = (double)nstep;
#pragma omp parallel for
    for (int n = B->ny_start - 1; n <= B->ny_end + 1; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end + 1; m++) {
            size_t i = I(m, n);
            if (g->llu[i] > 0.5f) { hup[i] = asselin(ts, hu[i], hun[i], hup[i], ns); hu[i] = hun[i]; }
            if (g->llv[i] > 0.5f) { hvp[i] = asselin(ts, hv[i], hvn[i], hvp[i], ns); hv[i] = hvn[i]; }
            if (g->lu[i] > 0.5f)  { hqp[i] = asselin(ts, hq[i], hqn[i], hqp[i], ns); hq[i] = hqn[i]; }
            if (g->luh[i] > 0.5f) { hhp[i] = asselin(ts, hh[i], hhn[i], hhp[i], ns); hh[i] = hhn[i]; }
        }
}

/* ------------------------------------------------------------------ */
/* Function/mixing.f90:115-168 */
void ora_stress_components(const ora_grid *g, const double *u, const double *v,
                           double *str_t, double *str_s)
{
    SETUP(&g->b);
    const double *dx = g->dx, *dy = g->dy, *dxh = g->dxh, *dyh = g->dyh;
    const double *dxt = g->dxt, *dyt = g->dyt, *dxb = g->dxb, *dyb = g->dyb;
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++)
            if (g->lu[I(m, n)] > 0.5f)
                /* :134-135 */
                str_t[I(m, n)] = dy[I(m, n)] / dx[I(m, n)] * (u[I(m, n)] / dyh[I(m, n)] - u[I(m - 1, n)] / dyh[I(m - 1, n)])
                               - dx[I(m, n)] / dy[I(m, n)] * (v[I(m, n)] / dxh[I(m, n)] - v[I(m, n - 1)] / dxh[I(m, n - 1)]);
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++)
            if (g->luu[I(m, n)] > 0.5f)
                /* :147-148 */
                str_s[I(m, n)] = dxb[I(m, n)] / dyb[I(m, n)] * (u[I(m, n + 1)] / dxt[I(m, n + 1)] - u[I(m, n)] / dxt[I(m, n)])
                               + dyb[I(m, n)] / dxb[I(m, n)] * (v[I(m + 1, n)] / dyt[I(m + 1, n)] - v[I(m, n)] / dyt[I(m, n)]);
    halo(B, str_t);
    halo(B, str_s);
}

/* Function/mixing.f90:171-219 (one level) */
void ora_smagorinsky_coeff(const ora_grid *g, double visc2, double dift,
                           const double *str_t, const double *str_s,
                           double *amts, double *amuv, double vonkarman,
                           double pi)
{
    SETUP(&g->b);
    const double prandtl = 0.1; /* :177 */
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++)
            if (g->lu[I(m, n)] > 0.5f) {
                double s0 = str_s[I(m, n)], s1 = str_s[I(m - 1, n)];
                double s2 = str_s[I(m, n - 1)], s3 = str_s[I(m - 1, n - 1)];
                double str_s2 = (s0 * s0 + s1 * s1 + s2 * s2 + s3 * s3) / 4.0;
                double k = vonkarman / pi;
                double st = str_t[I(m, n)];
                double mu_smag = k * k * g->dx[I(m, n)] * g->dy[I(m, n)] * sqrt(st * st + str_s2);
                amuv[I(m, n)] = visc2 + mu_smag;
                amts[I(m, n)] = dift + mu_smag * prandtl;
            }
    halo(B, amuv);
    halo(B, amts);
}

/* ------------------------------------------------------------------ */
/* Function/vel_ssh.f90:2-114 */
void ora_uv_trans(const ora_grid *g, const double *u, const double *v,
                  double *vort, const double *hq, const double *hu,
                  const double *hv, const double *hh, double *rhsx,
                  double *rhsy)
{
    SETUP(&g->b);
    (void)hq;
    const double *dxt = g->dxt, *dyt = g->dyt, *dxb = g->dxb, *dyb = g->dyb;
    const double *dxh = g->dxh, *dyh = g->dyh;
    /* :30-42 */
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++)
            if (g->luu[I(m, n)] > 0.5f)
                vort[I(m, n)] = (v[I(m + 1, n)] * dyt[I(m + 1, n)] - v[I(m, n)] * dyt[I(m, n)])
                              - (u[I(m, n + 1)] * dxt[I(m, n + 1)] - u[I(m, n)] * dxt[I(m, n)])
                              - ((v[I(m + 1, n)] - v[I(m, n)]) * dyb[I(m, n)] - (u[I(m, n + 1)] - u[I(m, n)]) * dxb[I(m, n)]);
    halo(B, vort); /* :44-52 */
    /* :54-109 */
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            if (g->lcu[I(m, n)] > 0.5f) {
                /* :63-77; "(a)/2.0d0*(b)/2.0d0" rounds as ((a/2)*b)/2 */
                double fx_p = (u[I(m, n)] * dyh[I(m, n)] * hu[I(m, n)] + u[I(m + 1, n)] * dyh[I(m + 1, n)] * hu[I(m + 1, n)]) / 2.0
                              * (u[I(m, n)] + u[I(m + 1, n)]) / 2.0;
                double fx_m = (u[I(m, n)] * dyh[I(m, n)] * hu[I(m, n)] + u[I(m - 1, n)] * dyh[I(m - 1, n)] * hu[I(m - 1, n)]) / 2.0
                              * (u[I(m, n)] + u[I(m - 1, n)]) / 2.0;
                double fy_p = (v[I(m, n)] * dxh[I(m, n)] * hv[I(m, n)] + v[I(m + 1, n)] * dxh[I(m + 1, n)] * hv[I(m + 1, n)]) / 2.0
                              * (u[I(m, n + 1)] + u[I(m, n)]) / 2.0 * (double)g->luu[I(m, n)];
                double fy_m = (v[I(m, n - 1)] * dxh[I(m, n - 1)] * hv[I(m, n - 1)] + v[I(m + 1, n - 1)] * dxh[I(m + 1, n - 1)] * hv[I(m + 1, n - 1)]) / 2.0
                              * (u[I(m, n - 1)] + u[I(m, n)]) / 2.0 * (double)g->luu[I(m, n - 1)];
                rhsx[I(m, n)] = -(fx_p - fx_m + fy_p - fy_m)
                                + (vort[I(m, n)] * hh[I(m, n)] * (v[I(m + 1, n)] + v[I(m, n)])
                                   + vort[I(m, n - 1)] * hh[I(m, n - 1)] * (v[I(m + 1, n - 1)] + v[I(m, n - 1)])) / 4.0;
            }
            if (g->lcv[I(m, n)] > 0.5f) {
                /* :88-102 */
                double fy_p = (v[I(m, n)] * dxh[I(m, n)] * hv[I(m, n)] + v[I(m, n + 1)] * dxh[I(m, n + 1)] * hv[I(m, n + 1)]) / 2.0
                              * (v[I(m, n)] + v[I(m, n + 1)]) / 2.0;
                double fy_m = (v[I(m, n)] * dxh[I(m, n)] * hv[I(m, n)] + v[I(m, n - 1)] * dxh[I(m, n - 1)] * hv[I(m, n - 1)]) / 2.0
                              * (v[I(m, n)] + v[I(m, n - 1)]) / 2.0;
                double fx_p = (u[I(m, n)] * dyh[I(m, n)] * hu[I(m, n)] + u[I(m, n + 1)] * dyh[I(m, n + 1)] * hu[I(m, n + 1)]) / 2.0
                              * (v[I(m + 1, n)] + v[I(m, n)]) / 2.0;
                double fx_m = (u[I(m - 1, n)] * dyh[I(m - 1, n)] * hu[I(m - 1, n)] + u[I(m - 1, n + 1)] * dyh[I(m - 1, n + 1)] * hu[I(m - 1, n + 1)]) / 2.0
                              * (v[I(m - 1, n)] + v[I(m, n)]) / 2.0;
                rhsy[I(m, n)] = -(fx_p - fx_m + fy_p - fy_m)
                                - (vort[I(m, n)] * hh[I(m, n)] * (u[I(m, n + 1)] + u[I(m, n)])
                                   + vort[I(m - 1, n)] * hh[I(m - 1, n)] * (u[I(m - 1, n + 1)] + u[I(m - 1, n)])) / 4.0;
            }
        }
}

/* the stress-divergence expressions of Function/vel_ssh.f90:153-156 and
 * :169-172 (also :228-231, :245-248, :286-289, :302-305) */
static inline double diff_x(const ora_grid *g, const double *mu, const double *str_t,
                            const double *str_s, const double *hq, const double *hh,
                            int m, int n)
{
    SETUP(&g->b);
    const double *dy = g->dy, *dyh = g->dyh, *dxb = g->dxb, *dxt = g->dxt;
    double muh_p = (mu[I(m, n)] + mu[I(m + 1, n)] + mu[I(m, n + 1)] + mu[I(m + 1, n + 1)]) / 4.0;
    double muh_m = (mu[I(m, n)] + mu[I(m + 1, n)] + mu[I(m, n - 1)] + mu[I(m + 1, n - 1)]) / 4.0;
    double dy1 = dy[I(m + 1, n)], dy0 = dy[I(m, n)], db0 = dxb[I(m, n)], db1 = dxb[I(m, n - 1)];
    return (dy1 * dy1 * mu[I(m + 1, n)] * hq[I(m + 1, n)] * str_t[I(m + 1, n)]
            - dy0 * dy0 * mu[I(m, n)] * hq[I(m, n)] * str_t[I(m, n)]) / dyh[I(m, n)]
           + (db0 * db0 * muh_p * hh[I(m, n)] * str_s[I(m, n)]
              - db1 * db1 * muh_m * hh[I(m, n - 1)] * str_s[I(m, n - 1)]) / dxt[I(m, n)];
}

static inline double diff_y_t(const ora_grid *g, const double *mu, const double *str_t,
                              const double *hq, int m, int n)
{
    SETUP(&g->b);
    const double *dx = g->dx;
    double dx1 = dx[I(m, n + 1)], dx0 = dx[I(m, n)];
    return (dx1 * dx1 * mu[I(m, n + 1)] * hq[I(m, n + 1)] * str_t[I(m, n + 1)]
            - dx0 * dx0 * mu[I(m, n)] * hq[I(m, n)] * str_t[I(m, n)]) / g->dxh[I(m, n)];
}

static inline double diff_y_s(const ora_grid *g, const double *mu, const double *str_s,
                              const double *hh, int m, int n)
{
    SETUP(&g->b);
    const double *dyb = g->dyb;
    double muh_p = (mu[I(m, n)] + mu[I(m + 1, n)] + mu[I(m, n + 1)] + mu[I(m + 1, n + 1)]) / 4.0;
    double muh_m = (mu[I(m, n)] + mu[I(m - 1, n)] + mu[I(m, n + 1)] + mu[I(m - 1, n + 1)]) / 4.0;
    double db0 = dyb[I(m, n)], db1 = dyb[I(m - 1, n)];
    return (db0 * db0 * muh_p * hh[I(m, n)] * str_s[I(m, n)]
            - db1 * db1 * muh_m * hh[I(m - 1, n)] * str_s[I(m - 1, n)]) / g->dyt[I(m, n)];
}

/* Function/vel_ssh.f90:117-184 */
void ora_uv_diff2(const ora_grid *g, const double *mu, const double *str_t,
                  const double *str_s, const double *hq, const double *hu,
                  const double *hv, const double *hh, double *rhsx,
                  double *rhsy)
{
    SETUP(&g->b);
    (void)hu;
    (void)hv;
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            if (g->lcu[I(m, n)] > 0.5f)
                rhsx[I(m, n)] = diff_x(g, mu, str_t, str_s, hq, hh, m, n);
            if (g->lcv[I(m, n)] > 0.5f)
                /* :169-172: -(A-B)/dxh + (C-D)/dyt */
                rhsy[I(m, n)] = -diff_y_t(g, mu, str_t, hq, m, n) + diff_y_s(g, mu, str_s, hh, m, n);
        }
}

/* Function/vel_ssh.f90:187-317 */
void ora_uv_diff4(const ora_grid *g, const double *mu, double *str_t,
                  double *str_s, double *fx, double *fy, const double *hq,
                  const double *hu, const double *hv, const double *hh,
                  double *rhsx, double *rhsy)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
    memset(fx, 0, nt * sizeof(double)); /* :213-214 */
    memset(fy, 0, nt * sizeof(double));
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            size_t i = I(m, n);
            if (g->lcu[i] > 0.5f) {
                fx[i] = diff_x(g, mu, str_t, str_s, hq, hh, m, n);
                fx[i] = -fx[i] / hu[i] / g->dxt[i] / g->dyh[i]; /* :232 */
            }
            if (g->lcv[i] > 0.5f) {
                fy[i] = -diff_y_t(g, mu, str_t, hq, m, n) + diff_y_s(g, mu, str_s, hh, m, n);
                fy[i] = -fy[i] / hv[i] / g->dxh[i] / g->dyt[i]; /* :249 */
            }
        }
    halo(B, fx); /* :259-270 */
    halo(B, fy);
    ora_stress_components(g, fx, fy, str_t, str_s); /* :272 */
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            size_t i = I(m, n);
            if (g->lcu[i] > 0.5f) {
                /* :286-289: RHSx + (A-B)/dyh + (C-D)/dxt, left to right */
                const double *dy = g->dy, *dyh = g->dyh, *dxb = g->dxb, *dxt = g->dxt;
                double muh_p = (mu[I(m, n)] + mu[I(m + 1, n)] + mu[I(m, n + 1)] + mu[I(m + 1, n + 1)]) / 4.0;
                double muh_m = (mu[I(m, n)] + mu[I(m + 1, n)] + mu[I(m, n - 1)] + mu[I(m + 1, n - 1)]) / 4.0;
                double dy1 = dy[I(m + 1, n)], dy0 = dy[I(m, n)], db0 = dxb[I(m, n)], db1 = dxb[I(m, n - 1)];
                rhsx[i] = rhsx[i]
                          + (dy1 * dy1 * mu[I(m + 1, n)] * hq[I(m + 1, n)] * str_t[I(m + 1, n)]
                             - dy0 * dy0 * mu[I(m, n)] * hq[I(m, n)] * str_t[I(m, n)]) / dyh[I(m, n)]
                          + (db0 * db0 * muh_p * hh[I(m, n)] * str_s[I(m, n)]
                             - db1 * db1 * muh_m * hh[I(m, n - 1)] * str_s[I(m, n - 1)]) / dxt[I(m, n)];
            }
            if (g->lcv[i] > 0.5f)
                /* :302-305: RHSy - (A-B)/dxh + (C-D)/dyt */
                rhsy[i] = rhsy[i] - diff_y_t(g, mu, str_t, hq, m, n) + diff_y_s(g, mu, str_s, hh, m, n);
        }
}

/* ------------------------------------------------------------------ */
/* Function/vel_ssh.f90:379-679 */
void ora_barotropic_dynamics(const ora_grid *g, double tau, int nstep, int ksw4,
                             double *ubrtr_e, double *ubrtrp_e,
                             double *vbrtr_e, double *vbrtrp_e,
                             double *ssh_e, double *sshp_e,
                             double *ubrtr_i, double *vbrtr_i,
                             double *ssh4gradx, double *ssh4grady,
                             const double *rhsx, const double *rhsy,
                             const double *wflux, const double *mu,
                             const double *mu4, double *vort,
                             double *str_t2d, double *str_s2d,
                             double *fx, double *fy, const double *rdis,
                             double *rhsx_adv, double *rhsy_adv,
                             double *rhsx_dif, double *rhsy_dif)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
    const size_t bytes = nt * sizeof(double);
    const double grav = g->free_fall_acc, rho = g->ref_den, ts = g->time_smooth;
    const double ffs = (double)g->full_free_surface;
    const double *dx = g->dx, *dy = g->dy, *dxt = g->dxt, *dyt = g->dyt;
    const double *dxh = g->dxh, *dyh = g->dyh, *dxb = g->dxb, *dyb = g->dyb;
    const double *rlh = g->rlh_s;

    /* :454-462 work arrays */
    double *u = malloc(bytes), *v = malloc(bytes), *ssh = malloc(bytes);
    double *up = malloc(bytes), *vp = malloc(bytes), *sshp = malloc(bytes);
    double *un = malloc(bytes), *vn = malloc(bytes), *sshn = malloc(bytes);

    const double tau_inner = tau / (double)nstep; /* :465 */
    memset(un, 0, bytes); /* :467-469 */
    memset(vn, 0, bytes);
    memset(sshn, 0, bytes);
    memcpy(up, ubrtrp_e, bytes); /* :471-477 */
    memcpy(vp, vbrtrp_e, bytes);
    memcpy(sshp, sshp_e, bytes);
    memcpy(u, ubrtr_e, bytes);
    memcpy(v, vbrtr_e, bytes);
    memcpy(ssh, ssh_e, bytes);
    memset(ubrtr_i, 0, bytes); /* :479-482 */
    memset(vbrtr_i, 0, bytes);
    memset(ssh4gradx, 0, bytes);
    memset(ssh4grady, 0, bytes);

    const double four_nstep = (double)(4 * nstep);
    for (int step = 1; step <= 2 * nstep; step++) {
        /* :487-499 continuity */
#pragma omp parallel for
        for (int n = B->ny_start; n <= B->ny_end; n++)
            for (int m = B->nx_start; m <= B->nx_end; m++)
                if (g->lu[I(m, n)] > 0.5f)
                    sshn[I(m, n)] = sshp[I(m, n)] + 2.0 * tau_inner * (wflux[I(m, n)] / rho * ffs
                        - (u[I(m, n)] * g->hhu_e[I(m, n)] * dyh[I(m, n)] - u[I(m - 1, n)] * g->hhu_e[I(m - 1, n)] * dyh[I(m - 1, n)]
                           + v[I(m, n)] * g->hhv_e[I(m, n)] * dxh[I(m, n)] - v[I(m, n - 1)] * g->hhv_e[I(m, n - 1)] * dxh[I(m, n - 1)])
                          / (dx[I(m, n)] * dy[I(m, n)]));
        halo(B, sshn); /* :501-509 */
        if (g->full_free_surface > 0) /* :511-513 */
            ora_hh_update(g, g->hhqn_e, g->hhun_e, g->hhvn_e, g->hhhn_e, sshn, g->hhq_rest);
        ora_stress_components(g, up, vp, str_t2d, str_s2d); /* :516 */
        ora_uv_trans(g, u, v, vort, g->hhq_e, g->hhu_e, g->hhv_e, g->hhh_e, rhsx_adv, rhsy_adv); /* :518-520 */
        ora_uv_diff2(g, mu, str_t2d, str_s2d, g->hhq_e, g->hhu_e, g->hhv_e, g->hhh_e, rhsx_dif, rhsy_dif); /* :521-523 */
        if (ksw4 > 0) /* :525-529 */
            ora_uv_diff4(g, mu4, str_t2d, str_s2d, fx, fy, g->hhq_e, g->hhu_e, g->hhv_e, g->hhh_e, rhsx_dif, rhsy_dif);

        /* :531-573 momentum */
#pragma omp parallel for
        for (int n = B->ny_start; n <= B->ny_end; n++)
            for (int m = B->nx_start; m <= B->nx_end; m++) {
                size_t i = I(m, n);
                if (g->lcu[i] > 0.5f) {
                    double bp = g->hhun_e[i] * dxt[i] * dyh[i] / 2.0 / tau_inner;
                    double bp0 = g->hhup_e[i] * dxt[i] * dyh[i] / 2.0 / tau_inner;
                    double slx = -grav * (ssh[I(m + 1, n)] - ssh[i]) * dyh[i] * g->hhu_e[i];
                    double slxn = -grav * (sshn[I(m + 1, n)] - sshn[i]) * dyh[i] * g->hhun_e[i];
                    double grx = rhsx[i] + slx + rhsx_dif[i] + rhsx_adv[i]
                                 - (rdis[i] + rdis[I(m + 1, n)]) / 2.0 * up[i] * dxt[i] * dyh[i] * g->hhu_e[i]
                                 + (rlh[i] * g->hhh_e[i] * dxb[i] * dyb[i] * (v[I(m + 1, n)] + v[i])
                                    + rlh[I(m, n - 1)] * g->hhh_e[I(m, n - 1)] * dxb[I(m, n - 1)] * dyb[I(m, n - 1)]
                                      * (v[I(m + 1, n - 1)] + v[I(m, n - 1)])) / 4.0;
                    un[i] = (up[i] * bp0 + grx) / bp;
                    ubrtr_i[i] = ubrtr_i[i] + (u[i] * g->hhu_e[i] + un[i] * g->hhun_e[i]) / four_nstep;
                    ssh4gradx[i] = ssh4gradx[i] + (slx + slxn) / four_nstep;
                }
                if (g->lcv[i] > 0.5f) {
                    double bp = g->hhvn_e[i] * dyt[i] * dxh[i] / 2.0 / tau_inner;
                    double bp0 = g->hhvp_e[i] * dyt[i] * dxh[i] / 2.0 / tau_inner;
                    double sly = -grav * (ssh[I(m, n + 1)] - ssh[i]) * dxh[i] * g->hhv_e[i];
                    double slyn = -grav * (sshn[I(m, n + 1)] - sshn[i]) * dxh[i] * g->hhvn_e[i];
                    double gry = rhsy[i] + sly + rhsy_dif[i] + rhsy_adv[i]
                                 - (rdis[i] + rdis[I(m, n + 1)]) / 2.0 * vp[i] * dxh[i] * dyt[i] * g->hhv_e[i]
                                 - (rlh[i] * g->hhh_e[i] * dxb[i] * dyb[i] * (u[I(m, n + 1)] + u[i])
                                    + rlh[I(m - 1, n)] * g->hhh_e[I(m - 1, n)] * dxb[I(m - 1, n)] * dyb[I(m - 1, n)]
                                      * (u[I(m - 1, n + 1)] + u[I(m - 1, n)])) / 4.0;
                    vn[i] = (vp[i] * bp0 + gry) / bp;
                    vbrtr_i[i] = vbrtr_i[i] + (v[i] * g->hhv_e[i] + vn[i] * g->hhvn_e[i]) / four_nstep;
                    ssh4grady[i] = ssh4grady[i] + (sly + slyn) / four_nstep;
                }
            }
        halo(B, un); /* :575-586 */
        halo(B, vn);

        /* :589-612 Robert-Asselin filter and time shift, halo-inclusive */
        const double ns = (double)nstep;
#pragma omp parallel for
        for (int n = B->ny_start - 1; n <= B->ny_end + 1; n++)
            for (int m = B->nx_start - 1; m <= B->nx_end + 1; m++) {
                size_t i = I(m, n);
                if (g->lu[i] > 0.5f) { sshp[i] = asselin(ts, ssh[i], sshn[i], sshp[i], ns); ssh[i] = sshn[i]; }
                if (g->lcu[i] > 0.5f) { up[i] = asselin(ts, u[i], un[i], up[i], ns); u[i] = un[i]; }
                if (g->lcv[i] > 0.5f) { vp[i] = asselin(ts, v[i], vn[i], vp[i], ns); v[i] = vn[i]; }
            }
        if (g->full_free_surface > 0) /* :614-619 */
            ora_hh_shift(g, g->hhq_e, g->hhqp_e, g->hhqn_e, g->hhu_e, g->hhup_e, g->hhun_e,
                         g->hhv_e, g->hhvp_e, g->hhvn_e, g->hhh_e, g->hhhp_e, g->hhhn_e, nstep);
        if (step == nstep) { /* :638-648 */
            memcpy(ubrtrp_e, up, bytes);
            memcpy(vbrtrp_e, vp, bytes);
            memcpy(sshp_e, sshp, bytes);
            memcpy(ubrtr_e, u, bytes);
            memcpy(vbrtr_e, v, bytes);
            memcpy(ssh_e, ssh, bytes);
        }
    }
    halo(B, ubrtr_i); /* :652-666 */
    halo(B, vbrtr_i);
    if (g->full_free_surface > 0) /* :668-675 */
        ora_hh_init(g, g->hhq_e, g->hhqp_e, g->hhqn_e, g->hhu_e, g->hhup_e, g->hhun_e,
                    g->hhv_e, g->hhvp_e, g->hhvn_e, g->hhh_e, g->hhhp_e, g->hhhn_e,
                    ssh_e, sshp_e, g->hhq_rest);
    (void)ffs;
    free(sshn); free(vn); free(un); free(sshp); free(vp); free(up); free(ssh); free(v); free(u);
}

/* Function/vel_ssh.f90:682-751 */
void ora_ssh_internal(const ora_grid *g, double tau, double *ssh_i,
                      double *sshp_i, const double *u, const double *v,
                      const double *wflux, double *hhqn, double *hhun,
                      double *hhvn, double *hhhn)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
    const double rho = g->ref_den, ffs = (double)g->full_free_surface, ts = g->time_smooth;
    double *ssh_new = calloc(nt, sizeof(double)); /* :704-705 */
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++)
            if (g->lu[I(m, n)] > 0.5f)
                ssh_new[I(m, n)] = sshp_i[I(m, n)] + 2.0 * tau * (wflux[I(m, n)] / rho * ffs
                    - (u[I(m, n)] * g->dyh[I(m, n)] - u[I(m - 1, n)] * g->dyh[I(m - 1, n)]
                       + v[I(m, n)] * g->dxh[I(m, n)] - v[I(m, n - 1)] * g->dxh[I(m, n - 1)])
                      / (g->dx[I(m, n)] * g->dy[I(m, n)]));
    halo(B, ssh_new); /* :721-729 */
    if (g->full_free_surface > 0) /* :733-735 */
        ora_hh_update(g, hhqn, hhun, hhvn, hhhn, ssh_new, g->hhq_rest);
#pragma omp parallel for
    for (int n = B->ny_start - 1; n <= B->ny_end + 1; n++) /* :738-749 */
        for (int m = B->nx_start - 1; m <= B->nx_end + 1; m++) {
            size_t i = I(m, n);
            if (g->lu[i] > 0.5f) {
                sshp_i[i] = ssh_i[i] + ts * (ssh_new[i] - 2.0 * ssh_i[i] + sshp_i[i]) / 2.0;
                ssh_i[i] = ssh_new[i];
            }
        }
    free(ssh_new);
}

/* ------------------------------------------------------------------ */
/* Control/init_pars.f90:459-481 */
void ora_r_diss(const ora_grid *g, double r_fric, double *r_diss)
{
    SETUP(&g->b);
    const double *h = g->hhq_rest, *dxt = g->dxt, *dyt = g->dyt;
    const float *lcu = g->lcu, *lcv = g->lcv;
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++)
            if (g->lu[I(m, n)] > 0.5f) {
                double a = (h[I(m + 1, n)] - h[I(m, n)]) / dxt[I(m, n)];
                double c = (h[I(m, n)] - h[I(m - 1, n)]) / dxt[I(m - 1, n)];
                double hx2 = (a * a * (double)lcu[I(m, n)] + c * c * (double)lcu[I(m - 1, n)])
                             / (double)(lcu[I(m, n)] + lcu[I(m - 1, n)]);
                double d = (h[I(m, n + 1)] - h[I(m, n)]) / dyt[I(m, n)];
                double e = (h[I(m, n)] - h[I(m, n - 1)]) / dyt[I(m, n - 1)];
                double hy2 = (d * d * (double)lcv[I(m, n)] + e * e * (double)lcv[I(m, n - 1)])
                             / (double)(lcv[I(m, n)] + lcv[I(m, n - 1)]);
                r_diss[I(m, n)] = r_fric * sqrt(hx2 + hy2);
            }
    halo(B, r_diss);
}

/* Function/fluxes.f90:29-37 */
void ora_surface_stress(const ora_grid *g, const double *taux,
                        const double *tauy, double *ssx, double *ssy)
{
    SETUP(&g->b);
    const double *dx = g->dx, *dy = g->dy, rho = g->ref_den;
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            if (g->lcu[I(m, n)] > 0.5f)
                ssx[I(m, n)] = (taux[I(m, n)] * dx[I(m, n)] * dy[I(m, n)]
                                + taux[I(m + 1, n)] * dx[I(m + 1, n)] * dy[I(m + 1, n)])
                               / rho / 2.0 / g->dxt[I(m, n)] / g->dyh[I(m, n)];
            if (g->lcv[I(m, n)] > 0.5f)
                ssy[I(m, n)] = (tauy[I(m, n)] * dx[I(m, n)] * dy[I(m, n)]
                                + tauy[I(m, n + 1)] * dx[I(m, n + 1)] * dy[I(m, n + 1)])
                               / rho / 2.0 / g->dxh[I(m, n)] / g->dyt[I(m, n)];
        }
}

static inline double opt(const double *a, size_t i) { return a ? a[i] : 0.0; }

/* Control/dyncall.f90:110-130 */
void ora_rhs2d(const ora_grid *g, double *rhsx2d, double *rhsy2d,
               const double *diff_disp_x, const double *diff_disp_y,
               const double *tran_x, const double *tran_y,
               const double *tran_disp_x, const double *tran_disp_y,
               const double *ssx, const double *ssy, const double *bsx,
               const double *bsy, const double *slpr, const double *hhu,
               const double *hhv)
{
    SETUP(&g->b);
    const double rho = g->ref_den;
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            size_t i = I(m, n);
            if (g->lcu[i] > 0.5f)
                rhsx2d[i] = rhsx2d[i] - opt(diff_disp_x, i) + opt(tran_x, i) - opt(tran_disp_x, i)
                            + (opt(ssx, i) + opt(bsx, i)) * g->dxt[i] * g->dyh[i]
                            - (opt(slpr, I(m + 1, n)) - opt(slpr, i)) * hhu[i] * g->dyh[i] / rho;
            if (g->lcv[i] > 0.5f)
                rhsy2d[i] = rhsy2d[i] - opt(diff_disp_y, i) + opt(tran_y, i) - opt(tran_disp_y, i)
                            + (opt(ssy, i) + opt(bsy, i)) * g->dyt[i] * g->dxh[i]
                            - (opt(slpr, I(m, n + 1)) - opt(slpr, i)) * hhv[i] * g->dxh[i] / rho;
        }
}

/* Service/oc_algorithms.f90:494-524 factor8: the tridiagonal system
 * a(n) f(n-1) + b(n) f(n) + c(n) f(n+1) = eta(n), n = 1..nd (0-based here),
 * forward elimination then back substitution, in the reference's order. */
static void factor8(int nd, const double *a, const double *b, const double *c, const double *eta,
                    double *rksi, double *x, double *y)
{
    x[0] = -c[0] / b[0];
    y[0] = eta[0] / b[0];
    for (int j = 1; j < nd; j++) {
        const double scr = 1.0 / (a[j] * x[j - 1] + b[j]);
        x[j] = -c[j] * scr;
        y[j] = (eta[j] - a[j] * y[j - 1]) * scr;
    }
    rksi[nd - 1] = y[nd - 1];
    for (int j = nd - 2; j >= 0; j--) rksi[j] = x[j] * rksi[j + 1] + y[j];
}

/* Function/vel_ssh.f90:794-1027 baroclinic_dynamics: implicit vertical
 * viscosity per water column (factor8), vertical advection, Coriolis, drag,
 * surface and bottom stress, then the Robert-Asselin filter.  3-D arrays
 * are (bnd_x1:bnd_x2, bnd_y1:bnd_y2, levels), levels nz (nz+1 for ww, nu);
 * dz(nz), hzt(nz+1); hh* are the internal-mode depths of basin_grid. */
void ora_baroclinic_dynamics(const ora_grid *g, int nz, const double *dz, const double *hzt, double tau,
                             double *uu, double *uup, double *vv, double *vvp, const double *ww,
                             const double *nu, const double *rhsx, const double *rhsy,
                             const double *rhsx_tran, const double *rhsy_tran, const double *pgrx,
                             const double *pgry, const double *rdis, const double *tx_surf,
                             const double *ty_surf, const double *tx_bot, const double *ty_bot,
                             const double *hhu, const double *hhup, const double *hhun, const double *hhv,
                             const double *hhvp, const double *hhvn, const double *hhh)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
#define I3(m, n, k) (I(m, n) + (size_t)((k) - 1) * nt)
    double *un = calloc(nt * (size_t)nz, sizeof(double));
    double *vn = calloc(nt * (size_t)nz, sizeof(double));
    /* :847-983 */
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++) {
        double *a = malloc(6 * (size_t)nz * sizeof(double));
        double *bb = a + nz, *c = bb + nz, *eta = c + nz, *x = eta + nz, *y = x + nz;
        double *rksi = malloc((size_t)nz * sizeof(double));
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            const size_t i = I(m, n);
            if (g->lcu[i] > 0.5f) {
                const double bp = hhun[i] * g->dxt[i] * g->dyh[i] / tau / 2.0;
                const double bp0 = hhup[i] * g->dxt[i] * g->dyh[i] / tau / 2.0;
                double dp = 0.0, dm = 0.0, fz_p = 0.0, fz_m = 0.0;
                for (int k = 1; k <= nz; k++) {
                    dm = dp;
                    fz_m = fz_p;
                    if (k < nz) {
                        dp = (nu[I3(m, n, k + 1)] + nu[I3(m + 1, n, k + 1)]) / 2.0 / hhun[i] / hzt[k] * g->dxt[i] *
                             g->dyh[i];
                        fz_p = (ww[I3(m, n, k + 1)] * g->dx[i] * g->dy[i] +
                                ww[I3(m + 1, n, k + 1)] * g->dx[I(m + 1, n)] * g->dy[I(m + 1, n)]) /
                               2.0 * (uu[I3(m, n, k)] + uu[I3(m, n, k + 1)]) / 2.0;
                    } else {
                        dp = 0.0;
                        fz_p = 0.0;
                    }
                    const int q = k - 1;
                    c[q] = k < nz ? -dp / dz[q] : 0.0;
                    a[q] = k > 1 ? -dm / dz[q] : 0.0;
                    bb[q] = k == 1 ? bp + dp / dz[q] : (k < nz ? bp + (dp + dm) / dz[q] : bp + dm / dz[q]);
                    double e = bp0 * uup[I3(m, n, k)] + rhsx[I3(m, n, k)] + rhsx_tran[I3(m, n, k)] + pgrx[i] -
                               (fz_p - fz_m) / dz[q] +
                               (g->rlh_s[i] * hhh[i] * g->dxb[i] * g->dyb[i] *
                                    (vv[I3(m + 1, n, k)] + vv[I3(m, n, k)]) +
                                g->rlh_s[I(m, n - 1)] * hhh[I(m, n - 1)] * g->dxb[I(m, n - 1)] *
                                    g->dyb[I(m, n - 1)] * (vv[I3(m + 1, n - 1, k)] + vv[I3(m, n - 1, k)])) /
                                   4.0 -
                               (rdis[i] + rdis[I(m + 1, n)]) / 2.0 * uup[I3(m, n, k)] * g->dxt[i] * g->dyh[i] *
                                   hhu[i];
                    if (k == 1) e = e + tx_surf[i] / dz[q] * g->dxt[i] * g->dyh[i];
                    if (k == nz) e = e + tx_bot[i] / dz[q] * g->dxt[i] * g->dyh[i];
                    eta[q] = e;
                }
                factor8(nz, a, bb, c, eta, rksi, x, y);
                for (int k = 1; k <= nz; k++) un[I3(m, n, k)] = rksi[k - 1];
            }
            if (g->lcv[i] > 0.5f) {
                const double bp = hhvn[i] * g->dxh[i] * g->dyt[i] / tau / 2.0;
                const double bp0 = hhvp[i] * g->dxh[i] * g->dyt[i] / tau / 2.0;
                double dp = 0.0, dm = 0.0, fz_p = 0.0, fz_m = 0.0;
                for (int k = 1; k <= nz; k++) {
                    dm = dp;
                    fz_m = fz_p;
                    if (k < nz) {
                        dp = (nu[I3(m, n, k + 1)] + nu[I3(m, n + 1, k + 1)]) / 2.0 / hhvn[i] / hzt[k] * g->dxh[i] *
                             g->dyt[i];
                        fz_p = (ww[I3(m, n, k + 1)] * g->dx[i] * g->dy[i] +
                                ww[I3(m, n + 1, k + 1)] * g->dx[I(m, n + 1)] * g->dy[I(m, n + 1)]) /
                               2.0 * (vv[I3(m, n, k)] + vv[I3(m, n, k + 1)]) / 2.0;
                    } else {
                        dp = 0.0;
                        fz_p = 0.0;
                    }
                    const int q = k - 1;
                    c[q] = k < nz ? -dp / dz[q] : 0.0;
                    a[q] = k > 1 ? -dm / dz[q] : 0.0;
                    bb[q] = k == 1 ? bp + dp / dz[q] : (k < nz ? bp + (dp + dm) / dz[q] : bp + dm / dz[q]);
                    double e = bp0 * vvp[I3(m, n, k)] + rhsy[I3(m, n, k)] + rhsy_tran[I3(m, n, k)] + pgry[i] -
                               (fz_p - fz_m) / dz[q] -
                               (g->rlh_s[i] * hhh[i] * g->dxb[i] * g->dyb[i] *
                                    (uu[I3(m, n + 1, k)] + uu[I3(m, n, k)]) +
                                g->rlh_s[I(m - 1, n)] * hhh[I(m - 1, n)] * g->dxb[I(m - 1, n)] *
                                    g->dyb[I(m - 1, n)] * (uu[I3(m - 1, n + 1, k)] + uu[I3(m - 1, n, k)])) /
                                   4.0 -
                               (rdis[i] + rdis[I(m, n + 1)]) / 2.0 * vvp[I3(m, n, k)] * g->dxh[i] * g->dyt[i] *
                                   hhv[i];
                    if (k == 1) e = e + ty_surf[i] / dz[q] * g->dxh[i] * g->dyt[i];
                    if (k == nz) e = e + ty_bot[i] / dz[q] * g->dxh[i] * g->dyt[i];
                    eta[q] = e;
                }
                factor8(nz, a, bb, c, eta, rksi, x, y);
                for (int k = 1; k <= nz; k++) vn[I3(m, n, k)] = rksi[k - 1];
            }
        }
        free(a);
        free(rksi);
    }
    /* :988-998 halo: no exchange on one domain; periodic wrap per level */
    for (int k = 1; k <= nz; k++) {
        if (B->periodicity_x) {
            ora_cyclize8_x(B, un + (size_t)(k - 1) * nt);
            ora_cyclize8_x(B, vn + (size_t)(k - 1) * nt);
        }
        if (B->periodicity_y) {
            ora_cyclize8_y(B, un + (size_t)(k - 1) * nt);
            ora_cyclize8_y(B, vn + (size_t)(k - 1) * nt);
        }
    }
    /* :1002-1024 Robert-Asselin filter with time shift */
    const double ts = g->time_smooth;
#pragma omp parallel for
    for (int n = B->ny_start - 1; n <= B->ny_end + 1; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end + 1; m++) {
            const size_t i = I(m, n);
            if (g->lcu[i] > 0.5f)
                for (int k = 1; k <= nz; k++) {
                    const size_t j = I3(m, n, k);
                    uup[j] = uu[j] + ts * (un[j] - 2.0 * uu[j] + uup[j]) / 2.0;
                    uu[j] = un[j];
                }
            if (g->lcv[i] > 0.5f)
                for (int k = 1; k <= nz; k++) {
                    const size_t j = I3(m, n, k);
                    vvp[j] = vv[j] + ts * (vn[j] - 2.0 * vv[j] + vvp[j]) / 2.0;
                    vv[j] = vn[j];
                }
        }
    free(un);
    free(vn);
}

/* Function/depth.f90:223-254 depth_ave: utr = sum_k u(k)*dz(k) over the
 * points of mask, and u = u - kbcl*utr there; the loop covers the arrays
 * but their outermost ring */
void ora_depth_ave(const ora_grid *g, int nz, const double *dz, double *u, double *utr, const float *mask,
                   int kbcl)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
#pragma omp parallel for
    for (int n = B->bnd_y1 + 1; n <= B->bnd_y2 - 1; n++)
        for (int m = B->bnd_x1 + 1; m <= B->bnd_x2 - 1; m++) {
            const size_t i = I(m, n);
            if (!(mask[i] > 0.5f)) continue;
            double ff0 = 0.0;
            for (int k = 1; k <= nz; k++) ff0 = ff0 + u[I3(m, n, k)] * dz[k - 1];
            utr[i] = ff0;
            for (int k = 1; k <= nz; k++) u[I3(m, n, k)] = u[I3(m, n, k)] - (double)kbcl * ff0;
        }
}

/* Control/dyncall.f90:170-183 (sign < 0: uu = uu - uu2d, the barotropic
 * component removed before vertical_velocity) and :215-229 (sign > 0:
 * uu = uu + uu2d, restored after ssh_internal), at the ocean u (v) points of
 * the interior and its one-point ring, every level */
void ora_shift_barotropic(const ora_grid *g, int nz, double *uu, double *vv, const double *uu2d,
                          const double *vv2d, int sign)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
#pragma omp parallel for
    for (int n = B->ny_start - 1; n <= B->ny_end + 1; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end + 1; m++) {
            const size_t i = I(m, n);
            if (g->lcu[i] > 0.5f)
                for (int k = 1; k <= nz; k++)
                    uu[I3(m, n, k)] = sign < 0 ? uu[I3(m, n, k)] - uu2d[i] : uu[I3(m, n, k)] + uu2d[i];
            if (g->lcv[i] > 0.5f)
                for (int k = 1; k <= nz; k++)
                    vv[I3(m, n, k)] = sign < 0 ? vv[I3(m, n, k)] - vv2d[i] : vv[I3(m, n, k)] + vv2d[i];
        }
}

/* Function/tem_sal.f90:1-422 tracer_tran_diff: one tracer's step —
 * lateral advection, isoneutral diffusion and Gent-McWilliams fluxes on u
 * and v points (:108-251), the periodic wrap of those fluxes (:253-275),
 * the implicit vertical diffusion per water column with vertical
 * advection and the fluxes' vertical parts (:277-392, factor8), and the
 * Robert-Asselin filter (:405-419).  The lateral-boundary arguments of the
 * reference (ksw_lbc, numlbc, lqpx, lqpy, ind_lbc, flbc) are not read by
 * its body and are not taken here.  ig_top/ig_bot must be 1 or 2 at the
 * ocean points (other values leave the reference's b(1)/eta(1) unset). */
void ora_tracer_tran_diff(const ora_grid *g, int nz, const double *dz, const double *hzt, double *ff, double *ffp,
                          double tau, const double *uu, const double *vv, const double *ww, const double *mu,
                          double factor_mu, const double *nu, double factor_nu, const double *slrx,
                          const double *slry, const double *slzx, const double *slzy, double az, double ar,
                          double alpha_gm, const double *ff_top, const double *ff_bot, const int *ig_top,
                          const int *ig_bot, double *flux_f_x, double *flux_f_y, const double *swbal,
                          const double *src, double src_factor, const double *hhu, const double *hhv,
                          const double *hhqn, const double *hhqp)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
    const size_t n3 = nt * (size_t)nz, n31 = nt * (size_t)(nz + 1);
    double *flux_x = calloc(n3, sizeof(double)), *flux_y = calloc(n3, sizeof(double));
    double *flux_zx = calloc(n31, sizeof(double)), *flux_zy = calloc(n31, sizeof(double));
    double *coef_zx = calloc(n31, sizeof(double)), *coef_zy = calloc(n31, sizeof(double));
    double *sfgm_zx = calloc(n31, sizeof(double)), *sfgm_zy = calloc(n31, sizeof(double));
    double *fn = calloc(n3, sizeof(double));
    memset(flux_f_x, 0, 4 * nt * sizeof(double));
    memset(flux_f_y, 0, 4 * nt * sizeof(double));
#define F4(a, m, n, c) (a)[I(m, n) + (size_t)((c) - 1) * nt]
    /* :108-251 */
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++) {
        double *flux_1d = malloc((size_t)(nz + 2) * sizeof(double)), *mu_1d = malloc((size_t)(nz + 2) * sizeof(double));
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            const size_t i = I(m, n);
            for (int V = 0; V < 2; V++) {
                const float *mk = V ? g->lcv : g->lcu;
                if (!(mk[i] > 0.5f)) continue;
                /* the far point (u: m+1, v: n+1) and the u/v-specific metrics */
                const int mf = V ? m : m + 1, nf = V ? n + 1 : n;
                const double *hh = V ? hhv : hhu, *slr = V ? slry : slrx, *slz = V ? slzy : slzx;
                const double *vel = V ? vv : uu;
                const double dside = V ? g->dxh[i] : g->dyh[i];             /* dyh (u), dxh (v) */
                const double dnorm = V ? g->dyt[i] : g->dxt[i];             /* dxt (u), dyt (v) */
                double *flux = V ? flux_y : flux_x, *fz = V ? flux_zy : flux_zx;
                double *coef = V ? coef_zy : coef_zx, *sfgm = V ? sfgm_zy : sfgm_zx;
                double *ffo = V ? flux_f_y : flux_f_x;
                for (int k = 1; k <= nz + 1; k++) flux_1d[k] = 0.0, mu_1d[k] = 0.0;
                for (int k = 2; k <= nz; k++) {
                    const double dfdz = (ffp[I3(m, n, k)] - ffp[I3(m, n, k - 1)] + ffp[I3(mf, nf, k)] -
                                         ffp[I3(mf, nf, k - 1)]) / 2.0;
                    const double dfdh = (ffp[I3(mf, nf, k)] - ffp[I3(m, n, k)] + ffp[I3(mf, nf, k - 1)] -
                                         ffp[I3(m, n, k - 1)]) / 2.0;
                    mu_1d[k] = (mu[I3(m, n, k)] + mu[I3(m, n, k - 1)] + mu[I3(mf, nf, k)] + mu[I3(mf, nf, k - 1)]) /
                               4.0 * factor_mu * dside / dnorm;
                    const double slope = ar * slr[I3(m, n, k)] + az * slz[I3(m, n, k)];
                    flux_1d[k] = mu_1d[k] * (hh[i] * dfdh * hzt[k - 1] - slope * dfdz);
                    fz[I3(m, n, k)] = mu_1d[k] * slope * dfdh;
                    coef[I3(m, n, k)] = mu_1d[k] * (slope * slope) / hh[i] / hzt[k - 1];
                    sfgm[I3(m, n, k)] = mu_1d[k] * (slr[I3(m, n, k)] - slz[I3(m, n, k)]) * alpha_gm;
                }
                for (int k = 1; k <= nz; k++) {
                    double flux_diff;
                    if (k == 1) flux_diff = flux_1d[k + 1] / hzt[k];
                    else if (k < nz) flux_diff = (flux_1d[k] + flux_1d[k + 1]) / dz[k - 1] / 2.0;
                    else flux_diff = flux_1d[k] / hzt[k - 1];
                    const double flux_adv =
                        -(vel[I3(m, n, k)] * hh[i] * dside * (ff[I3(m, n, k)] + ff[I3(mf, nf, k)]) / 2.0);
                    const double vel_gm = (sfgm[I3(m, n, k + 1)] - sfgm[I3(m, n, k)]) / dz[k - 1];
                    const double flux_gm = -(vel_gm * (ff[I3(m, n, k)] + ff[I3(mf, nf, k)]) / 2.0);
                    flux[I3(m, n, k)] = flux_adv + flux_diff + flux_gm;
                    F4(ffo, m, n, 1) = F4(ffo, m, n, 1) + dz[k - 1] * (flux_adv + flux_diff + flux_gm);
                    F4(ffo, m, n, 2) = F4(ffo, m, n, 2) + dz[k - 1] * flux_adv;
                    F4(ffo, m, n, 3) = F4(ffo, m, n, 3) + dz[k - 1] * flux_diff;
                    F4(ffo, m, n, 4) = F4(ffo, m, n, 4) + dz[k - 1] * flux_gm;
                }
            }
        }
        free(flux_1d);
        free(mu_1d);
    }
    /* :253-275: x-fluxes wrap in x, y-fluxes in y */
    for (int k = 1; k <= nz + 1; k++) {
        const size_t o = (size_t)(k - 1) * nt;
        if (B->periodicity_x) {
            if (k <= nz) ora_cyclize8_x(B, flux_x + o);
            ora_cyclize8_x(B, flux_zx + o);
            ora_cyclize8_x(B, coef_zx + o);
            ora_cyclize8_x(B, sfgm_zx + o);
        }
        if (B->periodicity_y) {
            if (k <= nz) ora_cyclize8_y(B, flux_y + o);
            ora_cyclize8_y(B, flux_zy + o);
            ora_cyclize8_y(B, coef_zy + o);
            ora_cyclize8_y(B, sfgm_zy + o);
        }
    }
    /* :277-392 */
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++) {
        double *a = malloc(6 * (size_t)nz * sizeof(double));
        double *bb = a + nz, *c = bb + nz, *eta = c + nz, *x = eta + nz, *y = x + nz;
        double *rksi = malloc((size_t)nz * sizeof(double));
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            const size_t i = I(m, n);
            if (!(g->lu[i] > 0.5f)) continue;
            const double dxy_x = g->dx[i], dxy_y = g->dy[i];
            const double bp = hhqn[i] * dxy_x * dxy_y / tau / 2.0;
            const double bp0 = hhqp[i] * dxy_x * dxy_y / tau / 2.0;
            const double cu = (double)fmaxf(g->lcu[i] + g->lcu[I(m - 1, n)], 1e-10f);
            const double cv = (double)fmaxf(g->lcv[i] + g->lcv[I(m, n - 1)], 1e-10f);
            double fz_p = 0.0, fz_m, dp = 0.0, dm;
            for (int k = 1; k <= nz; k++) {
                const int q = k - 1;
                fz_m = fz_p;
                if (k < nz) {
                    const double vel_gm = -(sfgm_zx[I3(m, n, k + 1)] - sfgm_zx[I3(m - 1, n, k + 1)] +
                                            sfgm_zy[I3(m, n, k + 1)] - sfgm_zy[I3(m, n - 1, k + 1)]);
                    fz_p = -((flux_zx[I3(m, n, k + 1)] + flux_zx[I3(m - 1, n, k + 1)]) / cu) -
                           (flux_zy[I3(m, n, k + 1)] + flux_zy[I3(m, n - 1, k + 1)]) / cv +
                           (coef_zx[I3(m, n, k + 1)] * (ffp[I3(m + 1, n, k + 1)] - ffp[I3(m + 1, n, k)]) +
                            coef_zx[I3(m - 1, n, k + 1)] * (ffp[I3(m - 1, n, k + 1)] - ffp[I3(m - 1, n, k)])) /
                               cu / 2.0 +
                           (coef_zy[I3(m, n, k + 1)] * (ffp[I3(m, n + 1, k + 1)] - ffp[I3(m, n + 1, k)]) +
                            coef_zy[I3(m, n - 1, k + 1)] * (ffp[I3(m, n - 1, k + 1)] - ffp[I3(m, n - 1, k)])) /
                               cv / 2.0 -
                           (ww[I3(m, n, k + 1)] * dxy_x * dxy_y + vel_gm) * (ff[I3(m, n, k)] + ff[I3(m, n, k + 1)]) /
                               2.0;
                } else {
                    fz_p = 0.0;
                }
                const double nu_p = nu[I3(m, n, k + 1)] * factor_nu;
                if (k == 1) dm = nu[I3(m, n, k)] * factor_nu * dxy_x * dxy_y / hhqn[i] / hzt[0];
                else dm = dp;
                if (k < nz)
                    dp = (coef_zx[I3(m, n, k + 1)] + coef_zx[I3(m - 1, n, k + 1)]) / cu / 2.0 +
                         (coef_zy[I3(m, n, k + 1)] + coef_zy[I3(m, n - 1, k + 1)]) / cv / 2.0 +
                         nu_p * dxy_x * dxy_y / hhqn[i] / hzt[k];
                else
                    dp = nu_p * dxy_x * dxy_y / hhqn[i] / hzt[k];
                const double rhs = flux_x[I3(m, n, k)] - flux_x[I3(m - 1, n, k)] + flux_y[I3(m, n, k)] -
                                   flux_y[I3(m, n - 1, k)] + (fz_p - fz_m) / dz[q] +
                                   src[I3(m, n, k)] * g->hhq_rest[i] * swbal[i] * src_factor * dxy_x * dxy_y;
                if (k == 1) {
                    c[q] = -dp / dz[q];
                    a[q] = 0.0;
                    if (ig_top[i] == 1) {
                        bb[q] = bp + (dp + dm) / dz[q];
                        eta[q] = bp0 * ffp[I3(m, n, k)] + rhs + dm * ff_top[i] / dz[q];
                    } else {
                        bb[q] = bp + dp / dz[q];
                        eta[q] = bp0 * ffp[I3(m, n, k)] + rhs + ff_top[i] / dz[q] * dxy_x * dxy_y;
                    }
                } else if (k < nz) {
                    c[q] = -dp / dz[q];
                    a[q] = -dm / dz[q];
                    bb[q] = bp + (dp + dm) / dz[q];
                    eta[q] = bp0 * ffp[I3(m, n, k)] + rhs;
                } else {
                    c[q] = 0.0;
                    a[q] = -dm / dz[q];
                    if (ig_bot[i] == 1) {
                        bb[q] = bp + (dp + dm) / dz[q];
                        eta[q] = bp0 * ffp[I3(m, n, k)] + rhs + dp * ff_bot[i] / dz[q];
                    } else {
                        bb[q] = bp + dm / dz[q];
                        eta[q] = bp0 * ffp[I3(m, n, k)] + rhs + ff_bot[i] / dz[q] * dxy_x * dxy_y;
                    }
                }
            }
            factor8(nz, a, bb, c, eta, rksi, x, y);
            for (int k = 1; k <= nz; k++) fn[I3(m, n, k)] = rksi[k - 1];
        }
        free(a);
        free(rksi);
    }
    /* :394-402 */
    for (int k = 1; k <= nz; k++) {
        if (B->periodicity_x) ora_cyclize8_x(B, fn + (size_t)(k - 1) * nt);
        if (B->periodicity_y) ora_cyclize8_y(B, fn + (size_t)(k - 1) * nt);
    }
    /* :405-419 */
    const double ts = g->time_smooth;
#pragma omp parallel for
    for (int n = B->ny_start - 1; n <= B->ny_end + 1; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end + 1; m++) {
            if (!(g->lu[I(m, n)] > 0.5f)) continue;
            for (int k = 1; k <= nz; k++) {
                const size_t j = I3(m, n, k);
                ffp[j] = ff[j] + ts * (fn[j] - 2.0 * ff[j] + ffp[j]) / 2.0;
                ff[j] = fn[j];
            }
        }
#undef F4
    free(flux_x); free(flux_y); free(flux_zx); free(flux_zy);
    free(coef_zx); free(coef_zy); free(sfgm_zx); free(sfgm_zy); free(fn);
}

/* Function/vel_ssh.f90:1030-1076 vertical_velocity: w from the continuity
 * equation, integrated from the bottom (w(nz+1) = 0), on lu points */
void ora_vertical_velocity(const ora_grid *g, int nz, const double *dz, const double *u, const double *v,
                           double *w, const double *hu, const double *hv, const double *wflux)
{
    SETUP(&g->b);
    const size_t nt = NTOT(B);
    const double ffs = (double)g->full_free_surface;
#pragma omp parallel for
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            const size_t i = I(m, n);
            if (!(g->lu[i] > 0.5f)) continue;
            w[I3(m, n, nz + 1)] = 0.0;
            for (int k = nz; k >= 1; k--)
                w[I3(m, n, k)] = w[I3(m, n, k + 1)] + dz[k - 1] / (g->dx[i] * g->dy[i]) *
                                                          (u[I3(m, n, k)] * hu[i] * g->dyh[i] -
                                                           u[I3(m - 1, n, k)] * hu[I(m - 1, n)] * g->dyh[I(m - 1, n)] +
                                                           v[I3(m, n, k)] * hv[i] * g->dxh[i] -
                                                           v[I3(m, n - 1, k)] * hv[I(m, n - 1)] * g->dxh[I(m, n - 1)] +
                                                           wflux[i] / g->ref_den * ffs);
        }
    for (int k = 1; k <= nz + 1; k++) {
        if (B->periodicity_x) ora_cyclize8_x(B, w + (size_t)(k - 1) * nt);
        if (B->periodicity_y) ora_cyclize8_y(B, w + (size_t)(k - 1) * nt);
    }
#undef I3
}

/* Control/dyncall.f90:188-201: the corrected 2-D velocity from the time
 * means and the sea-level-pressure part of the time-mean pressure gradient,
 * over nx_start-1..nx_end+1 x ny_start-1..ny_end+1 */
void ora_velocity2d(const ora_grid *g, double *uu2d, double *vv2d, double *pgrx, double *pgry,
                    const double *ubrtr_i, const double *vbrtr_i, const double *slpr, const double *hhu,
                    const double *hhv)
{
    SETUP(&g->b);
    const double rho = g->ref_den;
#pragma omp parallel for
    for (int n = B->ny_start - 1; n <= B->ny_end + 1; n++)
        for (int m = B->nx_start - 1; m <= B->nx_end + 1; m++) {
            size_t i = I(m, n);
            if (g->lcu[i] > 0.5f) {
                uu2d[i] = ubrtr_i[i] / hhu[i];
                pgrx[i] = pgrx[i] - (slpr[I(m + 1, n)] - slpr[i]) * hhu[i] * g->dyh[i] / rho;
            }
            if (g->lcv[i] > 0.5f) {
                vv2d[i] = vbrtr_i[i] / hhv[i];
                pgry[i] = pgry[i] - (slpr[I(m, n + 1)] - slpr[i]) * hhv[i] * g->dxh[i] / rho;
            }
        }
}

/* Control/dyncall.f90:452-516 (barotropic fields only) */
long ora_guard(const ora_grid *g, const double *ssh, const double *u,
               const double *v)
{
    SETUP(&g->b);
    long bad = 0;
    for (int n = B->ny_start; n <= B->ny_end; n++)
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            size_t i = I(m, n);
            if (g->lu[i] > 0.5f && !(ssh[i] < 10.0 && ssh[i] > -10.0)) bad++;
            if (g->lcu[i] > 0.5f && !(u[i] < 100.0 && u[i] > -100.0)) bad++;
            if (g->lcv[i] > 0.5f && !(v[i] < 100.0 && v[i] > -100.0)) bad++;
        }
    return bad;
}

void ora_diag(const ora_grid *g, const double *ssh, const double *u,
              const double *v, const double *hu, const double *hv,
              double *volume, double *energy)
{
    SETUP(&g->b);
    double vol = 0.0, en = 0.0;
    const double grav = g->free_fall_acc;
    for (int n = B->ny_start; n <= B->ny_end; n++) {
        double rv = 0.0, re = 0.0;
        for (int m = B->nx_start; m <= B->nx_end; m++) {
            size_t i = I(m, n);
            if (g->lu[i] > 0.5f) {
                double a = g->dx[i] * g->dy[i];
                rv += (g->hhq_rest[i] + ssh[i]) * a;
                re += 0.5 * grav * ssh[i] * ssh[i] * a;
            }
            if (g->lcu[i] > 0.5f) re += 0.5 * hu[i] * u[i] * u[i] * g->dxt[i] * g->dyh[i];
            if (g->lcv[i] > 0.5f) re += 0.5 * hv[i] * v[i] * v[i] * g->dxh[i] * g->dyt[i];
        }
        vol += rv;
        en += re;
    }
    *volume = vol;
    *energy = en;
}
