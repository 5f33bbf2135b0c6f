// Per-loop kernels of the barotropic step ("general path").
//
// One kernel per loop of the reference routines, over the same index
// ranges, with the same masks and the same expression order; the file is
// compiled with --fmad=false, so every product and sum rounds where the
// Fortran expression rounds it.  This path handles everything the reference
// supports on one domain: 2-D metric arrays, periodic x/y wrap, the
// biharmonic option (ksw4) and ocean points in the halo ring.
#pragma once

#include "common.cuh"

namespace inmsom {
namespace general {

// whole-array helpers
void fill(const Dom &d, double *f, double v, cudaStream_t s);
void copy(const Dom &d, double *dst, const double *src, cudaStream_t s);
// syncborder_real8 (a no-op on one domain) + cyclize8_x/_y
void halo(const Dom &d, double *f, cudaStream_t s);

// Function/depth.f90:2-105
void hh_init(const Dom &d, const GridDev &g, const Consts &c,
             double *hq, double *hqp, double *hqn, double *hu, double *hup,
             double *hun, double *hv, double *hvp, double *hvn, double *hh,
             double *hhp, double *hhn, const double *sh, const double *shp,
             cudaStream_t s);
// Function/depth.f90:108-170
void hh_update(const Dom &d, const GridDev &g, double *hqn, double *hun,
               double *hvn, double *hhn, const double *sh, cudaStream_t s);
// Function/depth.f90:174-220
void hh_shift(const Dom &d, const GridDev &g, const Consts &c, double *const h[12],
              int nstep, cudaStream_t s);
// Function/mixing.f90:115-168
void stress_components(const Dom &d, const GridDev &g, const double *u,
                       const double *v, double *str_t, double *str_s,
                       cudaStream_t s);
// Function/vel_ssh.f90:2-114
void uv_trans(const Dom &d, const GridDev &g, const double *u, const double *v,
              double *vort, const double *hu, const double *hv,
              const double *hh, double *rhsx, double *rhsy, cudaStream_t s);
// Function/vel_ssh.f90:117-184
void uv_diff2(const Dom &d, const GridDev &g, const double *mu,
              const double *str_t, const double *str_s, const double *hq,
              const double *hh, double *rhsx, double *rhsy, cudaStream_t s);
// Function/vel_ssh.f90:187-317
void uv_diff4(const Dom &d, const GridDev &g, const double *mu, double *str_t,
              double *str_s, double *fx, double *fy, const double *hq,
              const double *hu, const double *hv, const double *hh,
              double *rhsx, double *rhsy, cudaStream_t s);

// Function/vel_ssh.f90:487-499 (and :707-719 with hu = hv = NULL)
void continuity(const Dom &d, const GridDev &g, const Consts &c, double dt,
                double *sshn, const double *sshp, const double *u,
                const double *v, const double *hu, const double *hv,
                const double *wflux, cudaStream_t s);

struct MomentumArgs {
    double *un, *vn, *ubrtr_i, *vbrtr_i, *gx, *gy;
    const double *u, *v, *up, *vp, *ssh, *sshn;
    const double *hu, *hup, *hun, *hv, *hvp, *hvn, *hh;
    const double *rhsx, *rhsy, *difx, *dify, *advx, *advy, *rdis;
    double rhs_scale;  // RHSx/RHSy are used as RHSx*rhs_scale (x*1.0 == x)
};
// Function/vel_ssh.f90:531-573
void momentum(const Dom &d, const GridDev &g, const Consts &c, double tau_inner,
              int nstep, const MomentumArgs &a, cudaStream_t s);
// Function/vel_ssh.f90:589-612 and, with nstep = 1 and u = v = NULL, :738-749
void asselin3(const Dom &d, const GridDev &g, const Consts &c, double nstep,
              double *ssh, double *sshp, const double *sshn, double *u,
              double *up, const double *un, double *v, double *vp,
              const double *vn, cudaStream_t s);

// Control/init_pars.f90:459-481
void r_diss(const Dom &d, const GridDev &g, double r_fric, double *r, cudaStream_t s);
// Function/fluxes.f90:29-37 followed by Control/dyncall.f90:110-130 (wind only)
void wind_forcing(const Dom &d, const GridDev &g, const Consts &c,
                  const double *taux, const double *tauy, double *rhsx,
                  double *rhsy, cudaStream_t s);
// Control/dyncall.f90:188-201: uu2d = ubrtr_i/hhu, pgrx -= slpr gradient (and v)
void velocity2d(const Dom &d, const GridDev &g, const Consts &c, double *uu2d, double *vv2d, double *pgrx,
                double *pgry, const double *ubrtr_i, const double *vbrtr_i, const double *slpr, const double *hhu,
                const double *hhv, cudaStream_t s);
// Control/dyncall.f90:110-130, one term of the barotropic RHS in the
// reference's order: 0 r -= a, 1 r += a, 2 r += (a + b) * (dxt*dyh | dyt*dxh),
// 3 r -= (a(next) - a) * b * (dyh | dxh) / rho (a = slpr, b = hhu | hhv)
void rhs2d_term(const Dom &d, const GridDev &g, const Consts &c, int term, double *rx, double *ry,
                const double *ax, const double *ay, const double *bx, const double *by, cudaStream_t s);
// Service/grid_construction.f90:59-112
void gridcon(const Dom &d, const float *lu, float *luu, float *luh, float *llu,
             float *llv, float *lcu, float *lcv, cudaStream_t s);
// Control/dyncall.f90:452-516 on (ssh, u, v); adds the count to *nbad
void guard(const Dom &d, const GridDev &g, const double *ssh, const double *u,
           const double *v, unsigned long long *nbad, cudaStream_t s);
// volume/energy partial sums per interior row (deterministic); rows holds
// 2*(ny_end-ny_start+1) doubles
void diag_rows(const Dom &d, const GridDev &g, const Consts &c,
               const double *ssh, const double *u, const double *v,
               const double *hu, const double *hv, double *rows, cudaStream_t s);
// sums the row partials in row order into out[0] (volume) and out[1] (energy)
void diag_final(int nrows, const double *rows, double *out, cudaStream_t s);

}  // namespace general
}  // namespace inmsom
