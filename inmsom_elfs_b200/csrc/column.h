// Per-water-column kernels of the 3-D part of the mode-split step: the
// implicit vertical viscosity solve of baroclinic_dynamics
// (Function/vel_ssh.f90:794-1027, tridiagonal sweep factor8 of
// Service/oc_algorithms.f90:494-524), the continuity integral of
// vertical_velocity (:1030-1076), one tracer's step tracer_tran_diff
// (Function/tem_sal.f90:1-422), depth_ave (Function/depth.f90:223-254) and
// the barotropic shift of Control/dyncall.f90:170-183, :215-229.
//
// 3-D fields are stacks of pitched 2-D levels: level k (0-based) of a field
// starts plane * k doubles after level 0, and element (m, n) of a level sits
// where ix(d, m, n) puts it.  column.cu is compiled with --fmad=false and
// follows the Fortran expression order, so the results are bit-exact with
// a non-contracting build of the reference.
#pragma once

#include "common.cuh"

namespace inmsom {
namespace column {

struct Levels {
    int nz;                 // s-levels; ww and nu have nz + 1
    long long plane;        // doubles per level
    const double *dz;       // nz layer thicknesses (device)
    const double *hzt;      // nz + 1 interface spacings (device)
};

struct BaroclinicArgs {
    double tau;
    // nz levels (ww, nu: nz + 1), read only
    const double *uu, *uup, *vv, *vvp, *ww, *nu, *rhsx, *rhsy, *rhsx_tran, *rhsy_tran;
    // 2-D
    const double *pgrx, *pgry, *rdis, *tx_surf, *ty_surf, *tx_bot, *ty_bot;
    const double *hhu, *hhup, *hhun, *hhv, *hhvp, *hhvn, *hhh;
    // nz levels: uu, uup, vv, vvp after the step (every point of the arrays)
    double *uu_out, *uup_out, *vv_out, *vvp_out;
    // set to nonzero when a bounded wait of the column kernel gave up (its
    // outputs are then incomplete); must be zero before the launch
    int *flag;
};

// largest nz the solves support
int max_levels();
// true when a periodic wrap column/row lies inside the interior (the filter
// would then need the wrapped value at an interior point; not supported)
bool wrap_inside(const Dom &d);

// Function/vel_ssh.f90:794-1027 on one domain.  Returns 0, or -1 when nz is
// out of range or a periodic wrap column/row lies inside the interior.
int baroclinic_dynamics(const Dom &d, const GridDev &g, const Consts &c, const Levels &L,
                        const BaroclinicArgs &a, cudaStream_t s);
// The same in parts: the column solves of interior rows n0..n1 (they read
// the inputs of rows n0-1..n1+1 and write the outputs of those interior
// rows only), then, after every interior row, the border (the ring's filter
// with the wrapped new velocity, copies elsewhere).
int baroclinic_rows(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const BaroclinicArgs &a,
                    int n0, int n1, cudaStream_t s);
int baroclinic_border(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const BaroclinicArgs &a,
                      cudaStream_t s);

// Function/vel_ssh.f90:1030-1076: w (nz + 1 levels) in place.
int vertical_velocity(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const double *u,
                      const double *v, double *w, const double *hu, const double *hv, const double *wflux,
                      cudaStream_t s);

struct TracerArgs {
    double tau, factor_mu, factor_nu, az, ar, alpha_gm, src_factor;
    // nz levels (ww, nu and the slopes nz + 1), read only
    const double *ff, *ffp, *uu, *vv, *ww, *mu, *nu, *slrx, *slry, *slzx, *slzy, *src;
    // 2-D
    const double *ff_top, *ff_bot, *swbal, *hhu, *hhv, *hhqn, *hhqp;
    const int *ig_top, *ig_bot;
    // outputs: ff, ffp after the step (every point); the flux diagnostics
    // (4 planes each: total, advection, diffusion, GM)
    double *ff_out, *ffp_out, *flux_f_x, *flux_f_y;
    // work: lateral fluxes (nz), their vertical parts, coefficients and GM
    // stream functions (nz + 1); zero outside the interior
    double *flux_x, *flux_y, *flux_zx, *flux_zy, *coef_zx, *coef_zy, *sfgm_zx, *sfgm_zy;
    // set to nonzero when a bounded wait of the solve gave up; zero before the launch
    int *flag;
};

// Function/tem_sal.f90:1-422 on one domain (hhq_rest from the grid's rest
// depth).  Returns 0, or -1 when nz is out of range or a periodic wrap
// column/row lies inside the interior.
int tracer_tran_diff(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const TracerArgs &a,
                     cudaStream_t s);
// The same in parts: the fluxes and column solves of interior rows n0..n1
// (the solves read the fluxes of row n0-1, which an earlier call wrote;
// with a periodic y the whole interior at once), then the border.
int tracer_rows(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const TracerArgs &a, int n0, int n1,
                cudaStream_t s);
int tracer_border(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const TracerArgs &a,
                  cudaStream_t s);

// Function/depth.f90:223-254: utr = sum_k u(k)*dz(k) at the points of mask
// (all but the arrays' outermost ring), u = u - kbcl*utr there; L.dz only.
int depth_ave(const Dom &d, const Levels &L, double *u, double *utr, const float *mask, int kbcl, cudaStream_t s);

// Function/mixing.f90:115-168 stress_components on L.nz levels: tension
// at the lu points and shear at the luu points of the interior (other
// points keep their values), then the periodic wraps of both.
int stress_components(const Dom &d, const GridDev &g, const Levels &L, const double *u, const double *v,
                      double *str_t, double *str_s, cudaStream_t s);

// Function/mixing.f90:171-219 smagorinsky_coeff on L.nz levels (kp =
// vonkarman/Pi): amuv, amts at the lu points of the interior, then the
// periodic wraps of both.
int smagorinsky_coeff(const Dom &d, const GridDev &g, const Levels &L, double visc2, double dift, double kp,
                      const double *str_t, const double *str_s, double *amts, double *amuv, cudaStream_t s);

// Control/dyncall.f90:170-183 (sign < 0: uu - uu2d) and :215-229 (sign > 0:
// uu + uu2d) at the ocean u (v) points of the interior and its ring.
int shift_barotropic(const Dom &d, const GridDev &g, const Levels &L, double *uu, double *vv, const double *uu2d,
                     const double *vv2d, int sign, cudaStream_t s);

}  // namespace column
}  // namespace inmsom
