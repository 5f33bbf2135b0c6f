/*
 * CPU oracle for the INMSOM barotropic (external-mode) step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path links, loads or
 * calls this code: it is the checker that tests, smoke() and the CPU-baseline
 * leg of bench.py compare the CUDA path against.
 *
 * It restates the reference Fortran loops one by one, in the same loop
 * order, index ranges and expression order (left-to-right evaluation of
 * Fortran's * / + - chains), in FP64.  It is built with
 * -O2 -fno-fast-math -ffp-contract=off so that every product and sum is
 * rounded exactly where the Fortran expression rounds it.
 *
 * PARITY UNPINNED: the reference is Fortran 90 + MPI and neither a Fortran
 * compiler nor MPI exists in this image, and the reference ships no tests,
 * golden vectors or fixtures.  The restatement is therefore checked by
 * physical known-answer tests (lake at rest, exact volume conservation,
 * mirror symmetry, gravity-wave phase speed) and by line-by-line review
 * against the cited reference lines, not against outputs of the reference.
 *
 * Array layout: every 2-D field is the Fortran array
 * f(bnd_x1:bnd_x2, bnd_y1:bnd_y2), column-major (x fastest), passed as a
 * base pointer; element (m,n) sits at (n-bnd_y1)*(bnd_x2-bnd_x1+1)+(m-bnd_x1).
 * Masks are real(4) 0/1 and are tested with "> 0.5" as in the reference.
 */
#ifndef INMSOM_ORACLE_H
#define INMSOM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Bounds of the local domain (Modules/mod_mpi_parallel_tools.f90:7-15) and
 * of the global significant area plus periodicity switches
 * (Inc/basinpar.fi:4-14). */
typedef struct ora_bounds {
    int nx_start, nx_end, ny_start, ny_end;
    int bnd_x1, bnd_x2, bnd_y1, bnd_y2;
    int mmm, mm, nnn, nn;
    int periodicity_x, periodicity_y;
} ora_bounds;

/* Module state read implicitly by the hot-path routines:
 * masks and metrics (Modules/mod_basin_grid.f90:6-37), the external-mode
 * depth arrays (Modules/mod_basin_grid.f90:52-63) and the constants of
 * Inc/basinpar.fi:3,46,76-77. */
typedef struct ora_grid {
    ora_bounds b;
    double time_smooth;     /* Inc/basinpar.fi:3 */
    double free_fall_acc;   /* Inc/basinpar.fi:77 */
    double ref_den;         /* Inc/basinpar.fi:76 */
    int full_free_surface;  /* Inc/basinpar.fi:46 */
    const float *lu, *luu, *luh, *lcu, *lcv, *llu, *llv;
    const double *dx, *dy, *dxt, *dyt, *dxh, *dyh, *dxb, *dyb;
    const double *rlh_s, *hhq_rest;
    double *hhq_e, *hhqp_e, *hhqn_e;
    double *hhu_e, *hhup_e, *hhun_e;
    double *hhv_e, *hhvp_e, *hhvn_e;
    double *hhh_e, *hhhp_e, *hhhn_e;
} ora_grid;

/* Service/grid_construction.f90:59-112: derived masks from the T mask lu. */
void ora_gridcon(const ora_bounds *b, const float *lu, float *luu, float *luh,
                 float *llu, float *llv, float *lcu, float *lcv);

/* Service/oc_algorithms.f90:50-95 (multi-process wrap semantics) and
 * :118-135. */
/* syncborder_real8 hook: called with every field the reference exchanges
 * between MPI ranks, at the point it exchanges it (NULL: one domain). */
typedef void (*ora_exchange_fn)(double *field, void *user);
void ora_set_exchange(ora_exchange_fn fn, void *user);

void ora_cyclize8_x(const ora_bounds *b, double *f);
void ora_cyclize8_y(const ora_bounds *b, double *f);

/* Function/depth.f90:2-105 */
void ora_hh_init(const ora_grid *g,
                 double *hq, double *hqp, double *hqn,
                 double *hu, double *hup, double *hun,
                 double *hv, double *hvp, double *hvn,
                 double *hh, double *hhp, double *hhn,
                 const double *sh, const double *shp, const double *h_r);
/* Function/depth.f90:108-170 */
void ora_hh_update(const ora_grid *g, double *hqn, double *hun, double *hvn,
                   double *hhn, const double *sh, const double *h_r);
/* Function/depth.f90:174-220 */
void ora_hh_shift(const ora_grid *g,
                  double *hq, double *hqp, double *hqn,
                  double *hu, double *hup, double *hun,
                  double *hv, double *hvp, double *hvn,
                  double *hh, double *hhp, double *hhn, int nstep);

/* Function/mixing.f90:115-168 (nlev = 1) */
void ora_stress_components(const ora_grid *g, const double *u, const double *v,
                           double *str_t, double *str_s);
/* Function/mixing.f90:171-219 (nz = 1): Smagorinsky viscosity. */
void ora_smagorinsky_coeff(const ora_grid *g, double visc2, double dift,
                           const double *str_t, const double *str_s,
                           double *amts, double *amuv, double vonkarman,
                           double pi);

/* Function/vel_ssh.f90:2-114 (nlev = 1) */
void ora_uv_trans(const ora_grid *g, const double *u, const double *v,
                  double *vort, const double *hq, const double *hu,
                  const double *hv, const double *hh, double *rhsx,
                  double *rhsy);
/* Function/vel_ssh.f90:117-184 (nlev = 1) */
void ora_uv_diff2(const ora_grid *g, const double *mu, const double *str_t,
                  const double *str_s, const double *hq, const double *hu,
                  const double *hv, const double *hh, double *rhsx,
                  double *rhsy);
/* Function/vel_ssh.f90:187-317 (nlev = 1) */
void ora_uv_diff4(const ora_grid *g, const double *mu, double *str_t,
                  double *str_s, double *fx, double *fy, const double *hq,
                  const double *hu, const double *hv, const double *hh,
                  double *rhsx, double *rhsy);

/* Function/vel_ssh.f90:379-679.  Same 28 arguments in the same order. */
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
                             double *rhsx_dif, double *rhsy_dif);

/* Function/vel_ssh.f90:682-751.  hhqn..hhhn are the internal-mode depth
 * arrays that ssh_internal updates through hh_update (vel_ssh.f90:733-735). */
void ora_ssh_internal(const ora_grid *g, double tau, double *ssh_i,
                      double *sshp_i, const double *u, const double *v,
                      const double *wflux, double *hhqn, double *hhun,
                      double *hhvn, double *hhhn);

/* Control/init_pars.f90:459-481: Rayleigh friction r_diss = r_fric*|grad H|. */
void ora_r_diss(const ora_grid *g, double r_fric, double *r_diss);

/* Function/fluxes.f90:29-37 (ksw_ssbc = 1): wind stress onto u/v points. */
void ora_surface_stress(const ora_grid *g, const double *taux,
                        const double *tauy, double *ssx, double *ssy);

/* Function/vel_ssh.f90:794-1027 baroclinic_dynamics (with factor8,
 * Service/oc_algorithms.f90:494-524) and :1030-1076 vertical_velocity.
 * 3-D arrays (bnd_x1:bnd_x2, bnd_y1:bnd_y2, levels); dz[nz], hzt[nz+1]. */
void ora_baroclinic_dynamics(const ora_grid *g, int nz, const double *dz, const double *hzt, double tau,
                             double *uu, double *uup, double *vv, double *vvp, const double *ww,
                             const double *nu, const double *rhsx, const double *rhsy,
                             const double *rhsx_tran, const double *rhsy_tran, const double *pgrx,
                             const double *pgry, const double *rdis, const double *tx_surf,
                             const double *ty_surf, const double *tx_bot, const double *ty_bot,
                             const double *hhu, const double *hhup, const double *hhun, const double *hhv,
                             const double *hhvp, const double *hhvn, const double *hhh);
void ora_vertical_velocity(const ora_grid *g, int nz, const double *dz, const double *u, const double *v,
                           double *w, const double *hu, const double *hv, const double *wflux);
/* Function/tem_sal.f90:1-422 tracer_tran_diff (without its unused
 * lateral-boundary arguments); hhu, hhv, hhqn, hhqp: internal-mode depths */
void ora_tracer_tran_diff(const ora_grid *g, int nz, const double *dz, const double *hzt, double *ff, double *ffp,
                          double tau, const double *uu, const double *vv, const double *ww, const double *mu,
                          double factor_mu, const double *nu, double factor_nu, const double *slrx,
                          const double *slry, const double *slzx, const double *slzy, double az, double ar,
                          double alpha_gm, const double *ff_top, const double *ff_bot, const int *ig_top,
                          const int *ig_bot, double *flux_f_x, double *flux_f_y, const double *swbal,
                          const double *src, double src_factor, const double *hhu, const double *hhv,
                          const double *hhqn, const double *hhqp);
/* Function/depth.f90:223-254 depth_ave */
void ora_depth_ave(const ora_grid *g, int nz, const double *dz, double *u, double *utr, const float *mask,
                   int kbcl);
/* Control/dyncall.f90:170-183 (sign < 0) and :215-229 (sign > 0) */
void ora_shift_barotropic(const ora_grid *g, int nz, double *uu, double *vv, const double *uu2d,
                          const double *vv2d, int sign);
/* Control/dyncall.f90:188-201: uu2d = ubrtr_i/hhu, pgrx -= slpr gradient
 * (and v), on the interior and its one-point ring. */
void ora_velocity2d(const ora_grid *g, double *uu2d, double *vv2d, double *pgrx, double *pgry,
                    const double *ubrtr_i, const double *vbrtr_i, const double *slpr, const double *hhu,
                    const double *hhv);
/* Control/dyncall.f90:110-130: barotropic forcing assembly.  Any of the
 * optional 3-D-coupling inputs may be NULL, meaning an all-zero field. */
void ora_rhs2d(const ora_grid *g, double *rhsx2d, double *rhsy2d,
               const double *diff_disp_x, const double *diff_disp_y,
               const double *tran_x, const double *tran_y,
               const double *tran_disp_x, const double *tran_disp_y,
               const double *ssx, const double *ssy, const double *bsx,
               const double *bsy, const double *slpr, const double *hhu,
               const double *hhv);

/* Control/dyncall.f90:452-516 restricted to the barotropic state: number of
 * interior points with |ssh| >= 10 (lu), |u| >= 100 (lcu) or |v| >= 100 (lcv),
 * NaN included. */
long ora_guard(const ora_grid *g, const double *ssh, const double *u,
               const double *v);

/* Volume and energy budget of the barotropic state (no reference
 * counterpart; the reference has no diagnostics).  Sums run over the
 * interior in row order and are independent of the thread count:
 *   volume = sum_lu  (hhq_rest + ssh) * dx * dy
 *   energy = sum_lu  0.5*g*ssh^2*dx*dy
 *          + sum_lcu 0.5*hu*u^2*dxt*dyh + sum_lcv 0.5*hv*v^2*dxh*dyt
 * with hu/hv the u/v-point depths passed in. */
void ora_diag(const ora_grid *g, const double *ssh, const double *u,
              const double *v, const double *hu, const double *hv,
              double *volume, double *energy);

#ifdef __cplusplus
}
#endif
#endif
