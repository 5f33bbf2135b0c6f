/*
 * inmsom_gpu.h -- C ABI of the B200 barotropic (external-mode) step of INMSOM.
 *
 * The Fortran model calls its hot path through implicit-interface external
 * subroutines with every argument by reference and every array an
 * explicit-shape, contiguous, column-major real(8) (or real(4) mask) array
 * with bounds (bnd_x1:bnd_x2, bnd_y1:bnd_y2).  Each entry point below takes
 * the same arguments in the same order as the routine it replaces, plus a
 * leading context handle; arrays are passed as base addresses of those host
 * arrays.  Scalars are passed by value (the ISO_C_BINDING shim adds VALUE).
 * No torch, CUDA or C++ types appear in any signature.
 *
 * Every function returns 0 on success or one of the INMSOM_E* codes;
 * inmsom_gpu_last_error() gives a one-line description of the last failure
 * on the calling thread.  The reference has no error returns (it calls
 * `stop` or `mpi_abort`); the Fortran shim turns a nonzero status into
 * `stop` with that message.
 *
 * Threading: a context is used by one host thread at a time and issues all
 * work on its own CUDA stream.  Several contexts may coexist.
 */
#ifndef INMSOM_GPU_H
#define INMSOM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define INMSOM_OK          0
#define INMSOM_ECUDA       1  /* a CUDA runtime call failed                       */
#define INMSOM_EARG        2  /* bad argument: null pointer, bad bounds, nstep<1  */
#define INMSOM_EGUARD      3  /* state non-finite or out of range (guard tripped) */
#define INMSOM_ETIMEOUT    4  /* a bounded device-side wait gave up               */
#define INMSOM_EUNSUPPORTED 5 /* option not supported by the requested path       */
#define INMSOM_EIO         6  /* a file could not be opened, read or written      */

/* context flags (inmsom_gpu_init) */
#define INMSOM_RESIDENT      0x1u /* state, depths and scratch stay on the device
                                     between calls; each barotropic_dynamics call
                                     copies in only the forcing (RHSx, RHSy, wflux,
                                     mu, rdis, and mu4 when ksw4 > 0) and copies
                                     out only the time-mean outputs (ubrtr_i,
                                     vbrtr_i, ssh4gradx, ssh4grady).  Without it
                                     every call copies every array argument in
                                     and out. */
#define INMSOM_FORCE_GENERAL 0x2u /* always use the per-loop kernels (exact
                                     reference rounding) even when the fused
                                     streaming kernel is eligible               */
#define INMSOM_GUARD         0x4u /* after every call apply the range/NaN guard of
                                     Control/dyncall.f90:452-516 to the saved
                                     state; a trip returns INMSOM_EGUARD        */
#define INMSOM_FP32_VELOCITY 0x8u /* inmsom_run_substeps keeps u, up, v, vp in
                                     FP32 on the device for the run (80 instead
                                     of 120 bytes per cell and substep); the
                                     arithmetic, SSH, the rest depth and the
                                     budgets stay FP64.  The FP64 state gets the
                                     FP32 velocities back at the end of each
                                     run.  Needs the fused path on a square
                                     uniform grid with uniform viscosity, drag
                                     and water flux (else INMSOM_EUNSUPPORTED);
                                     barotropic_dynamics stays FP64.           */
#define INMSOM_STATIC_COEFFS 0x10u /* with INMSOM_RESIDENT: the coefficient
                                     fields wflux, mu, rdis (and mu4) are
                                     copied in by the first barotropic_dynamics
                                     call that reads them and stay on the
                                     device; later calls copy in only RHSx and
                                     RHSy.  INMSOM sets mu and rdis once at
                                     start-up (Control/init_pars.f90:166-167,
                                     :459-481); a host that changes them (or
                                     wflux) calls inmsom_gpu_sync_from_host
                                     with INMSOM_SYNC_COEFFS, and the next call
                                     copies them in again.                      */

/* Domain bounds: Modules/mod_mpi_parallel_tools.f90:7-15 (local interior
 * nx_start..ny_end and array bounds bnd_x1..bnd_y2), global significant area
 * mmm..nn and periodicity switches of Inc/basinpar.fi:4-14. */
typedef struct inmsom_bounds {
    int nx_start, nx_end, ny_start, ny_end;
    int bnd_x1, bnd_x2, bnd_y1, bnd_y2;
    int mmm, mm, nnn, nn;
    int periodicity_x, periodicity_y;
} inmsom_bounds;

/* Compile-time constants of the reference, Inc/basinpar.fi:3,46,76-77. */
typedef struct inmsom_consts {
    double time_smooth;    /* time_smooth = 0.05 */
    double free_fall_acc;  /* FreeFallAcc = 9.8  */
    double ref_den;        /* RefDen = 1025      */
    int full_free_surface; /* full_free_surface = 1 */
} inmsom_consts;

typedef struct inmsom_ctx inmsom_ctx;

/* Create a context on CUDA device `device` for one domain.
 * Replaces the MPI/OpenMP set-up of Control/init_arrays.f90:21-88 for one
 * GPU: the bounds are the ones that routine (or its serial twin
 * non_mpi_array_boundary_definition, :2-17) computes. */
int inmsom_gpu_init(inmsom_ctx **ctx, const inmsom_bounds *bounds,
                    const inmsom_consts *consts, int device, unsigned flags);

/* Register the basin_grid module arrays that the hot-path routines read
 * implicitly through `use basin_grid` (Modules/mod_basin_grid.f90:6-63):
 * the seven real(4) masks, the eight metric arrays, the Coriolis parameter,
 * the rest depth (Control/init_pars.f90:150-153) and the twelve
 * external-mode depth arrays (in/out module state).  The grid is uploaded
 * once; the depth arrays are uploaded here and written back by
 * inmsom_gpu_sync_to_host(INMSOM_SYNC_DEPTHS) (or after every call without
 * INMSOM_RESIDENT).  The depth pointers may be NULL, in which case the
 * depths are initialised on the device by hh_init from the state of the
 * first call. */
int inmsom_gpu_register_grid(inmsom_ctx *ctx,
                             const float *lu, const float *luu, const float *luh,
                             const float *lcu, const float *lcv,
                             const float *llu, const float *llv,
                             const double *dx, const double *dy,
                             const double *dxt, const double *dyt,
                             const double *dxh, const double *dyh,
                             const double *dxb, const double *dyb,
                             const double *rlh_s, const double *hhq_rest,
                             double *hhq_e, double *hhqp_e, double *hhqn_e,
                             double *hhu_e, double *hhup_e, double *hhun_e,
                             double *hhv_e, double *hhvp_e, double *hhvn_e,
                             double *hhh_e, double *hhhp_e, double *hhhn_e);

/* Replaces barotropic_dynamics, Function/vel_ssh.f90:379-406 (called at
 * Control/dyncall.f90:137-164), with the same 28 arguments.  Runs 2*nstep
 * leap-frog substeps of length tau/nstep, saves the state after substep
 * nstep into *_e, accumulates the time-mean transports ubrtr_i/vbrtr_i and
 * pressure gradients ssh4gradx/ssh4grady over all 2*nstep substeps and ends
 * with hh_init of the external depths. */
int inmsom_barotropic_dynamics(inmsom_ctx *ctx, double tau, int nstep, int ksw4,
                               double *ubrtr_e, double *ubrtrp_e,
                               double *vbrtr_e, double *vbrtrp_e,
                               double *ssh_e, double *sshp_e,
                               double *ubrtr_i, double *vbrtr_i,
                               double *ssh4gradx, double *ssh4grady,
                               const double *RHSx, const double *RHSy,
                               const double *wflux, const double *mu,
                               const double *mu4, double *vort,
                               double *str_t2d, double *str_s2d,
                               double *fx, double *fy, const double *rdis,
                               double *RHSx_adv, double *RHSy_adv,
                               double *RHSx_dif, double *RHSy_dif);

/* Replaces ssh_internal, Function/vel_ssh.f90:682-751 (called at
 * Control/dyncall.f90:209-214).  hhqn..hhhn are the internal-mode depth
 * module arrays that ssh_internal updates through hh_update (:733-735);
 * copied in and out on every call. */
int inmsom_ssh_internal(inmsom_ctx *ctx, double tau, double *ssh_i,
                        double *sshp_i, const double *u, const double *v,
                        const double *wflux, double *hhqn, double *hhun,
                        double *hhvn, double *hhhn);

/* Replaces the mask construction of gridcon, Service/grid_construction.f90:
 * 59-112: luh, luu, llu, llv, lcu, lcv from the T mask lu (all real(4) 0/1
 * host arrays with the bounds given; outputs must be zero-initialised as
 * model_grid_allocate does).  Bit-exact. */
int inmsom_gridcon(const inmsom_bounds *bounds, const float *lu, float *luu,
                   float *luh, float *llu, float *llv, float *lcu, float *lcv,
                   int device);

/* Replaces the Rayleigh-friction set-up of Control/init_pars.f90:459-481:
 * r_diss = r_fric*|grad hhq_rest| on the registered grid. */
int inmsom_r_diss(inmsom_ctx *ctx, double r_fric, double *r_diss);

/* Replaces the ksw_ssbc=1 wind-stress interpolation of
 * Function/fluxes.f90:29-37 followed by the barotropic forcing assembly of
 * Control/dyncall.f90:110-130 for a barotropic-only model (no 3-D
 * dispersion terms, no bottom stress, no sea-level pressure):
 * RHSx2d = surf_stress_x*dxt*dyh on lcu, RHSy2d = surf_stress_y*dyt*dxh on
 * lcv; other points of RHSx2d/RHSy2d are left as passed. */
int inmsom_wind_forcing(inmsom_ctx *ctx, const double *taux, const double *tauy,
                        double *RHSx2d, double *RHSy2d);

/* After barotropic_dynamics, Control/dyncall.f90:188-201 (the 2-D part of
 * the mode-split step): at the ocean u points of the interior and its
 * one-point ring uu2d = ubrtr_i/hhu and pgrx = pgrx - (slpr(m+1,n) -
 * slpr(m,n))*hhu*dyh/RefDen; likewise vv2d, pgry at v points.  Host arrays;
 * uu2d, vv2d, pgrx, pgry are updated in place. */
int inmsom_velocity2d(inmsom_ctx *ctx, double *uu2d, double *vv2d, double *pgrx, double *pgry,
                      const double *ubrtr_i, const double *vbrtr_i, const double *slpr, const double *hhu,
                      const double *hhv);

/* Replaces baroclinic_dynamics, Function/vel_ssh.f90:794-1027: the 3-D
 * horizontal velocity after the implicit vertical viscosity solve of each
 * water column (the tridiagonal sweep factor8,
 * Service/oc_algorithms.f90:494-524) with vertical advection, Coriolis,
 * the pressure gradient, drag and surface/bottom stress, then the
 * Robert-Asselin filter on the interior and its one-point ring.  Same
 * arguments as the reference routine (Control/dyncall.f90:349-366 passes
 * anzu as nu, r_diss as rdis, the surface/bottom stresses as tx_*, ty_*),
 * plus what it reads from its modules: nz and the vertical grid dz (nz),
 * hzt (nz + 1) of main_basin_pars, and the internal-mode depths hhu, hhup,
 * hhun, hhv, hhvp, hhvn, hhh of basin_grid.  3-D host arrays are
 * (bnd_x1:bnd_x2, bnd_y1:bnd_y2, levels) in Fortran order with nz levels
 * (ww and nu nz + 1), the rest 2-D in the registered layout.  uu, uup, vv,
 * vvp are updated in place.  2 <= nz <= 200 (the reference's surface point
 * reads level 2), else INMSOM_EARG; a periodic wrap column inside the
 * interior gives INMSOM_EUNSUPPORTED.  inmsom_gpu_last_phases times it. */
int inmsom_baroclinic_dynamics(inmsom_ctx *ctx, int nz, const double *dz, const double *hzt, double tau,
                               double *uu, double *uup, double *vv, double *vvp, const double *ww,
                               const double *nu, const double *RHSx, const double *RHSy,
                               const double *RHSx_tran, const double *RHSy_tran, const double *pgrx,
                               const double *pgry, const double *rdis, const double *tx_surf,
                               const double *ty_surf, const double *tx_bot, const double *ty_bot,
                               const double *hhu, const double *hhup, const double *hhun, const double *hhv,
                               const double *hhvp, const double *hhvn, const double *hhh);

/* Replaces vertical_velocity, Function/vel_ssh.f90:1030-1076 (called at
 * Control/dyncall.f90:186): w from the continuity equation, integrated up
 * from w(nz+1) = 0 at the ocean T points of the interior, then the periodic
 * wrap.  u, v have nz levels, w nz + 1 (updated in place; other points keep
 * their values); hu, hv, wflux are 2-D; dz (nz) is the vertical grid.
 * inmsom_gpu_last_phases times it. */
int inmsom_vertical_velocity(inmsom_ctx *ctx, int nz, const double *dz, const double *u, const double *v,
                             double *w, const double *hu, const double *hv, const double *wflux);

/* Replaces tracer_tran_diff, Function/tem_sal.f90:1-422 (called for
 * temperature and salinity at Control/dyncall.f90:265-338): one tracer's
 * leap-frog step with lateral advection, isoneutral diffusion and
 * Gent-McWilliams fluxes, implicit vertical diffusion per water column
 * (factor8) with the surface/bottom conditions of types 1 and 2, the
 * periodic wrap and the Robert-Asselin filter.  Same arguments as the
 * reference routine, plus what it reads from its modules: nz, dz (nz), hzt
 * (nz + 1) and the internal-mode depths hhu, hhv, hhqn, hhqp (hhq_rest is
 * the registered rest depth).  3-D host arrays are (bnd_x1:bnd_x2,
 * bnd_y1:bnd_y2, levels) in Fortran order: ff, ffp, uu, vv, mu, src with nz
 * levels, ww, nu, slrx, slry, slzx, slzy with nz + 1; flux_f_x, flux_f_y
 * are (bnd_x1:bnd_x2, bnd_y1:bnd_y2, 4) outputs (total, advective,
 * diffusive, GM depth-integrated fluxes; zero outside the ocean u/v points
 * of the interior); ig_top, ig_bot are integer arrays with 1 or 2 at the
 * ocean points (else INMSOM_EARG).  ff, ffp are updated in place.  The
 * lateral-boundary arguments (ksw_lbc .. flbc) are accepted and, as in the
 * reference's body, not read.  2 <= nz <= 200.  inmsom_gpu_last_phases
 * times it. */
int inmsom_tracer_tran_diff(inmsom_ctx *ctx, int nz, const double *dz, const double *hzt, double *ff, double *ffp,
                            double tau, const double *uu, const double *vv, const double *ww, const double *mu,
                            double factor_mu, const double *nu, double factor_nu, const double *slrx,
                            const double *slry, const double *slzx, const double *slzy, double az, double ar,
                            double alpha_gm, const double *ff_top, const double *ff_bot, const int *ig_top,
                            const int *ig_bot, double *flux_f_x, double *flux_f_y, const double *swbal, int ksw_lbc,
                            int numlbc, const int *lqpx, const int *lqpy, const char *ind_lbc, const float *flbc,
                            const double *src, double src_factor, const double *hhu, const double *hhv,
                            const double *hhqn, const double *hhqp);

/* Replaces stress_components, Function/mixing.f90:115-168, on nlev levels
 * (Control/dyncall.f90:38 calls it with nz for uup, vvp): tension str_t at
 * the lu points and shear str_s at the luu points of the interior, then
 * the periodic wraps of both; the other points keep the values the caller
 * passed (the reference's arrays keep theirs).  u, v, str_t, str_s are
 * (bnd_x1:bnd_x2, bnd_y1:bnd_y2, nlev) host arrays. */
int inmsom_stress_components(inmsom_ctx *ctx, int nlev, const double *u, const double *v, double *str_t,
                             double *str_s);

/* Replaces smagorinsky_coeff, Function/mixing.f90:171-219 (called at
 * Control/dyncall.f90:41-43 when ksw_lat > 0): at the lu points of the
 * interior on nz levels, mu_smag = (vonkarman/Pi)^2 dx dy sqrt(str_t^2 +
 * the mean of the four str_s^2 around the point), amuv = visc2 + mu_smag,
 * amts = dift + 0.1 mu_smag (vonkarman = 0.4, Pi of Inc/basinpar.fi:72,89),
 * then the periodic wraps of both; other points keep the caller's values.
 * The barotropic viscosity of that step is then
 * inmsom_depth_ave(amuv -> amuv2d, kbcl = 0). */
int inmsom_smagorinsky_coeff(inmsom_ctx *ctx, int nz, double visc2, double dift, const double *str_t,
                             const double *str_s, double *amts, double *amuv);

/* Replaces depth_ave, Function/depth.f90:223-254 (called at
 * Control/dyncall.f90:101-105 to take the barotropic RHS out of the 3-D
 * one): at the points where mask > 0.5 (all but the arrays' outermost ring)
 * utr = sum over k of u(k)*dz(k), then u = u - kbcl*utr.  u has nz levels
 * (in place), utr and the real(4) mask are 2-D; other points of utr keep
 * their values. */
int inmsom_depth_ave(inmsom_ctx *ctx, int nz, const double *dz, double *u, double *utr, const float *mask,
                     int kbcl);

/* The two loops of Control/dyncall.f90 that move the barotropic velocity
 * in and out of the 3-D velocity around vertical_velocity and
 * ssh_internal: sign = -1 is :170-183 (uu = uu - uu2d), sign = +1 is
 * :215-229 (uu = uu + uu2d); likewise vv with vv2d; at the ocean u (v)
 * points of the interior and its one-point ring, every one of the nz
 * levels.  uu, vv in place. */
int inmsom_shift_barotropic(inmsom_ctx *ctx, int nz, double *uu, double *vv, const double *uu2d,
                            const double *vv2d, int sign);

/* The barotropic RHS of Control/dyncall.f90:110-130 (the mode-split caller
 * of barotropic_dynamics), at the ocean u (v) points, in the reference's
 * order of operations:
 *   RHSx2d = RHSx2d - RHSx2d_diff_disp + RHSx2d_tran - RHSx2d_tran_disp
 *          + (surf_stress_x + bot_stress_x)*dxt*dyh
 *          - (slpr(m+1,n) - slpr(m,n))*hhu*dyh/RefDen
 * and likewise for RHSy2d (dyt*dxh, slpr(m,n+1), hhv, dxh).  Host arrays
 * in the registered layout; any input may be NULL (that term is zero);
 * hhu and hhv are needed with slpr. */
int inmsom_rhs2d(inmsom_ctx *ctx, double *RHSx2d, double *RHSy2d, const double *RHSx2d_diff_disp,
                 const double *RHSy2d_diff_disp, const double *RHSx2d_tran, const double *RHSy2d_tran,
                 const double *RHSx2d_tran_disp, const double *RHSy2d_tran_disp, const double *surf_stress_x,
                 const double *surf_stress_y, const double *bot_stress_x, const double *bot_stress_y,
                 const double *slpr, const double *hhu, const double *hhv);

/* Replaces hh_init, Function/depth.f90:2-105, for the external-mode depths
 * (its call at Control/init_pars.f90:426-430): recomputes the twelve
 * registered external depth arrays from ssh_e, sshp_e and hhq_rest and
 * writes them to the registered host arrays. */
int inmsom_hh_init_external(inmsom_ctx *ctx, const double *ssh_e,
                            const double *sshp_e);

/* Guard of Control/dyncall.f90:452-516 on the resident external state:
 * counts interior points with |ssh_e|>=10 (lu), |ubrtr_e|>=100 (lcu) or
 * |vbrtr_e|>=100 (lcv), NaN included. */
int inmsom_guard(inmsom_ctx *ctx, long *nbad);

/* Volume and energy of the resident external state (no reference
 * counterpart): volume = sum_lu (hhq_rest+ssh)*dx*dy,
 * energy = sum_lu g/2*ssh^2*dx*dy + sum_lcu hu/2*u^2*dxt*dyh
 *        + sum_lcv hv/2*v^2*dxh*dyt, with hu, hv the u/v depths of hh_init
 * from ssh.  FP64, deterministic (fixed reduction order). */
int inmsom_gpu_diag(inmsom_ctx *ctx, double *volume, double *energy);

/* Largest interior row count (ny_end - ny_start + 1) that
 * inmsom_diag_noalloc accepts.  Its scratch is a fixed array of
 * 2 * INMSOM_DIAG_NOALLOC_MAX_ROWS doubles (256 KiB) in the library's device
 * image, which every GPU that loads that image holds until the process
 * exits. */
#define INMSOM_DIAG_NOALLOC_MAX_ROWS 16384

/* The volume/energy diagnostic of inmsom_gpu_diag without a context and
 * without allocating anything.  No counterpart in the reference: it exists
 * for callers that cannot allocate GPU memory -- a host model that gives all
 * device memory to its own pool at start-up, or one that must not call
 * cudaMalloc/cudaFree mid-step because those calls synchronise the device
 * and stall the model's streams.
 *
 * Array arguments are DEVICE pointers to f(bnd_x1:bnd_x2, bnd_y1:bnd_y2),
 * x fastest, consecutive rows `ld` elements apart (ld >= bnd_x2-bnd_x1+1):
 * masks lu, lcu, lcv; metrics dx, dy, dxt, dyt, dxh, dyh; rest depth
 * hhq_rest; state ssh, u, v; u/v-point depths hu, hv (hhu_e, hhv_e of
 * hh_init for this ssh).  `out` is a device pointer to two doubles that
 * receive the volume and the energy, defined as for inmsom_gpu_diag; only
 * free_fall_acc of `c` is used.  The call enqueues its two kernels on
 * `stream` (a cudaStream_t of the current device, NULL for its default
 * stream) and returns without waiting; `out` holds the result once the
 * stream has reached that point.
 *
 * It runs on the calling thread's current device and calls no cudaMalloc,
 * cudaFree or other allocating routine.  Its scratch, the per-row partial
 * sums, is the fixed array described above, shared by every call on a
 * device: each call writes every partial it later reads, so nothing is
 * cleared, but calls whose work overlaps on the GPU (unordered streams)
 * race on that array and may return wrong sums -- order them on one stream
 * or with events.  The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress) under the current CUDA context and
 * caches it for that context (a call under another context of the device,
 * e.g. after cudaDeviceReset, looks it up again); make that first call
 * before any stream capture begins.  CUDA loads device code lazily by
 * default (CUDA_MODULE_LOADING=LAZY), so that first call is also when the
 * driver loads this part of the library onto the device and reserves the
 * array there: a caller whose memory pool takes the device's memory makes
 * its first call before the pool does, or sets CUDA_MODULE_LOADING=EAGER
 * so that the array is reserved when the CUDA context is created.  More
 * than INMSOM_DIAG_NOALLOC_MAX_ROWS interior rows returns INMSOM_EARG
 * without touching the device.  An empty interior gives
 * volume = energy = 0. */
int inmsom_diag_noalloc(const inmsom_bounds *b, const inmsom_consts *c, long long ld,
                        const float *lu, const float *lcu, const float *lcv,
                        const double *dx, const double *dy, const double *dxt,
                        const double *dyt, const double *dxh, const double *dyh,
                        const double *hhq_rest, const double *ssh, const double *u,
                        const double *v, const double *hu, const double *hv,
                        double *out, void *stream);

/* Residency control for INMSOM_RESIDENT contexts: which host arrays to
 * refresh (to_host) or re-upload (from_host), using the pointers of the last
 * inmsom_barotropic_dynamics call and of inmsom_gpu_register_grid. */
#define INMSOM_SYNC_STATE   0x1u /* ubrtr_e ubrtrp_e vbrtr_e vbrtrp_e ssh_e sshp_e */
#define INMSOM_SYNC_DEPTHS  0x2u /* the twelve external depth arrays              */
#define INMSOM_SYNC_SCRATCH 0x4u /* vort str_t2d str_s2d fx fy RHS*_adv RHS*_dif  */
#define INMSOM_SYNC_COEFFS  0x8u /* from_host only, INMSOM_STATIC_COEFFS contexts:
                                    the next barotropic_dynamics call copies
                                    wflux, mu, rdis and mu4 in again          */
int inmsom_gpu_sync_to_host(inmsom_ctx *ctx, unsigned what);
int inmsom_gpu_sync_from_host(inmsom_ctx *ctx, unsigned what);

/* Standalone leap-frog driver (no reference counterpart as one routine;
 * it is the state evolution of calling barotropic_dynamics(tau=dt,
 * nstep=1) nsub times and keeping only the saved *_e state).  Each call of
 * barotropic_dynamics(dt,1) computes two substeps but only the first
 * advances *_e; the second feeds the time-mean outputs only.  A standalone
 * barotropic run does not consume those outputs, so this driver computes
 * only the advancing substep.  Works on the resident state of an
 * INMSOM_RESIDENT context after one barotropic_dynamics call or
 * sync_from_host(STATE) has set it.  rhs_scale, if not NULL, holds nsub
 * factors applied to RHSx/RHSy in the corresponding substep (a
 * time-varying wind amplitude); the forcing is otherwise the one of the
 * last call.  The device time of the run (ms) is returned in *ms if ms is
 * not NULL. */
int inmsom_run_substeps(inmsom_ctx *ctx, int nsub, double dt,
                        const double *rhs_scale, float *ms);

/* Upload the external state (*_e, in barotropic_dynamics order) and the
 * forcing of the standalone driver, and remember these host arrays for
 * inmsom_gpu_sync_to_host/from_host.  Counterpart of the first half of a
 * barotropic_dynamics call (its copy-in), without running it.  mu4 may be
 * NULL when the biharmonic term is off. */
int inmsom_load_state(inmsom_ctx *ctx, double *ubrtr_e, double *ubrtrp_e,
                      double *vbrtr_e, double *vbrtrp_e, double *ssh_e,
                      double *sshp_e, const double *RHSx, const double *RHSy,
                      const double *wflux, const double *mu, const double *mu4,
                      const double *rdis);

/* Which kernel path the context uses: 0 = per-loop kernels (exact
 * reference rounding), 1 = fused streaming kernel.  *reason receives a
 * static string saying why the fused path is not eligible (or "eligible"). */
int inmsom_gpu_path(inmsom_ctx *ctx, int *path, const char **reason);

/* Test hook of the fused kernel's bounded waits.  No counterpart in the
 * reference, which has no wait to bound: its failure path is `stop`
 * (Control/dyncall.f90:452-516).  Until called again with item = -1, work
 * item `item` of every fused substep launch on this context does not issue
 * the copies of its `ring_row`-th input row (0 = the first row it loads;
 * clamped to its last), so its wait for that row gives up, and every
 * bounded wait of those launches gives up after `wait_polls` polls of
 * mbarrier.try_wait (0 = the built-in 2^20).  The CTA that gave up sets a
 * status bit, waits (bounded) for the copies it did issue and returns; the
 * call that ran the launch returns INMSOM_ETIMEOUT and leaves its outputs
 * undefined (reload the state with inmsom_load_state or a copy-in call).
 * Nothing faults and the context stays usable: with item = -1 the next
 * calls compute normally. */
int inmsom_test_hold_copy(inmsom_ctx *ctx, int item, int ring_row, unsigned wait_polls);
/* Device time of the phases of the last completed
 * inmsom_barotropic_dynamics, inmsom_baroclinic_dynamics,
 * inmsom_vertical_velocity or inmsom_tracer_tran_diff call (CUDA events on the context's stream):
 * host->device copies, the computation (for the barotropic call the
 * substeps with the depth and time-mean work), device->host copies.  The
 * reference times the whole calls (Control/dyncall.f90:135,165-167 and
 * :348,367-368 start_timer/end_timer). */
int inmsom_gpu_last_phases(inmsom_ctx *ctx, float *upload_ms, float *compute_ms, float *download_ms);

/* ---- On-disk formats (host code, no GPU work) ------------------------- */

/* The reference's DIOGIN-standard direct-access files
 * (Service/input_output_data.f90:117-534, Inc/reclen.fi), same arguments
 * (the Fortran ierr becomes the return value): field(nx, ny, nz) and
 * lu(nx, ny) are column-major host arrays with 1-based positions; the box
 * nxb..nxe x nyb..nye of levels nzb..nze is stored as one record per level
 * (x fastest), record (nfield-1)*(nze-nzb+1) + (k-nzb+1), FP64 for the *8
 * forms and FP32 otherwise, in the host's byte order.  Writing puts undef
 * = -1.0e32 at the points with |lu| < 0.5 and, as the reference does, leaves
 * those points of `field` at 0 afterwards; an existing file is not
 * truncated.  Reading sets the |lu| < 0.5 points of the box to 0.  Errors:
 * INMSOM_EARG (box outside the field, no file name), INMSOM_EIO. */
int inmsom_wdstd8(const char *path, const char *fname, int nfield, double *field, const float *lu, int nx, int ny,
                  int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze);
int inmsom_wdstd(const char *path, const char *fname, int nfield, float *field, const float *lu, int nx, int ny,
                 int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze);
int inmsom_rdstd8(const char *path, const char *fname, int nfield, double *field, const float *lu, int nx, int ny,
                  int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze);
int inmsom_rdstd(const char *path, const char *fname, int nfield, float *field, const float *lu, int nx, int ny,
                 int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze);

/* The MPI-IO forms prdstd / pwdstd (Service/input_output_data.f90:535-652,
 * :657-819), same arguments with the rank's bounds first (the reference
 * takes them from mpi_parallel_tools): fild(bnd_x1:bnd_x2, bnd_y1:bnd_y2,
 * nz) and lu(bnd_x1:bnd_x2, bnd_y1:bnd_y2) are the rank's local FP32
 * arrays; nx, ny, nz and the box are global.  Each rank transfers only its
 * interior nx_start..nx_end x ny_start..ny_end of levels nzb..nze, which
 * must lie inside the box, at the place the single-process wdstd record
 * layout gives it (field nfild after (nfild-1) * (nze-nzb+1) records of
 * (nxe-nxb+1)*(nye-nyb+1) values), so the ranks together write or read the
 * same file as wdstd / rdstd.  Ranks call these independently: the writes
 * and reads are positioned on disjoint byte ranges, no collective.  As the
 * reference: pwdstd sets the land points (|lu| < 0.5) of the rank's
 * interior to undef = -1.0e32 in fild, and writes them so; the file is not
 * truncated; prdstd reads every point (lu unused) and leaves values past
 * the end of the file as they were.  Errors (the reference aborts):
 * INMSOM_EARG (no file name, box outside nx/ny/nz, interior outside the
 * box), INMSOM_EIO. */
int inmsom_pwdstd(const inmsom_bounds *b, const char *path, const char *fname, int nfild, float *fild,
                  const float *lu, int nx, int ny, int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze);
int inmsom_prdstd(const inmsom_bounds *b, const char *path, const char *fname, int nfild, float *fild,
                  const float *lu, int nx, int ny, int nz, int nxb, int nxe, int nyb, int nye, int nzb, int nze);

/* The GrADS descriptor of Service/rw_ctl_file.f90:1-139 ctl_file_write,
 * same arguments: writes <fname with .ctl> describing <fname with .dat>,
 * line by line as the reference's formatted WRITE statements (e12.5,
 * g15.8, i6, i2.2, i4.4 editing). */
int inmsom_ctl_file_write(const char *fname, float undef, int nx, int ny, int nz, int nt, int xtype, const double *x0,
                          double hx, int ytype, const double *y0, double hy, int ztype, const double *z0, double hz,
                          int yr_type, int year0, int month0, int day0, int hour0, int minute0, float ht,
                          const char *title, const char *varname);

/* The GrADS descriptor reader of Service/rw_ctl_file.f90:185-566
 * ctl_file_read, same arguments in the same order, with the capacity of
 * each array after it: datname (datname_len bytes), x0/y0/z0 (x0_cap ...
 * values), title (title_len bytes), varname (varname_cap names of
 * varname_len bytes each, one after another).  Character results are
 * NUL-terminated without trailing blanks; a name longer than its room is
 * cut as the Fortran character variable would cut it.  As the reference:
 * inform counts the definitions read (DSET, TITLE, UNDEF, OPTIONS, XDEF,
 * YDEF, ZDEF, VARS; TDEF is not counted), yr_type is 1 unless OPTIONS
 * starts with 365, a LINEAR x or y axis is filled as x0(1) + hx*(i-1) and a
 * LINEAR z axis as z0(1) + hz*i, LEVELS values may continue over the
 * following lines, the TDEF step is in seconds (yr = 365 days, mo = 30
 * days, dy, hr, mn) in single precision, and the read stops at ENDVARS
 * (at most 512 lines).  title and varname may be NULL.  Errors:
 * INMSOM_EIO (no such file), INMSOM_EARG (the reference's error messages,
 * an end of file before ENDVARS, more values than an array holds). */
int inmsom_ctl_file_read(const char *ctlname, char *datname, int datname_len, float *undef, int *nx, int *ny,
                         int *nz, int *nt, int *xtype, double *x0, int x0_cap, double *hx, int *ytype, double *y0,
                         int y0_cap, double *hy, int *ztype, double *z0, int z0_cap, double *hz, int *nvar,
                         int *yr_type, int *year0, int *month0, int *day0, int *hour0, int *minute0, float *ht,
                         char *title, int title_len, char *varname, int varname_len, int varname_cap, int *inform);

/* compare_grids (Service/rw_ctl_file.f90:628-714; the reference calls it
 * nowhere), same arguments: *ierr = 1 when a grid of descriptor a is longer
 * than maxgridlen or the x, y, z or t point counts differ, else 2 when an
 * x, y or z coordinate differs, else 0.  The undefined values, steps and
 * times are not compared, as in the reference. */
int inmsom_compare_grids(int maxgridlen, int *ierr, float undefa, int nxa, int nya, int nza, int nta,
                         const double *xa, double hxa, const double *ya, double hya, float ta, float hta,
                         const double *za, double hza, float undefb, int nxb, int nyb, int nzb, int ntb,
                         const double *xb, double hxb, const double *yb, double hyb, float tb, float htb,
                         const double *zb, double hzb);

/* The grid and calendar that the checkpoint's descriptors state
 * (basin_grid's xt, xu, yt, yv, dxst, dyst, xgr_type, ygr_type and the
 * model time of Control/output.f90:1454-1463): for a LINEAR axis (type 0)
 * the pointers give the first value only. */
typedef struct inmsom_ctl_axes {
    int xgr_type, ygr_type;
    const double *xt;   /* x of T points from mmm (nx_glob values if LEVELS)      */
    const double *xu;   /* x of u points from mmm-1 (nx_glob+1 values if LEVELS)  */
    const double *yt;   /* y of T points from nnn                                  */
    const double *yv;   /* y of v points from nnn-1                                */
    double dxst, dyst;
    int calendar, year, month, day, hour, minute;
    float tstep;
} inmsom_ctl_axes;

/* The prognostic fields of the reference's checkpoint: column-major host
 * arrays over (bnd_x1:bnd_x2, bnd_y1:bnd_y2), with nz levels (tt .. vvp),
 * nz+1 levels (q2 .. q2lp) or one (the sea surface heights and the
 * external transports).  A pair left NULL (both time levels) is skipped. */
typedef struct inmsom_ocean_state {
    double *tt, *ttp, *ss, *ssp, *uu, *uup, *vv, *vvp;
    double *q2, *q2p, *q2l, *q2lp;
    double *ssh_i, *sshp_i, *ssh_e, *sshp_e, *ubrtr_e, *ubrtrp_e, *vbrtr_e, *vbrtrp_e;
} inmsom_ocean_state;

/* The whole checkpoint ocpwrite (Control/output.f90:1454-1847) from host
 * arrays, same files: for each pair, cp<name>8.dat (FP64, present then
 * previous), cp<name>.dat (FP32) and its descriptor, over mmm..mm x
 * nnn..nn (u-point fields from mmm-1 with mask llu, v-point fields from
 * nnn-1 with mask llv, the others with lu); the 3-D descriptors carry
 * z*1000 (nz levels) or zw*1000 (nz+1 levels) as LEVELS.  As the
 * reference (wdstd8), the land points of the written box are 0 in the
 * caller's arrays afterwards.  The u transport's FP32 file is cpubi.dat
 * and its descriptor names cpube.dat, as the reference writes them. */
int inmsom_ocpwrite(const char *path, const inmsom_bounds *b, int nz, const float *lu, const float *llu,
                    const float *llv, const double *z, const double *zw, const inmsom_ctl_axes *axes,
                    inmsom_ocean_state *state);

/* The restart from those files (start_type > 0), which
 * Control/init_pars.f90:312-417 lists after a stop that leaves it
 * unimplemented: rdstd8 of every pair (land points of the box 0, the rest
 * of each array as it was), the periodic wraps (q2 and q2l wrapped in y
 * over their first nz levels only, as the reference passes nz there), then
 * q2, q2p, q2l, q2lp = max(., tur_var_min) over the whole arrays
 * (tur_var_min = 1.0e-8 in Inc/basinpar.fi:102). */
int inmsom_ocpread(const char *path, const inmsom_bounds *b, int nz, const float *lu, const float *llu,
                   const float *llv, double tur_var_min, inmsom_ocean_state *state);

/* The barotropic part of the reference's checkpoint ocpwrite
 * (Control/output.f90:1736-1847) from the context's resident state: in
 * `path`, cpsshe8.dat (ssh_e, sshp_e over mmm..mm x nnn..nn, mask lu),
 * cpube8.dat (ubrtr_e, ubrtrp_e from mmm-1, mask llu), cpvbe8.dat (vbrtr_e,
 * vbrtrp_e from nnn-1, mask llv), their FP32 copies cpsshe.dat, cpubi.dat,
 * cpvbe.dat and the descriptors cpsshe.ctl, cpube.ctl, cpvbe.ctl (file
 * names as the reference writes them: the u descriptor names cpube.dat).
 * Needs a resident state (inmsom_load_state or a resident
 * barotropic_dynamics call). */
int inmsom_write_checkpoint(inmsom_ctx *ctx, const char *path, const inmsom_ctl_axes *axes);

/* Restart of the barotropic state from such a checkpoint (the reads that
 * Control/init_pars.f90:384-411 lists for start_type > 0, which the
 * reference leaves unimplemented): rdstd8 of cpsshe8.dat, cpube8.dat and
 * cpvbe8.dat (land points 0), the periodic wrap, then the context's
 * resident state and, with full_free_surface, its external depths
 * (hh_init) are set from them.  With the host arrays given (else NULL),
 * the six fields are also returned there. */
int inmsom_read_checkpoint(inmsom_ctx *ctx, const char *path, double *ubrtr_e, double *ubrtrp_e, double *vbrtr_e,
                           double *vbrtrp_e, double *ssh_e, double *sshp_e);

/* Ensemble of independent basins (no counterpart in the reference, which
 * advances one basin per run).  The members are contexts on one device,
 * each with its grid registered, the fused path eligible and its state
 * resident (inmsom_load_state); they may differ in size and in every field.
 * inmsom_ens_run advances every member by nsub substeps of its own dt[i]
 * (the state evolution of inmsom_run_substeps), `group` substeps of all
 * members per launch of one CUDA graph in which each member's kernels run
 * on its own stream, so that members run concurrently and launch overhead
 * is paid once per group.  rhs_scale (nsub values, or NULL for 1) scales
 * every member's RHS at each substep.  group must be even (it keeps each
 * member's state in its set, so the graph can be replayed).  *ms receives
 * the device time of the run.  Creation re-cuts each member's work items
 * to 16 rows at least (a context alone cuts down to 4, which spreads a
 * small basin over more SMs; in an ensemble the other members fill them),
 * and the members keep that cut after the ensemble is destroyed. */
typedef struct inmsom_ens inmsom_ens;
int inmsom_ens_create(inmsom_ens **ens, inmsom_ctx *const *members, int nmembers, int group);
int inmsom_ens_run(inmsom_ens *ens, int nsub, const double *dt, const double *rhs_scale, float *ms);
/* Autotuner: for each size class of members (side length rounded to 256),
 * times `trial_groups` groups of substeps in the ensemble's current form
 * (graph or persistent: tune each form for itself) with each candidate
 * chunk height (one wave of cost-balanced chunks, or about 96, 64, 48 or 32
 * rows per chunk) and keeps the fastest; the combination is then timed
 * against the members' cut before tuning, which stays if it is faster.
 * rows_per_item[i] receives member i's choice (0 = one wave), which the
 * members keep.  The trial runs advance the members' states. */
int inmsom_ens_tune(inmsom_ens *ens, const double *dt, int trial_groups, int *rows_per_item);
/* on != 0: inmsom_ens_run advances each group of substeps of all members
 * with ONE persistent cooperative launch (still replayed as a CUDA graph)
 * instead of one launch per member and substep: one wave of CTAs claims the
 * members' work items in the order (substep, member, item), and an item of
 * a member starts once that member's items of the previous substep are
 * done (per-member completion counters, bounded waits), so members never
 * wait for one another and the substeps of a group have no launch
 * boundary.  The same work items and arithmetic: the same values bit for
 * bit.  on = 0 returns to the per-member graph. */
int inmsom_ens_persistent(inmsom_ens *ens, int on);
int inmsom_ens_destroy(inmsom_ens *ens);

/* Row strips of one basin on several contexts (one per GPU, or several on
 * one GPU); replaces the halo exchange of syncborder_real8
 * (Modules/mod_mpi_parallel_tools.f90:179-252) for the fused path of a
 * 1 x n process grid.  ctxs[0..n) hold consecutive strips, south to north,
 * with the bounds mpi_array_boundary_definition (Control/init_arrays.f90:
 * 21-88) gives for p_size = (1, n) -- the two halo rows next to another
 * strip hold that strip's values -- each with its state resident.
 * inmsom_strips_run advances every strip by nsub substeps of dt (the state
 * evolution of inmsom_run_substeps on the whole basin); after each substep
 * the two rows of the six state fields next to every internal boundary are
 * copied into the neighbour's halo rows (the fused kernel recomputes what
 * it needs in its halo rows, so one exchange per substep gives the
 * single-domain result bit for bit).  With halos of 2k rows between the
 * strips (the same width on both sides of a boundary, and at most a
 * strip's rows) the strips advance k substeps per exchange of 2k rows,
 * computing into their halos as inmsom_step_launch_rows describes.
 * Contexts on different devices get peer access. */
typedef struct inmsom_strips inmsom_strips;
int inmsom_strips_create(inmsom_strips **strips, inmsom_ctx *const *ctxs, int n);
int inmsom_strips_run(inmsom_strips *strips, int nsub, double dt, const double *rhs_scale, float *ms);
int inmsom_strips_destroy(inmsom_strips *strips);

/* Row strips with one process (rank) per GPU, replacing syncborder_real8's
 * MPI exchange (Modules/mod_mpi_parallel_tools.f90:179-252) for a 1 x P
 * process grid: each rank owns the context of its strip (its local bounds
 * from mpi_array_boundary_definition, Control/init_arrays.f90:21-88, with
 * two halo rows each side) and, per substep, calls inmsom_step_launch, packs
 * the two rows each neighbour needs, moves them with its own transport
 * (NCCL send/recv of the device buffers, ordered on inmsom_gpu_stream) and
 * unpacks what it received into its halo rows.  One exchange per substep
 * gives the single-domain result bit for bit (the fused kernel recomputes
 * its halo rows' intermediates).  FP64 state, fused path only.
 *
 * Wide halos (the GPU form of the reference's wide-halo exchange mode): a
 * strip whose halo on a side it shares with another strip is 2k rows (k
 * >= 1; its outer sides keep 2) advances k substeps per exchange of 2k
 * rows.  In substep i = 1..k of such a block it computes 2(k-i) rows into
 * each shared halo as well (inmsom_step_launch_rows), which the neighbour
 * computes alike from the same values, so the result stays the
 * single-domain one bit for bit while the exchanges drop k-fold.
 *   inmsom_step_begin: classify and stage the forcing for a run of substeps
 *     (synchronises the stream);
 *   inmsom_step_launch: enqueue one substep with RHS scale rhs_scale;
 *   inmsom_step_launch_rows: the same computing rows_south / rows_north
 *     rows beyond the interior (each at most the halo width on that side
 *     minus 2, and 0 on a side that is the basin's edge);
 *   inmsom_halo_pack: side 0 the w southernmost interior rows, side 1 the w
 *     northernmost, w the halo width on that side, of the six state fields
 *     into buf (device, 6 * w * pitch doubles, field-major, rows of `pitch`
 *     doubles: INMSOM_HALO_DOUBLES(pitch) for w = 2; pitch from
 *     inmsom_gpu_pitch, w from inmsom_gpu_halo);
 *   inmsom_halo_unpack: buf into the w southern (side 0) or northern
 *     (side 1) halo rows;
 *   inmsom_step_end: wait for the stream and read the kernel status. */
#define INMSOM_HALO_DOUBLES(pitch) (12LL * (long long)(pitch))
int inmsom_step_begin(inmsom_ctx *ctx);
int inmsom_step_launch(inmsom_ctx *ctx, double dt, double rhs_scale);
int inmsom_step_launch_rows(inmsom_ctx *ctx, double dt, double rhs_scale, int rows_south, int rows_north);
/* halo rows of the context south and north of its interior */
int inmsom_gpu_halo(inmsom_ctx *ctx, int *rows_south, int *rows_north);
int inmsom_halo_pack(inmsom_ctx *ctx, int side, void *buf);
int inmsom_halo_unpack(inmsom_ctx *ctx, int side, const void *buf);
int inmsom_step_end(inmsom_ctx *ctx);
/* the context's cudaStream_t, and its device row pitch in doubles */
void *inmsom_gpu_stream(inmsom_ctx *ctx);
long long inmsom_gpu_pitch(inmsom_ctx *ctx);

/* Learned subgrid momentum closure (no counterpart in the reference; it
 * stands in for the Laplacian viscosity of uv_diff2 on coarse grids): an
 * MLP 45 -> 64 -> 64 -> 2 with GELU, BF16 weights and activations on the
 * tensor cores, FP32 accumulate.  Buffers are the caller's device memory:
 * params: INMSOM_MLP_NPARAM floats, W1[48][64] b1[64] W2[64][64] b2[64]
 * W3[64][8] b3[8] (input rows 45..47 and output columns 2..7 zero);
 * wbf16: INMSOM_MLP_NBF16 BF16 values, W1 W2 W3 in that layout; a sample is
 * 48 BF16 features (the last 3 zero); targets 2 floats per sample.
 * `stream` is a cudaStream_t (NULL: default stream); the calls only
 * enqueue work. */
#define INMSOM_MLP_NPARAM 7816
#define INMSOM_MLP_NBF16 7680
#define INMSOM_MLP_PARTIAL 7817   /* floats per 128 samples in `partial` */
/* wbf16 := BF16(W1, W2, W3 of params) */
int inmsom_mlp_pack(const float *params, void *wbf16, void *stream);
/* y[n][0..1] = MLP(x[n]) for n < count */
int inmsom_mlp_forward(const void *x, long long count, const float *params, const void *wbf16, float *y,
                       void *stream);
/* Gradient of the mean squared error over the samples idx[0..batch) (or
 * 0..batch if idx is NULL), batch a multiple of 128: grad[0..NPARAM) and
 * grad[NPARAM] = the loss; partial holds batch/128 * INMSOM_MLP_PARTIAL
 * floats (at most one CTA per 128 samples writes its sums there; they are
 * added in CTA order: deterministic for a given device). */
int inmsom_mlp_grad(const void *x, const float *targets, const int *idx, int batch, const float *params,
                    const void *wbf16, float *partial, float *grad, void *stream);
/* One bias-corrected Adam step (step >= 1) on params, then wbf16. */
int inmsom_mlp_adam(float *params, void *wbf16, float *m, float *v, const float *grad, int step, float lr,
                    float beta1, float beta2, float eps, void *stream);
/* idx[i] uniform in [0, n), a function of (seed, step, i) only */
int inmsom_mlp_batch_indices(int *idx, int batch, long long n, unsigned long long seed, int step, void *stream);

/* The closure on a context's resident state (fused path, FP64 velocities).
 * Features of cell (m, n): field f of (u, v, ssh, rest depth, rlh_s) at
 * (m + dx, n + dy), dx, dy in -1..1, is feature 9 f + 3 (dy + 1) + (dx + 1),
 * normalised as (x - mean[f]) * inv_std[f]; outputs y_u, y_v are velocity
 * tendencies y * out_scale (m/s^2) at the u and v points of the cell. */
typedef struct inmsom_closure_norm {
    float mean[5];
    float inv_std[5];
    float out_scale[2];
} inmsom_closure_norm;
/* x (device, BF16): 48 features of every interior cell, cell (m, n) at row
 * (n - ny_start) * nx + (m - nx_start); enqueued on the context's stream
 * and waited for. */
int inmsom_closure_features(inmsom_ctx *ctx, const inmsom_closure_norm *norm, void *x);
/* nsub substeps as inmsom_run_substeps, the network re-evaluated on the
 * state every `every` substeps (even, dividing nsub): the substeps that
 * follow read RHSx + y_u * out_scale[0] * hu * dxt * dyh at the ocean u
 * points (RHSy likewise at the v points), i.e. the tendency is added to the
 * momentum equation; the registered RHSx, RHSy are not changed.  params and
 * wbf16 are device buffers as for inmsom_mlp_*.  Replayed as CUDA graphs.
 * INMSOM_EUNSUPPORTED without the fused path or with FP32 velocities. */
int inmsom_run_closure(inmsom_ctx *ctx, int nsub, double dt, int every, const float *params, const void *wbf16,
                       const inmsom_closure_norm *norm, float *ms);
/* The RHS increment the closure adds on the resident state (host arrays
 * in the registered layout): y_u * out_scale[0] * hu * dxt * dyh at the
 * ocean u points, likewise at the v points, 0 elsewhere. */
int inmsom_closure_tendency(inmsom_ctx *ctx, const float *params, const void *wbf16,
                            const inmsom_closure_norm *norm, double *rhsx, double *rhsy);

int inmsom_gpu_finalize(inmsom_ctx *ctx);
const char *inmsom_gpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
