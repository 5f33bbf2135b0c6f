// C ABI of the barotropic step (include/inmsom_gpu.h): context, device
// mirrors of the Fortran arrays, host<->device residency, and the drivers
// that sequence the kernels of general.cu (per-loop, exact rounding) and
// fused.cu (streaming, one kernel per substep).
#include "inmsom_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "common.cuh"
#include "closure.h"
#include "fused.h"
#include "general.h"

#include "context.h"

namespace inmsom {
namespace capi {

thread_local std::string g_last_error;

int set_err(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

}  // namespace capi
}  // namespace inmsom

namespace inmsom {
// Sets the message of inmsom_gpu_last_error() for entry points defined in
// other source files of the library.
int record_error(int code, const char *msg) { return set_err(code, "%s", msg); }
}  // namespace inmsom

namespace {
// advances the device-side substep counter of replayed graphs
__global__ void k_advance(int *base, int by) { *base += by; }
}  // namespace


namespace inmsom {
namespace capi {

int check_bounds(const inmsom_bounds *b)
{
    if (!b) return set_err(INMSOM_EARG, "bounds is NULL");
    if (b->nx_start > b->nx_end || b->ny_start > b->ny_end)
        return set_err(INMSOM_EARG, "empty interior %d..%d x %d..%d", b->nx_start, b->nx_end,
                       b->ny_start, b->ny_end);
    if (b->bnd_x1 > b->nx_start - 2 || b->bnd_x2 < b->nx_end + 2 || b->bnd_y1 > b->ny_start - 2 ||
        b->bnd_y2 < b->ny_end + 2)
        return set_err(INMSOM_EARG, "array bounds must leave a 2-point halo around the interior");
    if ((b->periodicity_x && (b->mmm - 1 < b->bnd_x1 || b->mm + 1 > b->bnd_x2)) ||
        (b->periodicity_y && (b->nnn - 1 < b->bnd_y1 || b->nn + 1 > b->bnd_y2)))
        return set_err(INMSOM_EARG, "periodic wrap columns/rows outside the arrays");
    return INMSOM_OK;
}

Dom make_dom(const inmsom_bounds *b, long long pitch, int xoff)
{
    Dom d;
    d.nx_start = b->nx_start; d.nx_end = b->nx_end; d.ny_start = b->ny_start; d.ny_end = b->ny_end;
    d.bnd_x1 = b->bnd_x1; d.bnd_x2 = b->bnd_x2; d.bnd_y1 = b->bnd_y1; d.bnd_y2 = b->bnd_y2;
    d.mmm = b->mmm; d.mm = b->mm; d.nnn = b->nnn; d.nn = b->nn;
    d.px = b->periodicity_x; d.py = b->periodicity_y;
    d.pitch = pitch;
    d.xoff = xoff;
    return d;
}

// host (Fortran, ld = nxa) <-> device (pitched)
int sync_stream(inmsom_ctx *c)
{
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaGetLastError());
    return INMSOM_OK;
}

// n fields in ONE allocation, field k at arr[0] + k * pitch * rows (the
// fused path's tensor maps read a state set as one block)
int alloc_block(inmsom_ctx *c, double **arr, int n)
{
    if (arr[0]) return INMSOM_OK;
    const size_t f = (size_t)c->dom.pitch * (size_t)c->dom.nya();
    double *b = nullptr;
    CK(cudaMalloc((void **)&b, (size_t)n * f * sizeof(double)));
    CK(cudaMemsetAsync(b, 0, (size_t)n * f * sizeof(double), c->stream));
    for (int k = 0; k < n; k++) arr[k] = b + k * f;
    return INMSOM_OK;
}

int alloc_set(inmsom_ctx *c, double **arr, int n)
{
    for (int k = 0; k < n; k++)
        if (!arr[k]) CKR(dalloc(c, &arr[k], sizeof(double)));
    return INMSOM_OK;
}

// external depths := hh_init(ssh_e, sshp_e), Function/depth.f90:2-105
void depths_from_state(inmsom_ctx *c)
{
    double **h = c->depth;
    general::hh_init(c->dom, c->gdev(), c->c, h[H_Q], h[H_QP], h[H_QN], h[H_U], h[H_UP], h[H_UN],
                     h[H_V], h[H_VP], h[H_VN], h[H_H], h[H_HP], h[H_HN], c->state[S_SSH],
                     c->state[S_SSHP], c->stream);
    c->depths_current = true;
}

// One substep of the Function/vel_ssh.f90:484-650 loop body on the work
// arrays, general path.  acc receives the time-mean sums (may be scratch).
void general_substep(inmsom_ctx *c, double ti, int nstep, int ksw4, double rhs_scale,
                     bool shift_depths)
{
    const Dom &d = c->dom;
    const GridDev g = c->gdev();
    cudaStream_t s = c->stream;
    double **w = c->work, **h = c->depth, **f = c->forc, **x = c->scr;

    general::continuity(d, g, c->c, ti, w[W_SSHN], w[W_SSHP], w[W_U], w[W_V], h[H_U], h[H_V],
                        f[F_WFLUX], s);
    general::halo(d, w[W_SSHN], s);
    if (c->c.ffs > 0) general::hh_update(d, g, h[H_QN], h[H_UN], h[H_VN], h[H_HN], w[W_SSHN], s);
    general::stress_components(d, g, w[W_UP], w[W_VP], x[C_STRT], x[C_STRS], s);
    general::uv_trans(d, g, w[W_U], w[W_V], x[C_VORT], h[H_U], h[H_V], h[H_H], x[C_ADVX],
                      x[C_ADVY], s);
    general::uv_diff2(d, g, f[F_MU], x[C_STRT], x[C_STRS], h[H_Q], h[H_H], x[C_DIFX], x[C_DIFY], s);
    if (ksw4 > 0)
        general::uv_diff4(d, g, f[F_MU4], x[C_STRT], x[C_STRS], x[C_FX], x[C_FY], h[H_Q], h[H_U],
                          h[H_V], h[H_H], x[C_DIFX], x[C_DIFY], s);
    general::MomentumArgs a;
    a.un = w[W_UN]; a.vn = w[W_VN];
    a.ubrtr_i = c->acc[A_UI]; a.vbrtr_i = c->acc[A_VI]; a.gx = c->acc[A_GX]; a.gy = c->acc[A_GY];
    a.u = w[W_U]; a.v = w[W_V]; a.up = w[W_UP]; a.vp = w[W_VP]; a.ssh = w[W_SSH]; a.sshn = w[W_SSHN];
    a.hu = h[H_U]; a.hup = h[H_UP]; a.hun = h[H_UN]; a.hv = h[H_V]; a.hvp = h[H_VP]; a.hvn = h[H_VN];
    a.hh = h[H_H];
    a.rhsx = f[F_RHSX]; a.rhsy = f[F_RHSY]; a.difx = x[C_DIFX]; a.dify = x[C_DIFY];
    a.advx = x[C_ADVX]; a.advy = x[C_ADVY]; a.rdis = f[F_RDIS]; a.rhs_scale = rhs_scale;
    general::momentum(d, g, c->c, ti, nstep, a, s);
    general::halo(d, w[W_UN], s);
    general::halo(d, w[W_VN], s);
    general::asselin3(d, g, c->c, (double)nstep, w[W_SSH], w[W_SSHP], w[W_SSHN], w[W_U], w[W_UP],
                      w[W_UN], w[W_V], w[W_VP], w[W_VN], s);
    if (c->c.ffs > 0 && shift_depths) general::hh_shift(d, g, c->c, h, nstep, s);
}

// Function/vel_ssh.f90:465-675 on the device, general path
void general_dynamics(inmsom_ctx *c, double tau, int nstep, int ksw4)
{
    const Dom &d = c->dom;
    cudaStream_t s = c->stream;
    double **w = c->work, **st = c->state;
    const double ti = tau / (double)nstep;
    general::fill(d, w[W_UN], 0.0, s);
    general::fill(d, w[W_VN], 0.0, s);
    general::fill(d, w[W_SSHN], 0.0, s);
    general::copy(d, w[W_UP], st[S_UP], s);
    general::copy(d, w[W_VP], st[S_VP], s);
    general::copy(d, w[W_SSHP], st[S_SSHP], s);
    general::copy(d, w[W_U], st[S_U], s);
    general::copy(d, w[W_V], st[S_V], s);
    general::copy(d, w[W_SSH], st[S_SSH], s);
    for (int k = 0; k < NACC; k++) general::fill(d, c->acc[k], 0.0, s);
    for (int step = 1; step <= 2 * nstep; step++) {
        general_substep(c, ti, nstep, ksw4, 1.0, true);
        if (step == nstep) {
            general::copy(d, st[S_UP], w[W_UP], s);
            general::copy(d, st[S_VP], w[W_VP], s);
            general::copy(d, st[S_SSHP], w[W_SSHP], s);
            general::copy(d, st[S_U], w[W_U], s);
            general::copy(d, st[S_V], w[W_V], s);
            general::copy(d, st[S_SSH], w[W_SSH], s);
        }
    }
    general::halo(d, c->acc[A_UI], s);
    general::halo(d, c->acc[A_VI], s);
    if (c->c.ffs > 0) depths_from_state(c);
}

int ensure_grid(inmsom_ctx *c)
{
    if (!c) return set_err(INMSOM_EARG, "context is NULL");
    if (!c->grid_ok) return set_err(INMSOM_EARG, "inmsom_gpu_register_grid has not been called");
    CK(cudaSetDevice(c->device));
    return INMSOM_OK;
}

// the error of the fused kernel's status bits (the last run's flags)
int fused_flag_error(const inmsom_ctx *c, const char *who)
{
    if (c->plan.last_flags & fused::FLAG_SMEM)
        return set_err(INMSOM_ECUDA, "%s: dynamic shared memory not 128-byte aligned, nothing computed", who);
    return set_err(INMSOM_ETIMEOUT, "%s: a bounded TMA wait timed out", who);
}

int run_guard(inmsom_ctx *c, long *nbad)
{
    CK(cudaMemsetAsync(c->d_nbad, 0, sizeof(unsigned long long), c->stream));
    general::guard(c->dom, c->gdev(), c->state[S_SSH], c->state[S_U], c->state[S_V], c->d_nbad,
                   c->stream);
    unsigned long long h = 0;
    CK(cudaMemcpyAsync(&h, c->d_nbad, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CKR(sync_stream(c));
    *nbad = (long)h;
    return INMSOM_OK;
}

}  // namespace capi
}  // namespace inmsom

// ===========================================================================
extern "C" {

const char *inmsom_gpu_last_error(void) { return g_last_error.c_str(); }

int inmsom_gpu_init(inmsom_ctx **out, const inmsom_bounds *b, const inmsom_consts *k, int device,
                    unsigned flags)
{
    if (!out || !k) return set_err(INMSOM_EARG, "NULL argument to inmsom_gpu_init");
    *out = nullptr;
    CKR(check_bounds(b));
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return set_err(INMSOM_EARG, "device %d of %d", device, ndev);
    CK(cudaSetDevice(device));
    inmsom_ctx *c = new inmsom_ctx();
    c->device = device;
    c->flags = flags;
    c->c.ts = k->time_smooth;
    c->c.g = k->free_fall_acc;
    c->c.rho = k->ref_den;
    c->c.ffs = k->full_free_surface;
    const int nxa = b->bnd_x2 - b->bnd_x1 + 1;
    c->plan = fused::make_plan(*b);
    const int xoff = fused::XOFF;
    long long need = nxa + xoff > c->plan.min_pitch ? nxa + xoff : c->plan.min_pitch;
    long long pitch = (need + 31) / 32 * 32;  // 256-byte rows
    c->dom = make_dom(b, pitch, xoff);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    for (int k = 0; k < 4 && e == cudaSuccess; k++) e = cudaEventCreate(&c->ph[k]);
    if (e != cudaSuccess) {
        delete c;
        return set_err(INMSOM_ECUDA, "stream/event creation failed: %s", cudaGetErrorString(e));
    }
    *out = c;
    return INMSOM_OK;
}

int inmsom_gpu_finalize(inmsom_ctx *c)
{
    if (!c) return INMSOM_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &p : c->mask) cudaFree(p);
    for (auto &p : c->met) cudaFree(p);
    for (auto &p : c->depth) cudaFree(p);
    cudaFree(c->state[0]);   // one block (see alloc_block)
    for (auto &p : c->work) cudaFree(p);
    for (auto &p : c->acc) cudaFree(p);
    for (auto &p : c->forc) cudaFree(p);
    for (auto &p : c->scr) cudaFree(p);
    for (auto &p : c->intl) cudaFree(p);
    for (auto &p : c->tmp) cudaFree(p);
    cudaFree(c->r2d[0]);   // one block
    cudaFree(c->v2d[0]);   // one block
    cudaFree(c->col);
    cudaFree(c->col_lev);
    cudaFree(c->trc);
    cudaFree(c->trc_lev);
    for (auto &e : c->bev)
        if (e) cudaEventDestroy(e);
    if (c->s_up) cudaStreamDestroy(c->s_up);
    if (c->s_dn) cudaStreamDestroy(c->s_dn);
    cudaFree(c->d_nbad);
    cudaFree(c->d_rows);
    cudaFree(c->d_out);
    if (c->rs_exec) cudaGraphExecDestroy(c->rs_exec);
    cudaFree(c->d_rs);
    cudaFreeHost(c->h_rs);
    cudaFree(c->d_base);
    if (c->cl_exec) cudaGraphExecDestroy(c->cl_exec);
    cudaFree(c->cl_fac[0]);   // one block with cl_fac[1]
    cudaFree(c->cl_tmp[0]);   // one block
    fused::free_plan(c->plan);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (auto &e : c->ph)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    cudaGetLastError();   // nothing from the teardown reaches the next call
    return INMSOM_OK;
}

int inmsom_gpu_register_grid(inmsom_ctx *c, const float *lu, const float *luu, const float *luh,
                             const float *lcu, const float *lcv, const float *llu, const float *llv,
                             const double *dx, const double *dy, const double *dxt,
                             const double *dyt, const double *dxh, const double *dyh,
                             const double *dxb, const double *dyb, const double *rlh_s,
                             const double *hhq_rest, double *hhq_e, double *hhqp_e,
                             double *hhqn_e, double *hhu_e, double *hhup_e, double *hhun_e,
                             double *hhv_e, double *hhvp_e, double *hhvn_e, double *hhh_e,
                             double *hhhp_e, double *hhhn_e)
{
    if (!c) return set_err(INMSOM_EARG, "context is NULL");
    CK(cudaSetDevice(c->device));
    const float *hm[NMASK] = {lu, luu, luh, lcu, lcv, llu, llv};
    const double *hg[NMET] = {dx, dy, dxt, dyt, dxh, dyh, dxb, dyb, rlh_s, hhq_rest};
    double *hd[NDEPTH] = {hhq_e, hhqp_e, hhqn_e, hhu_e, hhup_e, hhun_e,
                          hhv_e, hhvp_e, hhvn_e, hhh_e, hhhp_e, hhhn_e};
    for (int k = 0; k < NMASK; k++)
        if (!hm[k]) return set_err(INMSOM_EARG, "mask %d is NULL", k);
    for (int k = 0; k < NMET; k++)
        if (!hg[k]) return set_err(INMSOM_EARG, "grid array %d is NULL", k);
    int ndepth = 0;
    for (int k = 0; k < NDEPTH; k++) ndepth += hd[k] != nullptr;
    if (ndepth != 0 && ndepth != NDEPTH)
        return set_err(INMSOM_EARG, "pass all twelve depth arrays or none");

    for (int k = 0; k < NMASK; k++) {
        if (!c->mask[k]) CKR(dalloc(c, &c->mask[k], sizeof(float)));
        CKR(h2d(c, c->mask[k], hm[k]));
    }
    c->h_lu.assign(lu, lu + (size_t)c->dom.nxa() * c->dom.nya());
    CKR(alloc_set(c, c->met, NMET));
    for (int k = 0; k < NMET; k++) CKR(h2d(c, c->met[k], hg[k]));
    CKR(alloc_set(c, c->depth, NDEPTH));
    for (int k = 0; k < NDEPTH; k++) {
        c->h_depth[k] = hd[k];
        if (hd[k]) CKR(h2d(c, c->depth[k], (const double *)hd[k]));
    }
    c->depths_current = ndepth == NDEPTH;
    CKR(alloc_block(c, c->state, NSTATE));
    CKR(alloc_set(c, c->work, NWORK));
    CKR(alloc_set(c, c->acc, NACC));
    CKR(alloc_set(c, c->forc, NFORC));
    CKR(alloc_set(c, c->scr, NSCR));
    if (!c->d_nbad) CK(cudaMalloc(&c->d_nbad, sizeof(unsigned long long)));
    const int nrows = c->dom.ny_end - c->dom.ny_start + 1;
    if (!c->d_rows) CK(cudaMalloc(&c->d_rows, 2 * (size_t)nrows * sizeof(double)));
    if (!c->d_out) CK(cudaMalloc(&c->d_out, 2 * sizeof(double)));
    c->grid_ok = true;
    c->state_on_device = false;
    c->scratch_on_device = false;
    for (int k = 0; k < NFORC; k++) c->coef_on_device[k] = false;
    // fused-path eligibility and its static tables (host-side checks)
    c->fused_ok = false;
    if (c->flags & INMSOM_FORCE_GENERAL) {
        c->fused_reason = "INMSOM_FORCE_GENERAL";
    } else {
        c->fused_reason = fused::check_eligible(c->plan, c->dom, c->c, hm, hg);
        if (!c->fused_reason) {
            CKR(fused::setup(c->plan, c->dom, c->c, hm, hg, c->met[G_HREST], c->mask[M_LU], c->state, c->stream) == 0
                    ? INMSOM_OK
                    : set_err(INMSOM_ECUDA, "fused path set-up failed: %s",
                              cudaGetErrorString(cudaGetLastError())));
            c->plan.f32 = (c->flags & INMSOM_FP32_VELOCITY) != 0;
            c->fused_ok = true;
            c->fused_reason = "eligible";
        }
    }
    return sync_stream(c);
}

int inmsom_gpu_path(inmsom_ctx *c, int *path, const char **reason)
{
    if (!c || !path) return set_err(INMSOM_EARG, "NULL argument");
    *path = c->fused_ok ? 1 : 0;
    if (reason) *reason = c->fused_reason;
    return INMSOM_OK;
}

int inmsom_test_hold_copy(inmsom_ctx *c, int item, int ring_row, unsigned wait_polls)
{
    if (!c) return set_err(INMSOM_EARG, "NULL context");
    if (item < -1 || ring_row < 0) return set_err(INMSOM_EARG, "inmsom_test_hold_copy: item < -1 or ring_row < 0");
    c->plan.hold_item = item;
    c->plan.hold_row = item < 0 ? -1 : ring_row;
    c->plan.wait_limit = item < 0 ? 0u : wait_polls;
    c->plan.generation++;   // captured graphs hold the old parameters
    return INMSOM_OK;
}

int inmsom_barotropic_dynamics(inmsom_ctx *c, double tau, int nstep, int ksw4, double *ubrtr_e,
                               double *ubrtrp_e, double *vbrtr_e, double *vbrtrp_e, double *ssh_e,
                               double *sshp_e, double *ubrtr_i, double *vbrtr_i,
                               double *ssh4gradx, double *ssh4grady, const double *RHSx,
                               const double *RHSy, const double *wflux, const double *mu,
                               const double *mu4, double *vort, double *str_t2d,
                               double *str_s2d, double *fx, double *fy, const double *rdis,
                               double *RHSx_adv, double *RHSy_adv, double *RHSx_dif,
                               double *RHSy_dif)
{
    CKR(ensure_grid(c));
    if (nstep < 1) return set_err(INMSOM_EARG, "nstep = %d < 1", nstep);
    if (!(tau > 0.0)) return set_err(INMSOM_EARG, "tau must be > 0");
    double *hs[NSTATE] = {ubrtr_e, ubrtrp_e, vbrtr_e, vbrtrp_e, ssh_e, sshp_e};
    double *ha[NACC] = {ubrtr_i, vbrtr_i, ssh4gradx, ssh4grady};
    const double *hf[NFORC] = {RHSx, RHSy, wflux, mu, mu4, rdis};
    double *hc[NSCR] = {vort, str_t2d, str_s2d, fx, fy, RHSx_adv, RHSy_adv, RHSx_dif, RHSy_dif};
    const bool resident = (c->flags & INMSOM_RESIDENT) != 0;
    for (int k = 0; k < NSTATE; k++) c->h_state[k] = hs[k];
    for (int k = 0; k < NSCR; k++) c->h_scr[k] = hc[k];
    c->ph_valid = false;
    c->ph_direct = false;
    CK(cudaEventRecord(c->ph[0], c->stream));

    if (!resident || !c->state_on_device) {
        for (int k = 0; k < NSTATE; k++) CKR(h2d(c, c->state[k], (const double *)hs[k]));
        c->state_on_device = true;
        fused::mark_state_changed(c->plan);
    }
    if (!resident || !c->scratch_on_device) {
        for (int k = 0; k < NSCR; k++) CKR(h2d(c, c->scr[k], (const double *)hc[k]));
        c->scratch_on_device = true;
    }
    const bool static_coef = resident && (c->flags & INMSOM_STATIC_COEFFS);
    for (int k = 0; k < NFORC; k++) {
        if (k == F_MU4 && ksw4 <= 0) continue;   // read only by uv_diff4
        const bool coef = k != F_RHSX && k != F_RHSY;
        if (static_coef && coef && c->coef_on_device[k]) continue;
        CKR(h2d(c, c->forc[k], hf[k]));
        c->coef_on_device[k] = static_coef && coef;
        c->forc_gen++;
    }
    if (!resident) {
        for (int k = 0; k < NDEPTH; k++)
            if (c->h_depth[k]) CKR(h2d(c, c->depth[k], (const double *)c->h_depth[k]));
        if (c->h_depth[0]) c->depths_current = true;
    }
    CK(cudaEventRecord(c->ph[1], c->stream));
    const bool fused_run = c->fused_ok && ksw4 <= 0;
    // the fused path derives the depths from SSH; the per-loop path reads them
    if (!c->depths_current && !fused_run) depths_from_state(c);

    int rc = INMSOM_OK;
    if (fused_run) {
        if (fused::dynamics(c->plan, c->dom, c->c, tau, nstep, c->state, c->acc, c->forc,
                            c->stream))
            return set_err(INMSOM_ECUDA, "fused dynamics failed: %s",
                           cudaGetErrorString(cudaGetLastError()));
        if (c->plan.last_flags & (fused::FLAG_TIMEOUT | fused::FLAG_SMEM)) return fused_flag_error(c, "fused kernel");
        // the call ends with hh_init(ssh_e, sshp_e) (vel_ssh.f90:668-675):
        // resident depths are derived when next read (per-loop path, diag,
        // sync_to_host), host depths now
        if (c->c.ffs > 0) {
            if (resident) c->depths_current = false;
            else depths_from_state(c);
        }
    } else {
        general_dynamics(c, tau, nstep, ksw4);
    }

    CK(cudaEventRecord(c->ph[2], c->stream));
    for (int k = 0; k < NACC; k++) CKR(d2h(c, ha[k], c->acc[k]));
    if (!resident) {
        for (int k = 0; k < NSTATE; k++) CKR(d2h(c, hs[k], c->state[k]));
        for (int k = 0; k < NSCR; k++) CKR(d2h(c, hc[k], c->scr[k]));
        for (int k = 0; k < NDEPTH; k++)
            if (c->h_depth[k]) CKR(d2h(c, c->h_depth[k], c->depth[k]));
    }
    CK(cudaEventRecord(c->ph[3], c->stream));
    CKR(sync_stream(c));
    c->ph_valid = true;
    if (c->flags & INMSOM_GUARD) {
        long nbad = 0;
        CKR(run_guard(c, &nbad));
        if (nbad) return set_err(INMSOM_EGUARD, "guard: %ld interior points out of range or NaN", nbad);
    }
    return rc;
}

int inmsom_gpu_last_phases(inmsom_ctx *c, float *upload_ms, float *compute_ms, float *download_ms)
{
    if (!c || !upload_ms || !compute_ms || !download_ms) return set_err(INMSOM_EARG, "NULL argument");
    if (!c->ph_valid) return set_err(INMSOM_EARG, "no completed timed call");
    if (c->ph_direct) {
        *upload_ms = c->ph_ms[0];
        *compute_ms = c->ph_ms[1];
        *download_ms = c->ph_ms[2];
        return INMSOM_OK;
    }
    CK(cudaEventElapsedTime(upload_ms, c->ph[0], c->ph[1]));
    CK(cudaEventElapsedTime(compute_ms, c->ph[1], c->ph[2]));
    CK(cudaEventElapsedTime(download_ms, c->ph[2], c->ph[3]));
    return INMSOM_OK;
}

int inmsom_load_state(inmsom_ctx *c, double *ubrtr_e, double *ubrtrp_e, double *vbrtr_e,
                      double *vbrtrp_e, double *ssh_e, double *sshp_e, const double *RHSx,
                      const double *RHSy, const double *wflux, const double *mu, const double *mu4,
                      const double *rdis)
{
    CKR(ensure_grid(c));
    double *hs[NSTATE] = {ubrtr_e, ubrtrp_e, vbrtr_e, vbrtrp_e, ssh_e, sshp_e};
    const double *hf[NFORC] = {RHSx, RHSy, wflux, mu, mu4, rdis};
    for (int k = 0; k < NSTATE; k++) {
        CKR(h2d(c, c->state[k], (const double *)hs[k]));
        c->h_state[k] = hs[k];
    }
    const bool static_coef = (c->flags & INMSOM_RESIDENT) && (c->flags & INMSOM_STATIC_COEFFS);
    for (int k = 0; k < NFORC; k++) {
        if (k == F_MU4 && !mu4) continue;
        CKR(h2d(c, c->forc[k], hf[k]));
        c->coef_on_device[k] = static_coef && k != F_RHSX && k != F_RHSY;
        c->forc_gen++;
    }
    c->state_on_device = true;
    fused::mark_state_changed(c->plan);
    if (c->fused_ok || !c->depths_current) depths_from_state(c);
    return sync_stream(c);
}

namespace {

constexpr int RS_GROUP = 50;   // most substeps per graph replay

// substeps per replayed graph for a run of nsub: even, so that a replay
// leaves the state in the set it started from
int rs_length(int nsub) { return std::min(RS_GROUP, nsub & ~1); }

bool rs_current(const inmsom_ctx *c, int len, double dt)
{
    const fused::Plan &p = c->plan;
    return c->rs_exec && c->rs_len == len && c->rs_gen == p.generation && c->rs_dt == dt &&
           c->rs_src == c->state[0] && c->rs_pgen == p.prep_gen && c->rs_mu0 == p.prep_mu0 &&
           c->rs_rd0 == p.prep_rd0 && c->rs_wq0 == p.prep_wq0;
}

// capture len fused launches (and the counter advance) as the context's
// replayed graph, with the forcing mode of the plan's last preparation
int rs_capture(inmsom_ctx *c, int len, double dt)
{
    const bool f32 = (c->flags & INMSOM_FP32_VELOCITY) != 0;
    fused::Plan &p = c->plan;
    if (c->rs_exec) cudaGraphExecDestroy(c->rs_exec);
    c->rs_exec = nullptr;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int lrc = f32 ? fused::launch_steps_f32(p, c->dom, c->c, dt, len, c->d_rs, c->d_base, nullptr, c->state,
                                                  c->stream)
                        : fused::launch_steps(p, c->dom, c->c, dt, len, c->d_rs, c->d_base, c->state, c->stream);
    if (lrc == 0) k_advance<<<1, 1, 0, c->stream>>>(c->d_base, len);
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
    if (lrc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return set_err(INMSOM_ECUDA, "fused substeps: graph capture failed: %s", cudaGetErrorString(ce));
    }
    const cudaError_t ie = cudaGraphInstantiate(&c->rs_exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return set_err(INMSOM_ECUDA, "fused substeps: %s", cudaGetErrorString(ie));
    // put the graph on the device now, not at its first launch
    CK(cudaGraphUpload(c->rs_exec, c->stream));
    c->rs_len = len;
    c->rs_gen = p.generation;
    c->rs_dt = dt;
    c->rs_src = c->state[0];
    c->rs_pgen = p.prep_gen;
    c->rs_mu0 = p.prep_mu0;
    c->rs_rd0 = p.prep_rd0;
    c->rs_wq0 = p.prep_wq0;
    return INMSOM_OK;
}

// Set-up of a graph run that needs no device work: the per-substep scale
// buffer and, when an earlier graph run prepared the plan, the capture of
// this run's graph with that run's forcing mode (kept if the preparation
// of this run finds the same mode).  Host work only, so it stays out of
// the run's timed region.
int rs_setup(inmsom_ctx *c, int nsub, double dt)
{
    if (!c->d_base) CK(cudaMalloc(&c->d_base, sizeof(int)));
    if ((size_t)nsub > c->rs_cap) {
        if (c->rs_exec) cudaGraphExecDestroy(c->rs_exec);
        c->rs_exec = nullptr;   // it holds the old buffer
        CK(cudaStreamSynchronize(c->stream));
        cudaFree(c->d_rs);
        c->d_rs = nullptr;
        c->rs_cap = 0;
        CK(cudaMalloc(&c->d_rs, (size_t)nsub * sizeof(double)));
        c->rs_cap = (size_t)nsub;
    }
    if ((size_t)nsub > c->h_rs_cap) {
        CK(cudaStreamSynchronize(c->stream));
        cudaFreeHost(c->h_rs);
        c->h_rs = nullptr;
        c->h_rs_cap = 0;
        CK(cudaMallocHost(&c->h_rs, (size_t)nsub * sizeof(double)));
        c->h_rs_cap = (size_t)nsub;
    }
    const int len = rs_length(nsub);
    if (c->rs_pgen >= 0 && c->plan.prepared && !rs_current(c, len, dt)) CKR(rs_capture(c, len, dt));
    return INMSOM_OK;
}

// inmsom_run_substeps on the fused path as replays of one captured graph of
// rs_length(nsub) launches (launch gaps removed: 2-3 % on the 2048 x 1536
// basin); the RHS scale of every substep is read on the device at a counter
// the graph advances.  The graph is recaptured when its length, dt, the
// work items, the state's set or the forcing mode change.  FP32 velocity
// storage: the same with its kernel, between the conversions to and from
// FP32.
int run_substeps_graph(inmsom_ctx *c, int nsub, double dt, const double *rhs_scale, bool *ev1_recorded)
{
    const bool f32 = (c->flags & INMSOM_FP32_VELOCITY) != 0;
    if (f32) {
        const int rc = fused::prepare_steps_f32(c->plan, c->dom, c->c, c->state, c->forc, c->stream, c->forc_gen);
        if (rc == 2)
            return set_err(INMSOM_EUNSUPPORTED,
                           "FP32 velocity storage needs a square uniform grid with uniform viscosity, drag and "
                           "water flux");
        if (rc) return set_err(INMSOM_ECUDA, "fused substeps: prepare failed: %s", cudaGetErrorString(cudaGetLastError()));
    } else if (fused::prepare_steps(c->plan, c->dom, c->c, c->state, c->forc, c->stream, c->forc_gen)) {
        return set_err(INMSOM_ECUDA, "fused substeps: prepare failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    auto launch = [&](int n) {
        return f32 ? fused::launch_steps_f32(c->plan, c->dom, c->c, dt, n, c->d_rs, c->d_base, nullptr, c->state,
                                             c->stream)
                   : fused::launch_steps(c->plan, c->dom, c->c, dt, n, c->d_rs, c->d_base, c->state, c->stream);
    };
    // the scales go through pinned memory (an asynchronous copy); the
    // previous run ended with a synchronisation, so the buffer is free
    for (int k = 0; k < nsub; k++) c->h_rs[k] = rhs_scale ? rhs_scale[k] : 1.0;
    CK(cudaMemcpyAsync(c->d_rs, c->h_rs, (size_t)nsub * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->d_base, 0, sizeof(int), c->stream));
    const int len = rs_length(nsub);
    if (!rs_current(c, len, dt)) CKR(rs_capture(c, len, dt));
    const int groups = nsub / len, rest = nsub % len;
    for (int gi = 0; gi < groups; gi++) CK(cudaGraphLaunch(c->rs_exec, c->stream));
    if (rest && launch(rest)) return set_err(INMSOM_ECUDA, "fused substeps: launch failed");
    // the end of the run's device work, before the status read-back waits
    // for it (the FP32 run's last work is its conversion back to FP64)
    if (!f32) {
        CK(cudaEventRecord(c->ev1, c->stream));
        *ev1_recorded = true;
    }
    const int frc = f32 ? fused::finish_steps_f32(c->plan, c->dom, c->state, c->stream)
                        : fused::finish_steps(c->plan, c->stream);
    if (frc) return set_err(INMSOM_ECUDA, "fused substeps: %s", cudaGetErrorString(cudaGetLastError()));
    return INMSOM_OK;
}

}  // namespace

int inmsom_run_substeps(inmsom_ctx *c, int nsub, double dt, const double *rhs_scale, float *ms)
{
    CKR(ensure_grid(c));
    if (nsub < 0) return set_err(INMSOM_EARG, "nsub < 0");
    if (!(dt > 0.0)) return set_err(INMSOM_EARG, "dt must be > 0");
    if (!c->state_on_device)
        return set_err(INMSOM_EARG, "no resident state: call inmsom_load_state or barotropic_dynamics first");
    if ((c->flags & INMSOM_FP32_VELOCITY) && !c->fused_ok)
        return set_err(INMSOM_EUNSUPPORTED, "FP32 velocity storage needs the fused path (%s)", c->fused_reason);
    const bool graph = c->fused_ok && nsub >= 2;
    bool ev1_recorded = false;
    if (graph) CKR(rs_setup(c, nsub, dt));
    CK(cudaEventRecord(c->ev0, c->stream));
    if (graph) {
        CKR(run_substeps_graph(c, nsub, dt, rhs_scale, &ev1_recorded));
        c->depths_current = false;
        if (c->plan.last_flags & (fused::FLAG_TIMEOUT | fused::FLAG_SMEM)) return fused_flag_error(c, "fused kernel");
    } else if (c->fused_ok) {
        const int rc = fused::run_substeps(c->plan, c->dom, c->c, nsub, dt, rhs_scale, c->state, c->forc,
                                           c->stream);
        if (rc == 2)
            return set_err(INMSOM_EUNSUPPORTED,
                           "FP32 velocity storage needs a square uniform grid with uniform viscosity, drag and "
                           "water flux");
        if (rc)
            return set_err(INMSOM_ECUDA, "fused substeps failed: %s",
                           cudaGetErrorString(cudaGetLastError()));
        c->depths_current = false;
        if (c->plan.last_flags & (fused::FLAG_TIMEOUT | fused::FLAG_SMEM)) return fused_flag_error(c, "fused kernel");
    } else {
        // nsub calls of barotropic_dynamics(dt, 1) keeping *_e: the first
        // substep of each call, run in place on the saved state, followed by
        // the hh_init that ends every call
        const Dom &d = c->dom;
        double **w = c->work, **st = c->state;
        double *saved[NWORK];
        for (int k = 0; k < NWORK; k++) saved[k] = w[k];
        w[W_U] = st[S_U]; w[W_UP] = st[S_UP]; w[W_V] = st[S_V]; w[W_VP] = st[S_VP];
        w[W_SSH] = st[S_SSH]; w[W_SSHP] = st[S_SSHP];
        general::fill(d, w[W_UN], 0.0, c->stream);
        general::fill(d, w[W_VN], 0.0, c->stream);
        general::fill(d, w[W_SSHN], 0.0, c->stream);
        if (!c->depths_current) depths_from_state(c);
        for (int k = 0; k < nsub; k++) {
            general_substep(c, dt, 1, 0, rhs_scale ? rhs_scale[k] : 1.0, false);
            if (c->c.ffs > 0) depths_from_state(c);
        }
        for (int k = 0; k < NWORK; k++) w[k] = saved[k];
    }
    if (!ev1_recorded) CK(cudaEventRecord(c->ev1, c->stream));
    CKR(sync_stream(c));
    if (ms) CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
    if (c->flags & INMSOM_GUARD) {
        long nbad = 0;
        CKR(run_guard(c, &nbad));
        if (nbad) return set_err(INMSOM_EGUARD, "guard: %ld interior points out of range or NaN", nbad);
    }
    return INMSOM_OK;
}

// ===================================================================== closure
namespace {

// the closure arguments of a context (fields of the resident state)
int closure_args(inmsom_ctx *c, const inmsom_closure_norm *norm, closure::Args &a)
{
    std::memset(&a, 0, sizeof a);
    const Dom &d = c->dom;
    a.fld[0] = c->state[S_U];
    a.fld[1] = c->state[S_V];
    a.fld[2] = c->state[S_SSH];
    a.fld[3] = c->met[G_HREST];
    a.fld[4] = c->met[G_RLH];
    for (int k = 0; k < 5; k++) {
        if (!a.fld[k]) return set_err(INMSOM_EARG, "closure: grid or state not on the device");
        a.mean[k] = norm->mean[k];
        a.inv_std[k] = norm->inv_std[k];
    }
    a.out_scale[0] = norm->out_scale[0];
    a.out_scale[1] = norm->out_scale[1];
    a.pitch = d.pitch;
    a.x1 = d.bnd_x1; a.x2 = d.bnd_x2; a.y1 = d.bnd_y1; a.y2 = d.bnd_y2; a.xoff = d.xoff;
    a.mx0 = d.nx_start; a.mx1 = d.nx_end; a.ny0 = d.ny_start; a.ny1 = d.ny_end;
    return INMSOM_OK;
}

int closure_factors(inmsom_ctx *c, closure::Args &a)
{
    if (!c->cl_fac[0]) {
        double *f[2] = {};
        CKR(alloc_block(c, f, 2));
        c->cl_fac[0] = f[0];
        c->cl_fac[1] = f[1];
        if (closure::factors(a, c->mask[M_LCU], c->mask[M_LCV], c->met[G_DXT], c->met[G_DYH], c->met[G_DYT],
                             c->met[G_DXH], c->cl_fac[0], c->cl_fac[1], c->stream))
            return INMSOM_ECUDA;
    }
    a.fac[0] = c->cl_fac[0];
    a.fac[1] = c->cl_fac[1];
    return INMSOM_OK;
}

// one group: the network on the state, then `every` substeps
int closure_group(inmsom_ctx *c, const closure::Args &a, double dt, int every)
{
    if (closure::apply(a, c->plan.nsm, c->stream)) return INMSOM_ECUDA;
    if (fused::launch_steps(c->plan, c->dom, c->c, dt, every, nullptr, nullptr, c->state, c->stream))
        return set_err(INMSOM_ECUDA, "closure: substep launch failed");
    return INMSOM_OK;
}

}  // namespace

int inmsom_closure_features(inmsom_ctx *c, const inmsom_closure_norm *norm, void *x)
{
    CKR(ensure_grid(c));
    if (!norm || !x) return set_err(INMSOM_EARG, "inmsom_closure_features: NULL argument");
    if (!c->state_on_device)
        return set_err(INMSOM_EARG, "no resident state: call inmsom_load_state first");
    closure::Args a;
    CKR(closure_args(c, norm, a));
    a.feat = x;
    if (closure::features(a, c->plan.nsm, c->stream)) return INMSOM_ECUDA;
    return sync_stream(c);
}

int inmsom_closure_tendency(inmsom_ctx *c, const float *params, const void *wbf16, const inmsom_closure_norm *norm,
                            double *rhsx, double *rhsy)
{
    CKR(ensure_grid(c));
    if (!params || !wbf16 || !norm || !rhsx || !rhsy)
        return set_err(INMSOM_EARG, "inmsom_closure_tendency: NULL argument");
    if (!c->state_on_device)
        return set_err(INMSOM_EARG, "no resident state: call inmsom_load_state first");
    closure::Args a;
    CKR(closure_args(c, norm, a));
    CKR(closure_factors(c, a));
    CKR(alloc_block(c, c->cl_tmp, 3));   // zeroed once; field 2 stays zero
    CK(cudaMemsetAsync(c->cl_tmp[0], 0, 2 * c->plan.fstride * sizeof(double), c->stream));
    a.base[0] = a.base[1] = c->cl_tmp[2];
    a.out[0] = c->cl_tmp[0];
    a.out[1] = c->cl_tmp[1];
    a.prm = params;
    a.wb = wbf16;
    if (closure::apply(a, c->plan.nsm, c->stream)) return INMSOM_ECUDA;
    CKR(d2h(c, rhsx, c->cl_tmp[0]));
    CKR(d2h(c, rhsy, c->cl_tmp[1]));
    return sync_stream(c);
}

int inmsom_run_closure(inmsom_ctx *c, int nsub, double dt, int every, const float *params, const void *wbf16,
                       const inmsom_closure_norm *norm, float *ms)
{
    CKR(ensure_grid(c));
    if (!params || !wbf16 || !norm) return set_err(INMSOM_EARG, "inmsom_run_closure: NULL argument");
    if (every < 2 || every % 2 || nsub < 0 || nsub % every)
        return set_err(INMSOM_EARG, "inmsom_run_closure: every must be even and divide nsub");
    if (!(dt > 0.0)) return set_err(INMSOM_EARG, "dt must be > 0");
    if (!c->state_on_device)
        return set_err(INMSOM_EARG, "no resident state: call inmsom_load_state or barotropic_dynamics first");
    if (!c->fused_ok) return set_err(INMSOM_EUNSUPPORTED, "the closure needs the fused path (%s)", c->fused_reason);
    if (c->flags & INMSOM_FP32_VELOCITY)
        return set_err(INMSOM_EUNSUPPORTED, "the closure runs with FP64 velocities");
    closure::Args a;
    CKR(closure_args(c, norm, a));
    CKR(closure_factors(c, a));
    fused::Plan &p = c->plan;
    a.base[0] = c->forc[F_RHSX];
    a.base[1] = c->forc[F_RHSY];
    a.out[0] = p.stat + fused::T_RX * p.fstride;
    a.out[1] = p.stat + fused::T_RY * p.fstride;
    a.prm = params;
    a.wb = wbf16;
    CK(cudaEventRecord(c->ev0, c->stream));
    // stages RHSx, RHSy into the static block (the closure then overwrites
    // its ocean u/v points every group) and classifies the forcing
    if (fused::prepare_steps(p, c->dom, c->c, c->state, c->forc, c->stream))
        return set_err(INMSOM_ECUDA, "closure: prepare failed: %s", cudaGetErrorString(cudaGetLastError()));
    const int ngroups = nsub / every;
    const int per_graph = every >= RS_GROUP ? 1 : RS_GROUP / every;
    if (ngroups >= 2 * per_graph) {
        if (!c->cl_exec || c->cl_gen != p.generation || c->cl_dt != dt || c->cl_every != every ||
            c->cl_groups != per_graph || std::memcmp(&c->cl_args, &a, sizeof a) != 0) {
            if (c->cl_exec) cudaGraphExecDestroy(c->cl_exec);
            c->cl_exec = nullptr;
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            int rc = INMSOM_OK;
            for (int k = 0; k < per_graph && rc == INMSOM_OK; k++) rc = closure_group(c, a, dt, every);
            const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
            if (rc || ce != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return set_err(INMSOM_ECUDA, "closure: graph capture failed: %s", cudaGetErrorString(ce));
            }
            const cudaError_t ie = cudaGraphInstantiate(&c->cl_exec, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return set_err(INMSOM_ECUDA, "closure: %s", cudaGetErrorString(ie));
            c->cl_gen = p.generation;
            c->cl_dt = dt;
            c->cl_every = every;
            c->cl_groups = per_graph;
            c->cl_args = a;
        }
        for (int k = 0; k < ngroups / per_graph; k++) CK(cudaGraphLaunch(c->cl_exec, c->stream));
        for (int k = 0; k < ngroups % per_graph; k++) CKR(closure_group(c, a, dt, every));
    } else {
        for (int k = 0; k < ngroups; k++) CKR(closure_group(c, a, dt, every));
    }
    if (fused::finish_steps(p, c->stream))
        return set_err(INMSOM_ECUDA, "closure: %s", cudaGetErrorString(cudaGetLastError()));
    c->depths_current = false;
    CK(cudaEventRecord(c->ev1, c->stream));
    CKR(sync_stream(c));
    if (ms) CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
    if (p.last_flags & (fused::FLAG_TIMEOUT | fused::FLAG_SMEM)) return fused_flag_error(c, "fused kernel");
    if (c->flags & INMSOM_GUARD) {
        long nbad = 0;
        CKR(run_guard(c, &nbad));
        if (nbad) return set_err(INMSOM_EGUARD, "guard: %ld interior points out of range or NaN", nbad);
    }
    return INMSOM_OK;
}

int inmsom_ssh_internal(inmsom_ctx *c, double tau, double *ssh_i, double *sshp_i, const double *u,
                        const double *v, const double *wflux, double *hhqn, double *hhun,
                        double *hhvn, double *hhhn)
{
    CKR(ensure_grid(c));
    CKR(alloc_set(c, c->intl, NINT));
    double **I = c->intl;
    CKR(h2d(c, I[I_SSH], (const double *)ssh_i));
    CKR(h2d(c, I[I_SSHP], (const double *)sshp_i));
    CKR(h2d(c, I[I_U], u));
    CKR(h2d(c, I[I_V], v));
    CKR(h2d(c, I[I_WFLUX], wflux));
    double *hi[4] = {hhqn, hhun, hhvn, hhhn};
    for (int k = 0; k < 4; k++) CKR(h2d(c, I[I_HQN + k], (const double *)hi[k]));
    const Dom &d = c->dom;
    const GridDev g = c->gdev();
    general::fill(d, I[I_NEW], 0.0, c->stream);  // vel_ssh.f90:704-705
    general::continuity(d, g, c->c, tau, I[I_NEW], I[I_SSHP], I[I_U], I[I_V], nullptr, nullptr,
                        I[I_WFLUX], c->stream);
    general::halo(d, I[I_NEW], c->stream);
    if (c->c.ffs > 0)
        general::hh_update(d, g, I[I_HQN], I[I_HUN], I[I_HVN], I[I_HHN], I[I_NEW], c->stream);
    general::asselin3(d, g, c->c, 1.0, I[I_SSH], I[I_SSHP], I[I_NEW], nullptr, nullptr, nullptr,
                      nullptr, nullptr, nullptr, c->stream);
    CKR(d2h(c, ssh_i, I[I_SSH]));
    CKR(d2h(c, sshp_i, I[I_SSHP]));
    for (int k = 0; k < 4; k++) CKR(d2h(c, hi[k], I[I_HQN + k]));
    return sync_stream(c);
}

int inmsom_gridcon(const inmsom_bounds *b, const float *lu, float *luu, float *luh, float *llu,
                   float *llv, float *lcu, float *lcv, int device)
{
    CKR(check_bounds(b));
    if (!lu || !luu || !luh || !llu || !llv || !lcu || !lcv)
        return set_err(INMSOM_EARG, "NULL mask array");
    CK(cudaSetDevice(device));
    const int nxa = b->bnd_x2 - b->bnd_x1 + 1, nya = b->bnd_y2 - b->bnd_y1 + 1;
    Dom d = make_dom(b, nxa, 0);
    const size_t bytes = (size_t)nxa * nya * sizeof(float);
    float *dv[7] = {};
    const float *src[7] = {lu, luu, luh, llu, llv, lcu, lcv};
    float *dst[7] = {nullptr, luu, luh, llu, llv, lcu, lcv};
    int rc = INMSOM_OK;
    for (int k = 0; k < 7 && rc == INMSOM_OK; k++) {
        cudaError_t e = cudaMalloc(&dv[k], bytes);
        if (e == cudaSuccess) e = cudaMemcpy(dv[k], src[k], bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) rc = set_err(INMSOM_ECUDA, "gridcon upload: %s", cudaGetErrorString(e));
    }
    if (rc == INMSOM_OK) {
        general::gridcon(d, dv[0], dv[1], dv[2], dv[3], dv[4], dv[5], dv[6], 0);
        cudaError_t e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaGetLastError();
        for (int k = 1; k < 7 && e == cudaSuccess; k++)
            e = cudaMemcpy(dst[k], dv[k], bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = set_err(INMSOM_ECUDA, "gridcon: %s", cudaGetErrorString(e));
    }
    for (auto p : dv) cudaFree(p);
    return rc;
}

int inmsom_r_diss(inmsom_ctx *c, double r_fric, double *r_diss)
{
    CKR(ensure_grid(c));
    if (!c->tmp[0]) CKR(dalloc(c, &c->tmp[0], sizeof(double)));
    CKR(h2d(c, c->tmp[0], (const double *)r_diss));
    general::r_diss(c->dom, c->gdev(), r_fric, c->tmp[0], c->stream);
    CKR(d2h(c, r_diss, c->tmp[0]));
    return sync_stream(c);
}

int inmsom_wind_forcing(inmsom_ctx *c, const double *taux, const double *tauy, double *RHSx2d,
                        double *RHSy2d)
{
    CKR(ensure_grid(c));
    for (int k = 0; k < 4; k++)
        if (!c->tmp[k]) CKR(dalloc(c, &c->tmp[k], sizeof(double)));
    CKR(h2d(c, c->tmp[0], taux));
    CKR(h2d(c, c->tmp[1], tauy));
    CKR(h2d(c, c->tmp[2], (const double *)RHSx2d));
    CKR(h2d(c, c->tmp[3], (const double *)RHSy2d));
    general::wind_forcing(c->dom, c->gdev(), c->c, c->tmp[0], c->tmp[1], c->tmp[2], c->tmp[3],
                          c->stream);
    CKR(d2h(c, RHSx2d, c->tmp[2]));
    CKR(d2h(c, RHSy2d, c->tmp[3]));
    return sync_stream(c);
}

int inmsom_rhs2d(inmsom_ctx *c, double *RHSx2d, double *RHSy2d, const double *RHSx2d_diff_disp,
                 const double *RHSy2d_diff_disp, const double *RHSx2d_tran, const double *RHSy2d_tran,
                 const double *RHSx2d_tran_disp, const double *RHSy2d_tran_disp, const double *surf_stress_x,
                 const double *surf_stress_y, const double *bot_stress_x, const double *bot_stress_y,
                 const double *slpr, const double *hhu, const double *hhv)
{
    CKR(ensure_grid(c));
    if (!RHSx2d || !RHSy2d) return set_err(INMSOM_EARG, "inmsom_rhs2d: NULL RHSx2d or RHSy2d");
    if (slpr && (!hhu || !hhv)) return set_err(INMSOM_EARG, "inmsom_rhs2d: slpr needs hhu and hhv");
    CKR(alloc_block(c, c->r2d, 7));   // zeroed once; field 6 stays zero
    double **r = c->r2d, *zero = c->r2d[6];
    // an input on the device, or the zero field for a NULL argument (a
    // missing term adds or subtracts 0, as in the reference with the term zero)
    auto in = [&](double *dev, const double *host, int *rc) -> const double * {
        if (!host) return zero;
        *rc = h2d(c, dev, host);
        return dev;
    };
    int rc = INMSOM_OK;
    CKR(h2d(c, r[0], (const double *)RHSx2d));
    CKR(h2d(c, r[1], (const double *)RHSy2d));
    const GridDev g = c->gdev();
    const double *pairs[3][2] = {{RHSx2d_diff_disp, RHSy2d_diff_disp}, {RHSx2d_tran, RHSy2d_tran},
                                 {RHSx2d_tran_disp, RHSy2d_tran_disp}};
    const int term_of[3] = {0, 1, 0};
    for (int t = 0; t < 3; t++) {
        const double *ax = in(r[2], pairs[t][0], &rc), *ay = in(r[3], pairs[t][1], &rc);
        CKR(rc);
        general::rhs2d_term(c->dom, g, c->c, term_of[t], r[0], r[1], ax, ay, nullptr, nullptr, c->stream);
    }
    {
        const double *ax = in(r[2], surf_stress_x, &rc), *bx = in(r[3], bot_stress_x, &rc);
        const double *ay = in(r[4], surf_stress_y, &rc), *by = in(r[5], bot_stress_y, &rc);
        CKR(rc);
        general::rhs2d_term(c->dom, g, c->c, 2, r[0], r[1], ax, ay, bx, by, c->stream);
    }
    {
        const double *a = in(r[2], slpr, &rc), *bx = in(r[3], hhu, &rc), *by = in(r[4], hhv, &rc);
        CKR(rc);
        general::rhs2d_term(c->dom, g, c->c, 3, r[0], r[1], a, a, bx, by, c->stream);
    }
    CK(cudaGetLastError());
    CKR(d2h(c, RHSx2d, r[0]));
    CKR(d2h(c, RHSy2d, r[1]));
    return sync_stream(c);
}

int inmsom_velocity2d(inmsom_ctx *c, double *uu2d, double *vv2d, double *pgrx, double *pgry,
                      const double *ubrtr_i, const double *vbrtr_i, const double *slpr, const double *hhu,
                      const double *hhv)
{
    CKR(ensure_grid(c));
    double *const out[4] = {uu2d, vv2d, pgrx, pgry};
    const double *in[5] = {ubrtr_i, vbrtr_i, slpr, hhu, hhv};
    for (auto *p : out)
        if (!p) return set_err(INMSOM_EARG, "inmsom_velocity2d: NULL argument");
    for (auto *p : in)
        if (!p) return set_err(INMSOM_EARG, "inmsom_velocity2d: NULL argument");
    CKR(alloc_block(c, c->v2d, 9));
    double **v = c->v2d;
    for (int k = 0; k < 4; k++) CKR(h2d(c, v[k], (const double *)out[k]));
    for (int k = 0; k < 5; k++) CKR(h2d(c, v[4 + k], in[k]));
    general::velocity2d(c->dom, c->gdev(), c->c, v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], c->stream);
    CK(cudaGetLastError());
    for (int k = 0; k < 4; k++) CKR(d2h(c, out[k], v[k]));
    return sync_stream(c);
}

int inmsom_hh_init_external(inmsom_ctx *c, const double *ssh_e, const double *sshp_e)
{
    CKR(ensure_grid(c));
    CKR(h2d(c, c->state[S_SSH], ssh_e));
    CKR(h2d(c, c->state[S_SSHP], sshp_e));
    fused::mark_state_changed(c->plan);
    depths_from_state(c);
    for (int k = 0; k < NDEPTH; k++)
        if (c->h_depth[k]) CKR(d2h(c, c->h_depth[k], c->depth[k]));
    // the other state fields are not known here: the next call uploads them
    c->state_on_device = false;
    return sync_stream(c);
}

int inmsom_guard(inmsom_ctx *c, long *nbad)
{
    CKR(ensure_grid(c));
    if (!nbad) return set_err(INMSOM_EARG, "nbad is NULL");
    if (!c->state_on_device) return set_err(INMSOM_EARG, "no resident state");
    return run_guard(c, nbad);
}

int inmsom_gpu_diag(inmsom_ctx *c, double *volume, double *energy)
{
    CKR(ensure_grid(c));
    if (!volume || !energy) return set_err(INMSOM_EARG, "NULL output");
    if (!c->state_on_device) return set_err(INMSOM_EARG, "no resident state");
    if (!c->depths_current) depths_from_state(c);
    const int nrows = c->dom.ny_end - c->dom.ny_start + 1;
    general::diag_rows(c->dom, c->gdev(), c->c, c->state[S_SSH], c->state[S_U], c->state[S_V],
                       c->depth[H_U], c->depth[H_V], c->d_rows, c->stream);
    general::diag_final(nrows, c->d_rows, c->d_out, c->stream);
    double h[2];
    CK(cudaMemcpyAsync(h, c->d_out, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CKR(sync_stream(c));
    *volume = h[0];
    *energy = h[1];
    return INMSOM_OK;
}

int inmsom_gpu_sync_to_host(inmsom_ctx *c, unsigned what)
{
    CKR(ensure_grid(c));
    if (what & INMSOM_SYNC_STATE) {
        if (!c->state_on_device) return set_err(INMSOM_EARG, "no resident state");
        for (int k = 0; k < NSTATE; k++) CKR(d2h(c, c->h_state[k], c->state[k]));
    }
    if (what & INMSOM_SYNC_DEPTHS) {
        if (!c->depths_current) depths_from_state(c);
        for (int k = 0; k < NDEPTH; k++)
            if (c->h_depth[k]) CKR(d2h(c, c->h_depth[k], c->depth[k]));
    }
    if (what & INMSOM_SYNC_SCRATCH)
        for (int k = 0; k < NSCR; k++) CKR(d2h(c, c->h_scr[k], c->scr[k]));
    return sync_stream(c);
}

int inmsom_gpu_sync_from_host(inmsom_ctx *c, unsigned what)
{
    CKR(ensure_grid(c));
    if (what & INMSOM_SYNC_STATE) {
        for (int k = 0; k < NSTATE; k++) CKR(h2d(c, c->state[k], (const double *)c->h_state[k]));
        c->state_on_device = true;
        fused::mark_state_changed(c->plan);
        if (c->fused_ok) c->depths_current = false;
    }
    if (what & INMSOM_SYNC_DEPTHS) {
        for (int k = 0; k < NDEPTH; k++)
            if (c->h_depth[k]) CKR(h2d(c, c->depth[k], (const double *)c->h_depth[k]));
        c->depths_current = true;
    }
    if (what & INMSOM_SYNC_SCRATCH) {
        for (int k = 0; k < NSCR; k++) CKR(h2d(c, c->scr[k], (const double *)c->h_scr[k]));
        c->scratch_on_device = true;
    }
    if (what & INMSOM_SYNC_COEFFS)
        for (int k = 0; k < NFORC; k++) c->coef_on_device[k] = false;
    return sync_stream(c);
}

}  // extern "C"

// ===========================================================================
// Ensemble of contexts advanced by one CUDA graph per group of substeps.
constexpr int ENS_MIN_ROWS = 16;   // shortest work item of an ensemble member

struct inmsom_ens {
    std::vector<inmsom_ctx *> m;
    int device = 0, group = 2;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t exec = nullptr;
    std::vector<double> graph_dt;          // dt per member the graph was captured with
    std::vector<unsigned> graph_gen;       // plan generation per member at capture
    std::vector<const double *> graph_src; // state set per member at capture (an odd run moves the state)
    std::vector<double> graph_prep;        // forcing mode per member at capture (variant, mu0, rd0, wq0)
    double *d_rs = nullptr;                // RHS scale per substep of the run
    size_t rs_cap = 0;
    int *d_base = nullptr;                 // first substep of the next group
    bool persistent = false;               // one persistent launch per group (fused::ens_launch)
    fused::EnsTable table;                 // its device tables (rebuilt with the graph)
};

namespace {

void ens_drop_graph(inmsom_ens *e)
{
    if (e->exec) cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
    fused::ens_free(e->table);
    e->graph_dt.clear();
    e->graph_gen.clear();
    e->graph_src.clear();
    e->graph_prep.clear();
}

int ens_capture(inmsom_ens *e, const double *dt)
{
    ens_drop_graph(e);
    if (e->persistent) {
        std::vector<fused::EnsMemberIn> in;
        for (size_t i = 0; i < e->m.size(); i++) {
            inmsom_ctx *c = e->m[i];
            in.push_back({&c->plan, &c->dom, &c->c, dt[i], c->state});
        }
        if (fused::ens_table(in, e->group, e->d_rs, e->d_base, e->table, e->origin))
            return set_err(INMSOM_ECUDA, "persistent ensemble tables: %s", cudaGetErrorString(cudaGetLastError()));
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal));
    int rc = INMSOM_OK;
    cudaError_t ce = cudaEventRecord(e->fork, e->origin);
    if (e->persistent && ce == cudaSuccess && fused::ens_launch(e->table, e->origin))
        rc = set_err(INMSOM_ECUDA, "persistent ensemble launch failed during graph capture");
    for (size_t i = 0; i < e->m.size() && !e->persistent && ce == cudaSuccess && rc == INMSOM_OK; i++) {
        inmsom_ctx *c = e->m[i];
        ce = cudaStreamWaitEvent(c->stream, e->fork, 0);
        if (ce == cudaSuccess &&
            fused::launch_steps(c->plan, c->dom, c->c, dt[i], e->group, e->d_rs, e->d_base, c->state, c->stream))
            rc = set_err(INMSOM_ECUDA, "ensemble member %zu: launch failed during graph capture", i);
        if (ce == cudaSuccess && rc == INMSOM_OK) ce = cudaEventRecord(e->join[i], c->stream);
        if (ce == cudaSuccess && rc == INMSOM_OK) ce = cudaStreamWaitEvent(e->origin, e->join[i], 0);
    }
    if (ce == cudaSuccess && rc == INMSOM_OK) {
        k_advance<<<1, 1, 0, e->origin>>>(e->d_base, e->group);
        ce = cudaGetLastError();
    }
    cudaError_t ee = cudaStreamEndCapture(e->origin, &g);
    if (rc != INMSOM_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess || ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return set_err(INMSOM_ECUDA, "ensemble graph capture failed: %s",
                       cudaGetErrorString(ce != cudaSuccess ? ce : ee));
    }
    ce = cudaGraphInstantiate(&e->exec, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return set_err(INMSOM_ECUDA, "ensemble graph instantiate: %s", cudaGetErrorString(ce));
    e->graph_dt.assign(dt, dt + e->m.size());
    for (auto *c : e->m) e->graph_gen.push_back(c->plan.generation);
    for (auto *c : e->m) e->graph_src.push_back(c->state[0]);
    for (auto *c : e->m)
        e->graph_prep.insert(e->graph_prep.end(),
                             {(double)c->plan.prep_gen, c->plan.prep_mu0, c->plan.prep_rd0, c->plan.prep_wq0});
    return INMSOM_OK;
}

bool ens_graph_current(const inmsom_ens *e, const double *dt)
{
    if (!e->exec) return false;
    for (size_t i = 0; i < e->m.size(); i++)
        if (e->graph_dt[i] != dt[i] || e->graph_gen[i] != e->m[i]->plan.generation ||
            e->graph_src[i] != e->m[i]->state[0])
            return false;
    for (size_t i = 0; i < e->m.size(); i++) {
        const fused::Plan &p = e->m[i]->plan;
        const double *g = &e->graph_prep[4 * i];
        if (g[0] != (double)p.prep_gen || g[1] != p.prep_mu0 || g[2] != p.prep_rd0 || g[3] != p.prep_wq0) return false;
    }
    return true;
}

}  // namespace

int inmsom_ens_create(inmsom_ens **out, inmsom_ctx *const *members, int n, int group)
{
    if (!out || !members || n < 1) return set_err(INMSOM_EARG, "inmsom_ens_create: no members");
    *out = nullptr;
    if (group < 2 || group % 2) return set_err(INMSOM_EARG, "group = %d must be even and >= 2", group);
    for (int i = 0; i < n; i++) {
        inmsom_ctx *c = members[i];
        if (!c || !c->grid_ok) return set_err(INMSOM_EARG, "member %d: grid not registered", i);
        if (!c->fused_ok) return set_err(INMSOM_EUNSUPPORTED, "member %d: fused path not eligible (%s)", i, c->fused_reason);
        if (c->flags & INMSOM_FP32_VELOCITY)
            return set_err(INMSOM_EUNSUPPORTED, "member %d: the ensemble runs FP64 state only", i);
        if (c->device != members[0]->device) return set_err(INMSOM_EARG, "member %d on another device", i);
        for (int j = 0; j < i; j++)
            if (members[j] == c) return set_err(INMSOM_EARG, "member %d is member %d again", i, j);
    }
    CK(cudaSetDevice(members[0]->device));
    inmsom_ens *e = new inmsom_ens();
    e->m.assign(members, members + n);
    e->device = members[0]->device;
    e->group = group;
    cudaError_t ce = cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e->ev0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e->ev1);
    e->join.assign(n, nullptr);
    for (int i = 0; i < n && ce == cudaSuccess; i++) ce = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaMalloc(&e->d_base, sizeof(int));
    // members share the device: items of 16 rows at least (a basin alone
    // cuts down to 4 to spread a small basin over more SMs)
    for (int i = 0; i < n && ce == cudaSuccess; i++) {
        inmsom_ctx *c = members[i];
        if (c->plan.min_rows == ENS_MIN_ROWS) continue;
        c->plan.min_rows = ENS_MIN_ROWS;
        if (fused::repartition(c->plan, c->dom, c->plan.rows_per_item[0], c->stream)) {
            ce = cudaGetLastError();
            if (ce == cudaSuccess) ce = cudaErrorUnknown;
        }
    }
    if (ce != cudaSuccess) {
        inmsom_ens_destroy(e);
        return set_err(INMSOM_ECUDA, "inmsom_ens_create: %s", cudaGetErrorString(ce));
    }
    *out = e;
    return INMSOM_OK;
}

int inmsom_ens_persistent(inmsom_ens *e, int on)
{
    if (!e) return set_err(INMSOM_EARG, "NULL ensemble");
    if (e->persistent != (on != 0)) {
        CK(cudaSetDevice(e->device));
        ens_drop_graph(e);
        e->persistent = on != 0;
    }
    return INMSOM_OK;
}

int inmsom_ens_run(inmsom_ens *e, int nsub, const double *dt, const double *rhs_scale, float *ms)
{
    if (!e || !dt) return set_err(INMSOM_EARG, "NULL argument");
    if (nsub < 0) return set_err(INMSOM_EARG, "nsub < 0");
    CK(cudaSetDevice(e->device));
    const size_t n = e->m.size();
    for (size_t i = 0; i < n; i++) {
        inmsom_ctx *c = e->m[i];
        if (!(dt[i] > 0.0)) return set_err(INMSOM_EARG, "member %zu: dt must be > 0", i);
        if (!c->state_on_device) return set_err(INMSOM_EARG, "member %zu: no resident state", i);
        if (fused::prepare_steps(c->plan, c->dom, c->c, c->state, c->forc, c->stream))
            return set_err(INMSOM_ECUDA, "member %zu: prepare failed: %s", i, cudaGetErrorString(cudaGetLastError()));
        // the graph orders after the origin stream only: finish the copies
        // prepare_steps left on the member's stream
        CK(cudaStreamSynchronize(c->stream));
    }
    // RHS scale of every substep on the device, read by the kernels at the
    // device-side substep counter
    const size_t need = (size_t)std::max(nsub, 1);
    if (need > e->rs_cap) {
        ens_drop_graph(e);   // the graph holds the old buffer
        cudaFree(e->d_rs);
        e->d_rs = nullptr;
        e->rs_cap = 0;
        CK(cudaMalloc(&e->d_rs, need * sizeof(double)));
        e->rs_cap = need;
    }
    std::vector<double> rs(need, 1.0);
    if (rhs_scale)
        for (int k = 0; k < nsub; k++) rs[k] = rhs_scale[k];
    CK(cudaMemcpyAsync(e->d_rs, rs.data(), need * sizeof(double), cudaMemcpyHostToDevice, e->origin));
    CK(cudaMemsetAsync(e->d_base, 0, sizeof(int), e->origin));
    if (!ens_graph_current(e, dt)) CKR(ens_capture(e, dt));
    CK(cudaEventRecord(e->ev0, e->origin));
    const int groups = nsub / e->group, rest = nsub % e->group;
    for (int g = 0; g < groups; g++) CK(cudaGraphLaunch(e->exec, e->origin));
    if (rest) {
        // the remaining substeps, launched directly on the member streams
        CK(cudaEventRecord(e->fork, e->origin));
        for (size_t i = 0; i < n; i++) {
            inmsom_ctx *c = e->m[i];
            CK(cudaStreamWaitEvent(c->stream, e->fork, 0));
            if (fused::launch_steps(c->plan, c->dom, c->c, dt[i], rest, e->d_rs, e->d_base, c->state, c->stream))
                return set_err(INMSOM_ECUDA, "member %zu: launch failed", i);
            CK(cudaEventRecord(e->join[i], c->stream));
            CK(cudaStreamWaitEvent(e->origin, e->join[i], 0));
        }
    }
    CK(cudaEventRecord(e->ev1, e->origin));
    CK(cudaStreamSynchronize(e->origin));
    CK(cudaGetLastError());
    for (size_t i = 0; i < n; i++) {
        inmsom_ctx *c = e->m[i];
        if (fused::finish_steps(c->plan, c->stream))
            return set_err(INMSOM_ECUDA, "member %zu: %s", i, cudaGetErrorString(cudaGetLastError()));
        c->depths_current = false;
        if (c->plan.last_flags & (fused::FLAG_TIMEOUT | fused::FLAG_SMEM)) return fused_flag_error(c, "ensemble member");
    }
    if (ms) CK(cudaEventElapsedTime(ms, e->ev0, e->ev1));
    return INMSOM_OK;
}

int inmsom_ens_tune(inmsom_ens *e, const double *dt, int trial_groups, int *rows_out)
{
    if (!e || !dt) return set_err(INMSOM_EARG, "NULL argument");
    if (trial_groups < 1) return set_err(INMSOM_EARG, "trial_groups < 1");
    CK(cudaSetDevice(e->device));
    const int cand[] = {0, 96, 64, 48, 32};
    const size_t n = e->m.size();
    // size classes: side length rounded to 256
    std::vector<int> cls(n);
    int ncls = 0;
    for (size_t i = 0; i < n; i++) {
        const Dom &d = e->m[i]->dom;
        const double side = std::sqrt((double)(d.nx_end - d.nx_start + 1) * (d.ny_end - d.ny_start + 1));
        cls[i] = (int)std::lround(side / 256.0);
        ncls = std::max(ncls, cls[i] + 1);
    }
    // the members' cut before tuning, timed like the candidates: kept unless
    // the tuned combination (chosen class by class, the other classes as
    // they stand) is faster as a whole
    std::vector<int> start(n), chosen(n);
    for (size_t i = 0; i < n; i++) chosen[i] = start[i] = e->m[i]->plan.rows_per_item[0];
    float base = 0.0f, tuned = 0.0f;
    CKR(inmsom_ens_run(e, e->group * trial_groups, dt, nullptr, &base));   // warm-up, captures
    CKR(inmsom_ens_run(e, e->group * trial_groups, dt, nullptr, &base));
    for (int k = 0; k < ncls; k++) {
        bool any = false;
        for (size_t i = 0; i < n; i++) any |= cls[i] == k;
        if (!any) continue;
        float best = INFINITY;
        int best_c = 0;
        for (int cnd : cand) {
            for (size_t i = 0; i < n; i++)
                if (cls[i] == k && fused::repartition(e->m[i]->plan, e->m[i]->dom, cnd, e->m[i]->stream))
                    return set_err(INMSOM_ECUDA, "member %zu: repartition failed", i);
            float ms = 0.0f;
            CKR(inmsom_ens_run(e, e->group * trial_groups, dt, nullptr, &ms));   // warm-up, captures
            CKR(inmsom_ens_run(e, e->group * trial_groups, dt, nullptr, &ms));
            if (ms < best) {
                best = ms;
                best_c = cnd;
            }
        }
        for (size_t i = 0; i < n; i++)
            if (cls[i] == k) {
                if (fused::repartition(e->m[i]->plan, e->m[i]->dom, best_c, e->m[i]->stream))
                    return set_err(INMSOM_ECUDA, "member %zu: repartition failed", i);
                chosen[i] = best_c;
            }
    }
    CKR(inmsom_ens_run(e, e->group * trial_groups, dt, nullptr, &tuned));
    CKR(inmsom_ens_run(e, e->group * trial_groups, dt, nullptr, &tuned));
    if (tuned > base)
        for (size_t i = 0; i < n; i++) {
            if (fused::repartition(e->m[i]->plan, e->m[i]->dom, start[i], e->m[i]->stream))
                return set_err(INMSOM_ECUDA, "member %zu: repartition failed", i);
            chosen[i] = start[i];
        }
    if (rows_out)
        for (size_t i = 0; i < n; i++) rows_out[i] = chosen[i];
    return INMSOM_OK;
}

int inmsom_ens_destroy(inmsom_ens *e)
{
    if (!e) return INMSOM_OK;
    cudaSetDevice(e->device);
    if (e->origin) cudaStreamSynchronize(e->origin);
    ens_drop_graph(e);
    for (auto ev : e->join)
        if (ev) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->origin) cudaStreamDestroy(e->origin);
    cudaFree(e->d_rs);
    cudaFree(e->d_base);
    delete e;
    return INMSOM_OK;
}

// ===========================================================================
// Row strips of one basin: one fused substep per strip, then the rows next
// to every internal boundary copied into the neighbour's halo rows.
struct inmsom_strips {
    std::vector<inmsom_ctx *> m;
    std::vector<cudaEvent_t> done;   // per strip: its substep kernel finished
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

// copy rows [r, r+nrows) of the six fields of `from`'s current state set into
// rows [h, h+1] of `to`'s, on `to`'s stream... or the stream given
int copy_rows(const inmsom_ctx *from, int r, inmsom_ctx *to, int h, int nrows, cudaStream_t s)
{
    const size_t pitch_b = (size_t)from->dom.pitch * sizeof(double);
    const size_t fs_from = (size_t)from->dom.pitch * from->dom.nya() * sizeof(double);
    const size_t fs_to = (size_t)to->dom.pitch * to->dom.nya() * sizeof(double);
    CK(cudaMemcpy2DAsync(to->state[0] + (size_t)h * to->dom.pitch, fs_to, from->state[0] + (size_t)r * from->dom.pitch,
                         fs_from, (size_t)nrows * pitch_b, NSTATE, cudaMemcpyDefault, s));
    return INMSOM_OK;
}

// halo rows south / north of the interior
int halo_s(const inmsom_ctx *c) { return c->dom.ny_start - c->dom.bnd_y1; }
int halo_n(const inmsom_ctx *c) { return c->dom.bnd_y2 - c->dom.ny_end; }

}  // namespace

int inmsom_strips_create(inmsom_strips **out, inmsom_ctx *const *ctxs, int n)
{
    if (!out || !ctxs || n < 1) return set_err(INMSOM_EARG, "inmsom_strips_create: no strips");
    *out = nullptr;
    for (int k = 0; k < n; k++) {
        const inmsom_ctx *c = ctxs[k];
        if (!c || !c->grid_ok) return set_err(INMSOM_EARG, "strip %d: grid not registered", k);
        if (!c->fused_ok) return set_err(INMSOM_EUNSUPPORTED, "strip %d: fused path not eligible (%s)", k, c->fused_reason);
        if (c->flags & INMSOM_FP32_VELOCITY) return set_err(INMSOM_EUNSUPPORTED, "strip %d: FP64 state only", k);
        if (k > 0) {
            const Dom &a = ctxs[k - 1]->dom, &b = c->dom;
            if (a.ny_end + 1 != b.ny_start || a.nx_start != b.nx_start || a.nx_end != b.nx_end ||
                a.bnd_x1 != b.bnd_x1 || a.bnd_x2 != b.bnd_x2 || a.pitch != b.pitch || a.nnn != b.nnn || a.nn != b.nn)
                return set_err(INMSOM_EARG, "strips %d and %d are not consecutive row strips of one basin", k - 1, k);
            if (halo_n(ctxs[k - 1]) != halo_s(c) || halo_s(c) > b.ny_end - b.ny_start + 1 ||
                halo_n(ctxs[k - 1]) > a.ny_end - a.ny_start + 1)
                return set_err(INMSOM_EARG, "strips %d and %d: halo widths differ or exceed a strip", k - 1, k);
        }
    }
    if (ctxs[0]->dom.ny_start != ctxs[0]->dom.nnn || ctxs[n - 1]->dom.ny_end != ctxs[n - 1]->dom.nn)
        return set_err(INMSOM_EARG, "the strips do not cover the basin's rows nnn..nn");
    // peer access between neighbouring strips on different devices
    for (int k = 0; k + 1 < n; k++) {
        const int a = ctxs[k]->device, b = ctxs[k + 1]->device;
        if (a == b) continue;
        int ok_ab = 0, ok_ba = 0;
        CK(cudaDeviceCanAccessPeer(&ok_ab, a, b));
        CK(cudaDeviceCanAccessPeer(&ok_ba, b, a));
        if (!ok_ab || !ok_ba) return set_err(INMSOM_EUNSUPPORTED, "devices %d and %d lack peer access", a, b);
        for (int t = 0; t < 2; t++) {
            CK(cudaSetDevice(t ? b : a));
            const cudaError_t e = cudaDeviceEnablePeerAccess(t ? a : b, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled) (void)cudaGetLastError();
            else CK(e);
        }
    }
    inmsom_strips *g = new inmsom_strips();
    g->m.assign(ctxs, ctxs + n);
    g->done.assign(n, nullptr);
    cudaError_t ce = cudaSuccess;
    for (int k = 0; k < n && ce == cudaSuccess; k++) {
        ce = cudaSetDevice(ctxs[k]->device);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&g->done[k], cudaEventDisableTiming);
    }
    if (ce == cudaSuccess) ce = cudaSetDevice(ctxs[0]->device);
    if (ce == cudaSuccess) ce = cudaEventCreate(&g->ev0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&g->ev1);
    if (ce != cudaSuccess) {
        inmsom_strips_destroy(g);
        return set_err(INMSOM_ECUDA, "inmsom_strips_create: %s", cudaGetErrorString(ce));
    }
    *out = g;
    return INMSOM_OK;
}

int inmsom_strips_run(inmsom_strips *g, int nsub, double dt, const double *rhs_scale, float *ms)
{
    if (!g) return set_err(INMSOM_EARG, "NULL argument");
    if (nsub < 0) return set_err(INMSOM_EARG, "nsub < 0");
    if (!(dt > 0.0)) return set_err(INMSOM_EARG, "dt must be > 0");
    const int n = (int)g->m.size();
    for (int k = 0; k < n; k++) {
        inmsom_ctx *c = g->m[k];
        if (!c->state_on_device) return set_err(INMSOM_EARG, "strip %d: no resident state", k);
        CK(cudaSetDevice(c->device));
        if (fused::prepare_steps(c->plan, c->dom, c->c, c->state, c->forc, c->stream))
            return set_err(INMSOM_ECUDA, "strip %d: prepare failed: %s", k, cudaGetErrorString(cudaGetLastError()));
    }
    inmsom_ctx *c0 = g->m[0];
    CK(cudaSetDevice(c0->device));
    CK(cudaEventRecord(g->ev0, c0->stream));
    for (int k = 1; k < n; k++) {   // every strip starts after ev0
        CK(cudaSetDevice(g->m[k]->device));
        CK(cudaStreamWaitEvent(g->m[k]->stream, g->ev0, 0));
    }
    // k substeps per exchange, k = half the narrowest halo between strips
    // (1 with 2-row halos): in substep i of a block each strip also computes
    // 2(k-i) rows into its halo on the sides it shares with another strip,
    // which that strip computes alike, so that after k substeps the 2k
    // halo rows are exchanged once
    int kb = 1 << 20;
    for (int k = 0; k + 1 < n; k++) kb = std::min(kb, halo_n(g->m[k]) / 2);
    if (n == 1) kb = 1;
    for (int step = 0; step < nsub;) {
        const int len = std::min(kb, nsub - step);
        for (int i = 1; i <= len; i++, step++) {
            const double rs = rhs_scale ? rhs_scale[step] : 1.0;
            for (int k = 0; k < n; k++) {
                inmsom_ctx *c = g->m[k];
                CK(cudaSetDevice(c->device));
                const int es = k > 0 ? 2 * (len - i) : 0, en = k + 1 < n ? 2 * (len - i) : 0;
                if (fused::launch_step_ext(c->plan, c->dom, c->c, dt, es, en, c->state, c->stream, rs))
                    return set_err(INMSOM_ECUDA, "strip %d: launch failed", k);
            }
        }
        for (int k = 0; k < n; k++) {
            CK(cudaSetDevice(g->m[k]->device));
            CK(cudaEventRecord(g->done[k], g->m[k]->stream));
        }
        // halo rows of the new state: strip k's 2k northernmost interior
        // rows into k+1's southern halo, k+1's 2k southernmost into k's
        // northern halo
        for (int k = 0; k + 1 < n; k++) {
            inmsom_ctx *a = g->m[k], *b = g->m[k + 1];
            const int w = halo_n(a);
            const int a_last = a->dom.ny_end - a->dom.bnd_y1;   // device row of ny_end
            CK(cudaSetDevice(b->device));
            CK(cudaStreamWaitEvent(b->stream, g->done[k], 0));
            CKR(copy_rows(a, a_last - w + 1, b, 0, w, b->stream));
            CK(cudaSetDevice(a->device));
            CK(cudaStreamWaitEvent(a->stream, g->done[k + 1], 0));
            CKR(copy_rows(b, w, a, a_last + 1, w, a->stream));
        }
    }
    // ev1 after every strip's last work
    for (int k = 0; k < n; k++) {
        CK(cudaSetDevice(g->m[k]->device));
        CK(cudaEventRecord(g->done[k], g->m[k]->stream));
    }
    CK(cudaSetDevice(c0->device));
    for (int k = 1; k < n; k++) CK(cudaStreamWaitEvent(c0->stream, g->done[k], 0));
    CK(cudaEventRecord(g->ev1, c0->stream));
    for (int k = 0; k < n; k++) {
        inmsom_ctx *c = g->m[k];
        CK(cudaSetDevice(c->device));
        if (fused::finish_steps(c->plan, c->stream))
            return set_err(INMSOM_ECUDA, "strip %d: %s", k, cudaGetErrorString(cudaGetLastError()));
        c->depths_current = false;
        if (c->plan.last_flags & (fused::FLAG_TIMEOUT | fused::FLAG_SMEM)) return fused_flag_error(c, "strip");
    }
    CK(cudaSetDevice(c0->device));
    CK(cudaEventSynchronize(g->ev1));
    if (ms) CK(cudaEventElapsedTime(ms, g->ev0, g->ev1));
    return INMSOM_OK;
}

int inmsom_step_begin(inmsom_ctx *c)
{
    CKR(ensure_grid(c));
    if (!c->state_on_device) return set_err(INMSOM_EARG, "no resident state: call inmsom_load_state first");
    if (!c->fused_ok) return set_err(INMSOM_EUNSUPPORTED, "fused path not eligible (%s)", c->fused_reason);
    if (c->flags & INMSOM_FP32_VELOCITY) return set_err(INMSOM_EUNSUPPORTED, "row strips keep an FP64 state");
    if (fused::prepare_steps(c->plan, c->dom, c->c, c->state, c->forc, c->stream))
        return set_err(INMSOM_ECUDA, "prepare failed: %s", cudaGetErrorString(cudaGetLastError()));
    return INMSOM_OK;
}

int inmsom_step_launch(inmsom_ctx *c, double dt, double rhs_scale)
{
    return inmsom_step_launch_rows(c, dt, rhs_scale, 0, 0);
}

int inmsom_step_launch_rows(inmsom_ctx *c, double dt, double rhs_scale, int rows_south, int rows_north)
{
    if (!c) return set_err(INMSOM_EARG, "context is NULL");
    if (!c->plan.prepared) return set_err(INMSOM_EARG, "inmsom_step_begin has not been called");
    if (!(dt > 0.0)) return set_err(INMSOM_EARG, "dt must be > 0");
    if (rows_south < 0 || rows_north < 0 || rows_south > halo_s(c) - 2 || rows_north > halo_n(c) - 2 ||
        (rows_south && c->dom.ny_start == c->dom.nnn) || (rows_north && c->dom.ny_end == c->dom.nn))
        return set_err(INMSOM_EARG, "inmsom_step_launch_rows: %d / %d rows beyond the interior need a halo 2 rows "
                                    "wider on a side shared with another strip (halo %d / %d)",
                       rows_south, rows_north, halo_s(c), halo_n(c));
    CK(cudaSetDevice(c->device));
    if (fused::launch_step_ext(c->plan, c->dom, c->c, dt, rows_south, rows_north, c->state, c->stream, rhs_scale))
        return set_err(INMSOM_ECUDA, "substep launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    c->depths_current = false;
    return INMSOM_OK;
}

int inmsom_gpu_halo(inmsom_ctx *c, int *rows_south, int *rows_north)
{
    if (!c || !rows_south || !rows_north) return set_err(INMSOM_EARG, "NULL argument");
    CKR(ensure_grid(c));
    *rows_south = halo_s(c);
    *rows_north = halo_n(c);
    return INMSOM_OK;
}

namespace {
// device row of the first of the w rows a side packs (interior) or unpacks
// (halo), w the side's halo width: south w / 0, north ny_end-w+1 / ny_end+1
// (relative to bnd_y1)
int halo_row(const inmsom_ctx *c, int side, bool pack)
{
    const int last = c->dom.ny_end - c->dom.bnd_y1;
    if (side == 0) return pack ? halo_s(c) : 0;
    return pack ? last - halo_n(c) + 1 : last + 1;
}
}  // namespace

int inmsom_halo_pack(inmsom_ctx *c, int side, void *buf)
{
    CKR(ensure_grid(c));
    if (!buf || (side != 0 && side != 1)) return set_err(INMSOM_EARG, "inmsom_halo_pack: bad argument");
    const size_t row_b = (size_t)c->dom.pitch * sizeof(double);
    const size_t fs = row_b * c->dom.nya();
    const size_t w = (size_t)(side ? halo_n(c) : halo_s(c));
    CK(cudaMemcpy2DAsync(buf, w * row_b, c->state[0] + (size_t)halo_row(c, side, true) * c->dom.pitch, fs,
                         w * row_b, NSTATE, cudaMemcpyDeviceToDevice, c->stream));
    return INMSOM_OK;
}

int inmsom_halo_unpack(inmsom_ctx *c, int side, const void *buf)
{
    CKR(ensure_grid(c));
    if (!buf || (side != 0 && side != 1)) return set_err(INMSOM_EARG, "inmsom_halo_unpack: bad argument");
    const size_t row_b = (size_t)c->dom.pitch * sizeof(double);
    const size_t fs = row_b * c->dom.nya();
    const size_t w = (size_t)(side ? halo_n(c) : halo_s(c));
    CK(cudaMemcpy2DAsync(c->state[0] + (size_t)halo_row(c, side, false) * c->dom.pitch, fs, buf, w * row_b,
                         w * row_b, NSTATE, cudaMemcpyDeviceToDevice, c->stream));
    return INMSOM_OK;
}

int inmsom_step_end(inmsom_ctx *c)
{
    CKR(ensure_grid(c));
    if (fused::finish_steps(c->plan, c->stream))
        return set_err(INMSOM_ECUDA, "substeps: %s", cudaGetErrorString(cudaGetLastError()));
    if (c->plan.last_flags & (fused::FLAG_TIMEOUT | fused::FLAG_SMEM)) return fused_flag_error(c, "fused kernel");
    return INMSOM_OK;
}

void *inmsom_gpu_stream(inmsom_ctx *c) { return c ? (void *)c->stream : nullptr; }

long long inmsom_gpu_pitch(inmsom_ctx *c) { return c ? c->dom.pitch : 0; }

int inmsom_strips_destroy(inmsom_strips *g)
{
    if (!g) return INMSOM_OK;
    for (size_t k = 0; k < g->m.size(); k++) {
        cudaSetDevice(g->m[k]->device);
        if (g->m[k]->stream) cudaStreamSynchronize(g->m[k]->stream);
        if (g->done[k]) cudaEventDestroy(g->done[k]);
    }
    if (!g->m.empty()) cudaSetDevice(g->m[0]->device);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    delete g;
    return INMSOM_OK;
}
