// C ABI of the 3-D part of the mode-split step (include/inmsom_gpu.h):
// baroclinic_dynamics, vertical_velocity, depth_ave, the barotropic shifts
// and tracer_tran_diff on the context's grid, with their nz-level device
// blocks and the row-band copy pipeline (kernels in column.cu).
#include "context.h"

#include <algorithm>
#include <functional>

#include "column.h"

extern "C" {

namespace {

// the block of the 3-D velocity calls: NC3 fields of nz levels, ww and nu
// (nz + 1 levels each), then NC2 2-D fields
enum { C3_UU, C3_UUP, C3_VV, C3_VVP, C3_RHSX, C3_RHSY, C3_RHSXT, C3_RHSYT, C3_UUO, C3_UUPO, C3_VVO, C3_VVPO, NC3 };
constexpr int NC2 = 14;

size_t col_plane(const inmsom_ctx *c) { return (size_t)c->dom.pitch * (size_t)c->dom.nya(); }
double *col3(inmsom_ctx *c, int f) { return c->col + (size_t)f * c->col_nz * col_plane(c); }
double *colw(inmsom_ctx *c, int f) { return c->col + ((size_t)NC3 * c->col_nz + (size_t)f * (c->col_nz + 1)) * col_plane(c); }
double *col2(inmsom_ctx *c, int f)
{
    return c->col + ((size_t)NC3 * c->col_nz + 2 * (size_t)(c->col_nz + 1) + f) * col_plane(c);
}

int col_alloc(inmsom_ctx *c, int nz)
{
    if (c->col && c->col_nz == nz) return INMSOM_OK;
    cudaFree(c->col);
    cudaFree(c->col_lev);
    c->col = c->col_lev = nullptr;
    c->col_nz = 0;
    const size_t planes = (size_t)NC3 * nz + 2 * (size_t)(nz + 1) + NC2;
    CK(cudaMalloc((void **)&c->col, planes * col_plane(c) * sizeof(double)));
    CK(cudaMemsetAsync(c->col, 0, planes * col_plane(c) * sizeof(double), c->stream));
    CK(cudaMalloc((void **)&c->col_lev, (2 * (size_t)nz + 2) * sizeof(double)));   // + the staged kernel's flag
    c->col_nz = nz;
    return INMSOM_OK;
}

// nlev levels of a host array (bnd_x1:bnd_x2, bnd_y1:bnd_y2, nlev): the
// host rows of consecutive levels follow each other, as do the device rows
int h2d3(inmsom_ctx *c, double *dev, const double *host, int nlev)
{
    if (!host) return set_err(INMSOM_EARG, "NULL host array");
    const size_t w = (size_t)c->dom.nxa() * sizeof(double);
    CK(cudaMemcpy2DAsync(dev + c->dom.xoff, (size_t)c->dom.pitch * sizeof(double), host, w, w,
                         (size_t)c->dom.nya() * nlev, cudaMemcpyHostToDevice, c->stream));
    return INMSOM_OK;
}

int d2h3(inmsom_ctx *c, double *host, const double *dev, int nlev)
{
    const size_t w = (size_t)c->dom.nxa() * sizeof(double);
    CK(cudaMemcpy2DAsync(host, w, dev + c->dom.xoff, (size_t)c->dom.pitch * sizeof(double), w,
                         (size_t)c->dom.nya() * nlev, cudaMemcpyDeviceToHost, c->stream));
    return INMSOM_OK;
}

// rows r0..r1 and array columns x0..x1 (0-based from bnd_x1 / bnd_y1) of
// nlev levels between a host array (bnd_x1:bnd_x2, bnd_y1:bnd_y2, nlev) and
// its pitched device copy, as one 3-D copy
int box3(inmsom_ctx *c, double *dev, double *host, int nlev, int r0, int r1, int x0, int x1, bool up,
         cudaStream_t s)
{
    if (r1 < r0 || x1 < x0) return INMSOM_OK;
    const Dom &d = c->dom;
    cudaMemcpy3DParms p = {};
    cudaPitchedPtr hp = make_cudaPitchedPtr(host, (size_t)d.nxa() * sizeof(double), (size_t)d.nxa(), (size_t)d.nya());
    cudaPitchedPtr dp = make_cudaPitchedPtr(dev + d.xoff, (size_t)d.pitch * sizeof(double), (size_t)d.nxa(),
                                            (size_t)d.nya());
    const cudaPos pos = make_cudaPos((size_t)x0 * sizeof(double), (size_t)r0, 0);
    p.srcPtr = up ? hp : dp;
    p.dstPtr = up ? dp : hp;
    p.srcPos = pos;
    p.dstPos = pos;
    p.extent = make_cudaExtent((size_t)(x1 - x0 + 1) * sizeof(double), (size_t)(r1 - r0 + 1), (size_t)nlev);
    p.kind = up ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    CK(cudaMemcpy3DAsync(&p, s));
    return INMSOM_OK;
}

// A 3-D field of a banded call: its device copy, the host array, its levels
struct Field3 {
    double *dev;
    double *host;
    int nlev;
};

// The copy pipeline of the 3-D entry points.  The interior rows are cut into
// nb bands; band b's rows of the inputs are uploaded on s_up while band b-1
// runs on the context's stream (run(n0, n1)) and band b-2's interior
// results go back on s_dn.  Each input row is uploaded once: band b brings
// the rows from just after band b-1's last to one past its own last
// interior row (run reads rows n0-1..n1+1), the last band the rest of the
// arrays.  After every band, border() runs and everything of the outputs
// outside the interior is downloaded.  pre(s_up) issues the 2-D uploads;
// flag (4 bytes on the device) is read back at the end.  The phase times
// are the uploads, the kernels' own time (CUDA events around each run and
// the border) and from the last kernel to the end.
int pipelined(inmsom_ctx *c, int nb, const std::vector<Field3> &in, const std::vector<Field3> &out,
              const std::function<int(cudaStream_t)> &pre, const std::function<int(int, int)> &run,
              const std::function<int()> &border, const int *flag_dev, int *flag)
{
    const Dom &d = c->dom;
    if (!c->s_up) CK(cudaStreamCreateWithFlags(&c->s_up, cudaStreamNonBlocking));
    if (!c->s_dn) CK(cudaStreamCreateWithFlags(&c->s_dn, cudaStreamNonBlocking));
    for (auto &e : c->bev)
        if (!e) CK(cudaEventCreate(&e));
    cudaEvent_t *ev_up = c->bev, *ev_k0 = c->bev + 8, *ev_k1 = c->bev + 16, *ev_bd = c->bev + 32;
    const int nyi = d.ny_end - d.ny_start + 1;
    nb = std::max(1, std::min(nb, std::min(8, nyi)));
    const int nxa = d.nxa(), nya = d.nya();
    const int ix0 = d.nx_start - d.bnd_x1, ix1 = d.nx_end - d.bnd_x1;      // interior, 0-based
    const int iy0 = d.ny_start - d.bnd_y1, iy1 = d.ny_end - d.bnd_y1;
    c->ph_valid = false;
    c->ph_direct = false;
    CK(cudaEventRecord(c->ph[0], c->stream));
    CK(cudaStreamWaitEvent(c->s_up, c->ph[0], 0));
    CKR(pre(c->s_up));
    int up_next = 0;
    for (int b = 0; b < nb; b++) {
        const int n0 = d.ny_start + (int)((long long)nyi * b / nb);
        const int n1 = d.ny_start + (int)((long long)nyi * (b + 1) / nb) - 1;
        const int up_last = b == nb - 1 ? nya - 1 : n1 + 1 - d.bnd_y1;
        for (const Field3 &f : in) CKR(box3(c, f.dev, f.host, f.nlev, up_next, up_last, 0, nxa - 1, true, c->s_up));
        up_next = up_last + 1;
        CK(cudaEventRecord(ev_up[b], c->s_up));
        CK(cudaStreamWaitEvent(c->stream, ev_up[b], 0));
        CK(cudaEventRecord(ev_k0[b], c->stream));
        if (run(n0, n1)) return set_err(INMSOM_ECUDA, "launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        CK(cudaGetLastError());
        CK(cudaEventRecord(ev_k1[b], c->stream));
        CK(cudaStreamWaitEvent(c->s_dn, ev_k1[b], 0));
        for (const Field3 &f : out)
            CKR(box3(c, f.dev, f.host, f.nlev, n0 - d.bnd_y1, n1 - d.bnd_y1, ix0, ix1, false, c->s_dn));
    }
    CK(cudaEventRecord(ev_bd[0], c->stream));
    if (border()) return set_err(INMSOM_ECUDA, "launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    CK(cudaGetLastError());
    CK(cudaEventRecord(ev_bd[1], c->stream));
    CK(cudaStreamWaitEvent(c->s_dn, ev_bd[1], 0));
    CK(cudaMemcpyAsync(flag, flag_dev, sizeof(int), cudaMemcpyDeviceToHost, c->s_dn));
    for (const Field3 &f : out) {
        CKR(box3(c, f.dev, f.host, f.nlev, 0, iy0 - 1, 0, nxa - 1, false, c->s_dn));             // rows above
        CKR(box3(c, f.dev, f.host, f.nlev, iy1 + 1, nya - 1, 0, nxa - 1, false, c->s_dn));       // rows below
        CKR(box3(c, f.dev, f.host, f.nlev, iy0, iy1, 0, ix0 - 1, false, c->s_dn));              // columns left
        CKR(box3(c, f.dev, f.host, f.nlev, iy0, iy1, ix1 + 1, nxa - 1, false, c->s_dn));        // columns right
    }
    CK(cudaEventRecord(c->ph[3], c->s_dn));
    CK(cudaStreamWaitEvent(c->stream, c->ph[3], 0));
    CKR(sync_stream(c));
    float t = 0.0f, sum = 0.0f;
    CK(cudaEventElapsedTime(&c->ph_ms[0], c->ph[0], ev_up[nb - 1]));
    for (int b = 0; b < nb; b++) {
        CK(cudaEventElapsedTime(&t, ev_k0[b], ev_k1[b]));
        sum += t;
    }
    CK(cudaEventElapsedTime(&t, ev_bd[0], ev_bd[1]));
    c->ph_ms[1] = sum + t;
    CK(cudaEventElapsedTime(&c->ph_ms[2], ev_bd[1], c->ph[3]));
    c->ph_direct = true;
    return INMSOM_OK;
}

column::Levels col_levels(inmsom_ctx *c)
{
    column::Levels L;
    L.nz = c->col_nz;
    L.plane = (long long)col_plane(c);
    L.dz = c->col_lev;
    L.hzt = c->col_lev + c->col_nz;
    return L;
}

}  // namespace

int inmsom_baroclinic_dynamics(inmsom_ctx *c, int nz, const double *dz, const double *hzt, double tau,
                               double *uu, double *uup, double *vv, double *vvp, const double *ww,
                               const double *nu, const double *RHSx, const double *RHSy,
                               const double *RHSx_tran, const double *RHSy_tran, const double *pgrx,
                               const double *pgry, const double *rdis, const double *tx_surf,
                               const double *ty_surf, const double *tx_bot, const double *ty_bot,
                               const double *hhu, const double *hhup, const double *hhun, const double *hhv,
                               const double *hhvp, const double *hhvn, const double *hhh)
{
    CKR(ensure_grid(c));
    if (nz < 2 || nz > column::max_levels())
        return set_err(INMSOM_EARG, "inmsom_baroclinic_dynamics: nz = %d outside 2..%d", nz, column::max_levels());
    if (!(tau > 0.0)) return set_err(INMSOM_EARG, "tau must be > 0");
    double *const io[4] = {uu, uup, vv, vvp};
    const double *in3[4] = {RHSx, RHSy, RHSx_tran, RHSy_tran};
    const double *in2[NC2] = {pgrx, pgry, rdis, tx_surf, ty_surf, tx_bot, ty_bot,
                              hhu,  hhup, hhun, hhv,     hhvp,    hhvn,   hhh};
    bool null = !dz || !hzt || !ww || !nu;
    for (auto *p : io) null = null || !p;
    for (auto *p : in3) null = null || !p;
    for (auto *p : in2) null = null || !p;
    if (null) return set_err(INMSOM_EARG, "inmsom_baroclinic_dynamics: NULL argument");
    const Dom &d = c->dom;
    if (column::wrap_inside(d)) return set_err(INMSOM_EUNSUPPORTED, "inmsom_baroclinic_dynamics: a periodic wrap column/row lies in the interior");
    CKR(col_alloc(c, nz));
    column::BaroclinicArgs a;
    a.tau = tau;
    a.uu = col3(c, C3_UU); a.uup = col3(c, C3_UUP); a.vv = col3(c, C3_VV); a.vvp = col3(c, C3_VVP);
    a.ww = colw(c, 0); a.nu = colw(c, 1);
    a.rhsx = col3(c, C3_RHSX); a.rhsy = col3(c, C3_RHSY);
    a.rhsx_tran = col3(c, C3_RHSXT); a.rhsy_tran = col3(c, C3_RHSYT);
    a.pgrx = col2(c, 0); a.pgry = col2(c, 1); a.rdis = col2(c, 2);
    a.tx_surf = col2(c, 3); a.ty_surf = col2(c, 4); a.tx_bot = col2(c, 5); a.ty_bot = col2(c, 6);
    a.hhu = col2(c, 7); a.hhup = col2(c, 8); a.hhun = col2(c, 9);
    a.hhv = col2(c, 10); a.hhvp = col2(c, 11); a.hhvn = col2(c, 12); a.hhh = col2(c, 13);
    a.uu_out = col3(c, C3_UUO); a.uup_out = col3(c, C3_UUPO); a.vv_out = col3(c, C3_VVO); a.vvp_out = col3(c, C3_VVPO);
    a.flag = reinterpret_cast<int *>(c->col_lev + 2 * nz + 1);
    const column::Levels L = col_levels(c);
    const GridDev gd = c->gdev();
    // the nz-level inputs in the order of the block's fields C3_UU .. C3_RHSYT
    double *const up3[8] = {uu, uup, vv, vvp, (double *)RHSx, (double *)RHSy, (double *)RHSx_tran,
                            (double *)RHSy_tran};
    std::vector<Field3> in, out;
    for (int k = 0; k < 8; k++) in.push_back({col3(c, C3_UU + k), up3[k], nz});
    in.push_back({colw(c, 0), (double *)ww, nz + 1});
    in.push_back({colw(c, 1), (double *)nu, nz + 1});
    for (int k = 0; k < 4; k++) out.push_back({col3(c, C3_UUO + k), io[k], nz});
    CK(cudaMemsetAsync(a.flag, 0, sizeof(int), c->stream));
    auto pre = [&](cudaStream_t su) -> int {
        for (int k = 0; k < NC2; k++)
            CK(cudaMemcpy2DAsync(col2(c, k) + d.xoff, (size_t)d.pitch * sizeof(double), in2[k],
                                 d.nxa() * sizeof(double), d.nxa() * sizeof(double), d.nya(),
                                 cudaMemcpyHostToDevice, su));
        CK(cudaMemcpyAsync(c->col_lev, dz, nz * sizeof(double), cudaMemcpyHostToDevice, su));
        CK(cudaMemcpyAsync(c->col_lev + nz, hzt, (nz + 1) * sizeof(double), cudaMemcpyHostToDevice, su));
        return INMSOM_OK;
    };
    auto run = [&](int n0, int n1) { return column::baroclinic_rows(d, gd, c->c, L, a, n0, n1, c->stream); };
    auto border = [&]() { return column::baroclinic_border(d, gd, c->c, L, a, c->stream); };
    int flag = 0;
    CKR(pipelined(c, 8, in, out, pre, run, border, a.flag, &flag));
    if (flag) return set_err(INMSOM_ETIMEOUT, "inmsom_baroclinic_dynamics: a bounded wait of the column kernel gave up");
    c->ph_valid = true;
    return INMSOM_OK;
}

namespace {

// the tracer block: TN3 fields of nz levels, TN31 of nz + 1, then TN2 2-D planes
enum { T_FF, T_FFP, T_UU, T_VV, T_MU, T_SRC, T_FFO, T_FFPO, T_FLX, T_FLY, TN3 };
enum { T_WW, T_NU, T_SLRX, T_SLRY, T_SLZX, T_SLZY, T_FZX, T_FZY, T_COX, T_COY, T_SGX, T_SGY, TN31 };
enum { T_TOP, T_BOT, T_SWB, T_HU, T_HV, T_HQN, T_HQP, T_IGT, T_IGB, T_FFX, T_FFY = T_FFX + 4, TN2 = T_FFY + 4 };

double *trc3(inmsom_ctx *c, int f) { return c->trc + (size_t)f * c->trc_nz * col_plane(c); }
double *trc31(inmsom_ctx *c, int f)
{
    return c->trc + ((size_t)TN3 * c->trc_nz + (size_t)f * (c->trc_nz + 1)) * col_plane(c);
}
double *trc2(inmsom_ctx *c, int f)
{
    return c->trc + ((size_t)TN3 * c->trc_nz + (size_t)TN31 * (c->trc_nz + 1) + f) * col_plane(c);
}

int trc_alloc(inmsom_ctx *c, int nz)
{
    if (c->trc && c->trc_nz == nz) return INMSOM_OK;
    cudaFree(c->trc);
    cudaFree(c->trc_lev);
    c->trc = c->trc_lev = nullptr;
    c->trc_nz = 0;
    const size_t planes = (size_t)TN3 * nz + (size_t)TN31 * (nz + 1) + TN2;
    CK(cudaMalloc((void **)&c->trc, planes * col_plane(c) * sizeof(double)));
    CK(cudaMemsetAsync(c->trc, 0, planes * col_plane(c) * sizeof(double), c->stream));
    CK(cudaMalloc((void **)&c->trc_lev, (2 * (size_t)nz + 2) * sizeof(double)));   // + the solve's flag
    c->trc_nz = nz;
    return INMSOM_OK;
}

}  // namespace

int inmsom_tracer_tran_diff(inmsom_ctx *c, int nz, const double *dz, const double *hzt, double *ff, double *ffp,
                            double tau, const double *uu, const double *vv, const double *ww, const double *mu,
                            double factor_mu, const double *nu, double factor_nu, const double *slrx,
                            const double *slry, const double *slzx, const double *slzy, double az, double ar,
                            double alpha_gm, const double *ff_top, const double *ff_bot, const int *ig_top,
                            const int *ig_bot, double *flux_f_x, double *flux_f_y, const double *swbal, int ksw_lbc,
                            int numlbc, const int *lqpx, const int *lqpy, const char *ind_lbc, const float *flbc,
                            const double *src, double src_factor, const double *hhu, const double *hhv,
                            const double *hhqn, const double *hhqp)
{
    (void)ksw_lbc; (void)numlbc; (void)lqpx; (void)lqpy; (void)ind_lbc; (void)flbc;   // unread by the reference too
    CKR(ensure_grid(c));
    if (nz < 2 || nz > column::max_levels())
        return set_err(INMSOM_EARG, "inmsom_tracer_tran_diff: nz = %d outside 2..%d", nz, column::max_levels());
    if (!(tau > 0.0)) return set_err(INMSOM_EARG, "tau must be > 0");
    const double *in3[6] = {ff, ffp, uu, vv, mu, src};
    const double *in31[6] = {ww, nu, slrx, slry, slzx, slzy};
    const double *in2[7] = {ff_top, ff_bot, swbal, hhu, hhv, hhqn, hhqp};
    bool null = !dz || !hzt || !ig_top || !ig_bot || !flux_f_x || !flux_f_y;
    for (auto *p : in3) null = null || !p;
    for (auto *p : in31) null = null || !p;
    for (auto *p : in2) null = null || !p;
    if (null) return set_err(INMSOM_EARG, "inmsom_tracer_tran_diff: NULL argument");
    const Dom &d = c->dom;
    if (column::wrap_inside(d))
        return set_err(INMSOM_EUNSUPPORTED, "inmsom_tracer_tran_diff: a periodic wrap column/row lies in the interior");
    // the reference sets b(1), eta(1) (b(nz), eta(nz)) only for types 1 and 2
    const int nxa = d.nxa();
    for (int n = d.ny_start; n <= d.ny_end; n++)
        for (int m = d.nx_start; m <= d.nx_end; m++) {
            const size_t i = (size_t)(n - d.bnd_y1) * nxa + (size_t)(m - d.bnd_x1);
            if (c->h_lu[i] > 0.5f && ((ig_top[i] != 1 && ig_top[i] != 2) || (ig_bot[i] != 1 && ig_bot[i] != 2)))
                return set_err(INMSOM_EARG, "inmsom_tracer_tran_diff: ig_top/ig_bot must be 1 or 2 at ocean point (%d,%d)",
                               m, n);
        }
    CKR(trc_alloc(c, nz));
    column::TracerArgs a;
    a.tau = tau; a.factor_mu = factor_mu; a.factor_nu = factor_nu; a.az = az; a.ar = ar; a.alpha_gm = alpha_gm;
    a.src_factor = src_factor;
    a.ff = trc3(c, T_FF); a.ffp = trc3(c, T_FFP); a.uu = trc3(c, T_UU); a.vv = trc3(c, T_VV);
    a.mu = trc3(c, T_MU); a.src = trc3(c, T_SRC);
    a.ww = trc31(c, T_WW); a.nu = trc31(c, T_NU); a.slrx = trc31(c, T_SLRX); a.slry = trc31(c, T_SLRY);
    a.slzx = trc31(c, T_SLZX); a.slzy = trc31(c, T_SLZY);
    a.ff_top = trc2(c, T_TOP); a.ff_bot = trc2(c, T_BOT); a.swbal = trc2(c, T_SWB); a.hhu = trc2(c, T_HU);
    a.hhv = trc2(c, T_HV); a.hhqn = trc2(c, T_HQN); a.hhqp = trc2(c, T_HQP);
    a.ig_top = reinterpret_cast<const int *>(trc2(c, T_IGT)); a.ig_bot = reinterpret_cast<const int *>(trc2(c, T_IGB));
    a.ff_out = trc3(c, T_FFO); a.ffp_out = trc3(c, T_FFPO);
    a.flux_f_x = trc2(c, T_FFX); a.flux_f_y = trc2(c, T_FFY);
    a.flux_x = trc3(c, T_FLX); a.flux_y = trc3(c, T_FLY);
    a.flux_zx = trc31(c, T_FZX); a.flux_zy = trc31(c, T_FZY); a.coef_zx = trc31(c, T_COX); a.coef_zy = trc31(c, T_COY);
    a.sfgm_zx = trc31(c, T_SGX); a.sfgm_zy = trc31(c, T_SGY);
    a.flag = reinterpret_cast<int *>(c->trc_lev + 2 * nz + 1);
    column::Levels L;
    L.nz = nz;
    L.plane = (long long)col_plane(c);
    L.dz = c->trc_lev;
    L.hzt = c->trc_lev + nz;
    const GridDev gd = c->gdev();
    const int f3[6] = {T_FF, T_FFP, T_UU, T_VV, T_MU, T_SRC};
    const int f31[6] = {T_WW, T_NU, T_SLRX, T_SLRY, T_SLZX, T_SLZY};
    std::vector<Field3> in, out;
    for (int k = 0; k < 6; k++) in.push_back({trc3(c, f3[k]), (double *)in3[k], nz});
    for (int k = 0; k < 6; k++) in.push_back({trc31(c, f31[k]), (double *)in31[k], nz + 1});
    out.push_back({trc3(c, T_FFO), ff, nz});
    out.push_back({trc3(c, T_FFPO), ffp, nz});
    out.push_back({trc2(c, T_FFX), flux_f_x, 4});
    out.push_back({trc2(c, T_FFY), flux_f_y, 4});
    CK(cudaMemsetAsync(a.flag, 0, sizeof(int), c->stream));
    auto pre = [&](cudaStream_t su) -> int {
        const size_t w = (size_t)d.nxa() * sizeof(double), dp = (size_t)d.pitch * sizeof(double);
        for (int k = 0; k < 7; k++)
            CK(cudaMemcpy2DAsync(trc2(c, T_TOP + k) + d.xoff, dp, in2[k], w, w, d.nya(), cudaMemcpyHostToDevice, su));
        const size_t wi = (size_t)d.nxa() * sizeof(int), dpi = (size_t)d.pitch * sizeof(int);
        CK(cudaMemcpy2DAsync(reinterpret_cast<int *>(trc2(c, T_IGT)) + d.xoff, dpi, ig_top, wi, wi, d.nya(),
                             cudaMemcpyHostToDevice, su));
        CK(cudaMemcpy2DAsync(reinterpret_cast<int *>(trc2(c, T_IGB)) + d.xoff, dpi, ig_bot, wi, wi, d.nya(),
                             cudaMemcpyHostToDevice, su));
        CK(cudaMemcpyAsync(c->trc_lev, dz, nz * sizeof(double), cudaMemcpyHostToDevice, su));
        CK(cudaMemcpyAsync(c->trc_lev + nz, hzt, (nz + 1) * sizeof(double), cudaMemcpyHostToDevice, su));
        return INMSOM_OK;
    };
    auto run = [&](int n0, int n1) { return column::tracer_rows(d, gd, c->c, L, a, n0, n1, c->stream); };
    auto border = [&]() { return column::tracer_border(d, gd, c->c, L, a, c->stream); };
    int flag = 0;
    // a periodic y wraps the y-fluxes of every row before any solve: one band
    CKR(pipelined(c, d.py ? 1 : 8, in, out, pre, run, border, a.flag, &flag));
    if (flag) return set_err(INMSOM_ETIMEOUT, "inmsom_tracer_tran_diff: a bounded wait of the solve gave up");
    c->ph_valid = true;
    return INMSOM_OK;
}

int inmsom_vertical_velocity(inmsom_ctx *c, int nz, const double *dz, const double *u, const double *v, double *w,
                             const double *hu, const double *hv, const double *wflux)
{
    CKR(ensure_grid(c));
    if (nz < 1) return set_err(INMSOM_EARG, "inmsom_vertical_velocity: nz = %d < 1", nz);
    if (!dz || !u || !v || !w || !hu || !hv || !wflux)
        return set_err(INMSOM_EARG, "inmsom_vertical_velocity: NULL argument");
    CKR(col_alloc(c, nz));
    c->ph_valid = false;
    c->ph_direct = false;
    CK(cudaEventRecord(c->ph[0], c->stream));
    CKR(h2d3(c, col3(c, C3_UU), u, nz));
    CKR(h2d3(c, col3(c, C3_VV), v, nz));
    CKR(h2d3(c, colw(c, 0), w, nz + 1));
    CKR(h2d(c, col2(c, 0), hu));
    CKR(h2d(c, col2(c, 1), hv));
    CKR(h2d(c, col2(c, 2), wflux));
    CK(cudaMemcpyAsync(c->col_lev, dz, nz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->ph[1], c->stream));
    column::vertical_velocity(c->dom, c->gdev(), c->c, col_levels(c), col3(c, C3_UU), col3(c, C3_VV), colw(c, 0),
                              col2(c, 0), col2(c, 1), col2(c, 2), c->stream);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ph[2], c->stream));
    CKR(d2h3(c, w, colw(c, 0), nz + 1));
    CK(cudaEventRecord(c->ph[3], c->stream));
    CKR(sync_stream(c));
    c->ph_valid = true;
    return INMSOM_OK;
}

int inmsom_depth_ave(inmsom_ctx *c, int nz, const double *dz, double *u, double *utr, const float *mask, int kbcl)
{
    CKR(ensure_grid(c));
    if (nz < 1) return set_err(INMSOM_EARG, "inmsom_depth_ave: nz = %d < 1", nz);
    if (!dz || !u || !utr || !mask) return set_err(INMSOM_EARG, "inmsom_depth_ave: NULL argument");
    CKR(col_alloc(c, nz));
    float *dmask = (float *)col2(c, 1);     // a float plane fits in a double one
    CKR(h2d3(c, col3(c, C3_UU), u, nz));
    CKR(h2d(c, col2(c, 0), (const double *)utr));
    CKR(h2d(c, dmask, mask));
    CK(cudaMemcpyAsync(c->col_lev, dz, nz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    column::depth_ave(c->dom, col_levels(c), col3(c, C3_UU), col2(c, 0), dmask, kbcl, c->stream);
    CK(cudaGetLastError());
    CKR(d2h3(c, u, col3(c, C3_UU), nz));
    CKR(d2h(c, utr, col2(c, 0)));
    return sync_stream(c);
}

int inmsom_shift_barotropic(inmsom_ctx *c, int nz, double *uu, double *vv, const double *uu2d, const double *vv2d,
                            int sign)
{
    CKR(ensure_grid(c));
    if (nz < 1) return set_err(INMSOM_EARG, "inmsom_shift_barotropic: nz = %d < 1", nz);
    if (sign != 1 && sign != -1) return set_err(INMSOM_EARG, "inmsom_shift_barotropic: sign must be +1 or -1");
    if (!uu || !vv || !uu2d || !vv2d) return set_err(INMSOM_EARG, "inmsom_shift_barotropic: NULL argument");
    CKR(col_alloc(c, nz));
    CKR(h2d3(c, col3(c, C3_UU), uu, nz));
    CKR(h2d3(c, col3(c, C3_VV), vv, nz));
    CKR(h2d(c, col2(c, 0), uu2d));
    CKR(h2d(c, col2(c, 1), vv2d));
    column::shift_barotropic(c->dom, c->gdev(), col_levels(c), col3(c, C3_UU), col3(c, C3_VV), col2(c, 0),
                             col2(c, 1), sign, c->stream);
    CK(cudaGetLastError());
    CKR(d2h3(c, uu, col3(c, C3_UU), nz));
    CKR(d2h3(c, vv, col3(c, C3_VV), nz));
    return sync_stream(c);
}

int inmsom_stress_components(inmsom_ctx *c, int nlev, const double *u, const double *v, double *str_t,
                             double *str_s)
{
    CKR(ensure_grid(c));
    if (nlev < 1 || nlev > 65535) return set_err(INMSOM_EARG, "inmsom_stress_components: nlev = %d", nlev);
    if (!u || !v || !str_t || !str_s) return set_err(INMSOM_EARG, "inmsom_stress_components: NULL argument");
    CKR(col_alloc(c, nlev));
    CKR(h2d3(c, col3(c, C3_UU), u, nlev));
    CKR(h2d3(c, col3(c, C3_VV), v, nlev));
    CKR(h2d3(c, col3(c, C3_RHSX), str_t, nlev));   // points the routine does not set keep the caller's values
    CKR(h2d3(c, col3(c, C3_RHSY), str_s, nlev));
    if (column::stress_components(c->dom, c->gdev(), col_levels(c), col3(c, C3_UU), col3(c, C3_VV),
                                  col3(c, C3_RHSX), col3(c, C3_RHSY), c->stream))
        return set_err(INMSOM_EARG, "inmsom_stress_components: bad levels");
    CK(cudaGetLastError());
    CKR(d2h3(c, str_t, col3(c, C3_RHSX), nlev));
    CKR(d2h3(c, str_s, col3(c, C3_RHSY), nlev));
    return sync_stream(c);
}

int inmsom_smagorinsky_coeff(inmsom_ctx *c, int nz, double visc2, double dift, const double *str_t,
                             const double *str_s, double *amts, double *amuv)
{
    CKR(ensure_grid(c));
    if (nz < 1 || nz > 65535) return set_err(INMSOM_EARG, "inmsom_smagorinsky_coeff: nz = %d", nz);
    if (!str_t || !str_s || !amts || !amuv) return set_err(INMSOM_EARG, "inmsom_smagorinsky_coeff: NULL argument");
    // Inc/basinpar.fi:72,89: Pi, vonkarman
    const double kp = 0.4 / 3.141592653589793;
    CKR(col_alloc(c, nz));
    CKR(h2d3(c, col3(c, C3_UU), str_t, nz));
    CKR(h2d3(c, col3(c, C3_VV), str_s, nz));
    CKR(h2d3(c, col3(c, C3_RHSX), amts, nz));      // land points keep the caller's values
    CKR(h2d3(c, col3(c, C3_RHSY), amuv, nz));
    if (column::smagorinsky_coeff(c->dom, c->gdev(), col_levels(c), visc2, dift, kp, col3(c, C3_UU),
                                  col3(c, C3_VV), col3(c, C3_RHSX), col3(c, C3_RHSY), c->stream))
        return set_err(INMSOM_EARG, "inmsom_smagorinsky_coeff: bad levels");
    CK(cudaGetLastError());
    CKR(d2h3(c, amts, col3(c, C3_RHSX), nz));
    CKR(d2h3(c, amuv, col3(c, C3_RHSY), nz));
    return sync_stream(c);
}

}  // extern "C"
