// Per-loop kernels of the barotropic step (see general.h).  Compiled with
// --fmad=false: each expression below is written in the evaluation order of
// the Fortran line it cites (left to right through * / + - chains), so the
// rounding matches a non-contracting Fortran build.
#include "general.h"

namespace inmsom {
namespace general {

namespace {

constexpr int BX = 32, BY = 8;

// Launch over the inclusive index range [m0,m1] x [n0,n1].
template <typename K, typename... A>
void launch2d(K k, int m0, int m1, int n0, int n1, cudaStream_t s, A... a)
{
    if (m1 < m0 || n1 < n0) return;
    dim3 blk(BX, BY);
    dim3 grd((m1 - m0 + BX) / BX, (n1 - n0 + BY) / BY);
    k<<<grd, blk, 0, s>>>(m0, m1, n0, n1, a...);
}

#define RANGE_GUARD                                   \
    const int m = m0 + blockIdx.x * BX + threadIdx.x; \
    const int n = n0 + blockIdx.y * BY + threadIdx.y; \
    if (m > m1 || n > n1) return;
#define X(m_, n_) ix(D, (m_), (n_))

__global__ void k_fill(int m0, int m1, int n0, int n1, Dom D, double *f, double v)
{
    RANGE_GUARD
    f[X(m, n)] = v;
}

__global__ void k_copy(int m0, int m1, int n0, int n1, Dom D, double *dst, const double *src)
{
    RANGE_GUARD
    dst[X(m, n)] = src[X(m, n)];
}

// Service/oc_algorithms.f90:50-95 (wrap: ff(mmm-1)=ff(mm), ff(mm+1)=ff(mmm))
__global__ void k_cyclize_x(Dom D, double *f)
{
    const int n = D.bnd_y1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > D.bnd_y2) return;
    double left = f[X(D.mm, n)], right = f[X(D.mmm, n)];
    f[X(D.mmm - 1, n)] = left;
    f[X(D.mm + 1, n)] = right;
}

// Service/oc_algorithms.f90:118-135
__global__ void k_cyclize_y(Dom D, double *f)
{
    const int m = D.bnd_x1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (m > D.bnd_x2) return;
    f[X(m, D.nnn - 1)] = f[X(m, D.nn)];
    f[X(m, D.nn + 1)] = f[X(m, D.nnn)];
}

// ---- depth interpolation, Function/depth.f90:29-66 ----------------------
__device__ __forceinline__ double h_on_u(const Dom &D, const GridDev &g, const double *hq, int m, int n)
{
    const float *lu = g.lu;
    double slu = (double)(lu[X(m, n)] + lu[X(m + 1, n)]);
    return (hq[X(m, n)] * g.dx[X(m, n)] * g.dy[X(m, n)] * (double)lu[X(m, n)]
            + hq[X(m + 1, n)] * g.dx[X(m + 1, n)] * g.dy[X(m + 1, n)] * (double)lu[X(m + 1, n)])
           / slu / g.dxt[X(m, n)] / g.dyh[X(m, n)];
}
__device__ __forceinline__ double h_on_v(const Dom &D, const GridDev &g, const double *hq, int m, int n)
{
    const float *lu = g.lu;
    double slu = (double)(lu[X(m, n)] + lu[X(m, n + 1)]);
    return (hq[X(m, n)] * g.dx[X(m, n)] * g.dy[X(m, n)] * (double)lu[X(m, n)]
            + hq[X(m, n + 1)] * g.dx[X(m, n + 1)] * g.dy[X(m, n + 1)] * (double)lu[X(m, n + 1)])
           / slu / g.dxh[X(m, n)] / g.dyt[X(m, n)];
}
__device__ __forceinline__ double h_on_h(const Dom &D, const GridDev &g, const double *hq, int m, int n)
{
    const float *lu = g.lu;
    double slu = (double)(lu[X(m, n)] + lu[X(m + 1, n)] + lu[X(m, n + 1)] + lu[X(m + 1, n + 1)]);
    return (hq[X(m, n)] * g.dx[X(m, n)] * g.dy[X(m, n)] * (double)lu[X(m, n)]
            + hq[X(m + 1, n)] * g.dx[X(m + 1, n)] * g.dy[X(m + 1, n)] * (double)lu[X(m + 1, n)]
            + hq[X(m, n + 1)] * g.dx[X(m, n + 1)] * g.dy[X(m, n + 1)] * (double)lu[X(m, n + 1)]
            + hq[X(m + 1, n + 1)] * g.dx[X(m + 1, n + 1)] * g.dy[X(m + 1, n + 1)] * (double)lu[X(m + 1, n + 1)])
           / slu / g.dxb[X(m, n)] / g.dyb[X(m, n)];
}

// hq = h_r + sh*ffs over the whole array (depth.f90:21-23, :121)
__global__ void k_hq_set(int m0, int m1, int n0, int n1, Dom D, const double *hr,
                         double *hq, const double *sh, double ffs, int use_sh)
{
    RANGE_GUARD
    hq[X(m, n)] = use_sh ? hr[X(m, n)] + sh[X(m, n)] * ffs : hr[X(m, n)];
}

// depth.f90:25-70 / :123-152 for one time level
__global__ void k_hh_interp(int m0, int m1, int n0, int n1, Dom D, GridDev g,
                            const double *hq, double *hu, double *hv, double *hh)
{
    RANGE_GUARD
    if (g.llu[X(m, n)] > 0.5f) hu[X(m, n)] = h_on_u(D, g, hq, m, n);
    if (g.llv[X(m, n)] > 0.5f) hv[X(m, n)] = h_on_v(D, g, hq, m, n);
    if (g.luh[X(m, n)] > 0.5f) hh[X(m, n)] = h_on_h(D, g, hq, m, n);
}

__device__ __forceinline__ double asselin(double ts, double f, double fn, double fp, double div2, double ns)
{
    // f + ts*(fn - 2f + fp)/2/nstep, rounded as f + (((ts*((fn-2f)+fp))/2)/nstep)
    return f + ts * (fn - 2.0 * f + fp) / div2 / ns;
}

// depth.f90:191-217
struct H12 { double *p[12]; };
__global__ void k_hh_shift(int m0, int m1, int n0, int n1, Dom D, GridDev g, double ts,
                           H12 h, double ns)
{
    RANGE_GUARD
    const long long i = X(m, n);
    double *hq = h.p[0], *hqp = h.p[1], *hqn = h.p[2];
    double *hu = h.p[3], *hup = h.p[4], *hun = h.p[5];
    double *hv = h.p[6], *hvp = h.p[7], *hvn = h.p[8];
    double *hh = h.p[9], *hhp = h.p[10], *hhn = h.p[11];
    if (g.llu[i] > 0.5f) { hup[i] = asselin(ts, hu[i], hun[i], hup[i], 2.0, ns); hu[i] = hun[i]; }
    if (g.llv[i] > 0.5f) { hvp[i] = asselin(ts, hv[i], hvn[i], hvp[i], 2.0, ns); hv[i] = hvn[i]; }
    if (g.lu[i] > 0.5f)  { hqp[i] = asselin(ts, hq[i], hqn[i], hqp[i], 2.0, ns); hq[i] = hqn[i]; }
    if (g.luh[i] > 0.5f) { hhp[i] = asselin(ts, hh[i], hhn[i], hhp[i], 2.0, ns); hh[i] = hhn[i]; }
}

// ---- Function/mixing.f90:129-153 ---------------------------------------
__global__ void k_stress(int m0, int m1, int n0, int n1, Dom D, GridDev g,
                         const double *u, const double *v, double *str_t, double *str_s)
{
    RANGE_GUARD
    const double *dx = g.dx, *dy = g.dy, *dxh = g.dxh, *dyh = g.dyh;
    const double *dxt = g.dxt, *dyt = g.dyt, *dxb = g.dxb, *dyb = g.dyb;
    if (g.lu[X(m, n)] > 0.5f)
        str_t[X(m, n)] = dy[X(m, n)] / dx[X(m, n)] * (u[X(m, n)] / dyh[X(m, n)] - u[X(m - 1, n)] / dyh[X(m - 1, n)])
                       - dx[X(m, n)] / dy[X(m, n)] * (v[X(m, n)] / dxh[X(m, n)] - v[X(m, n - 1)] / dxh[X(m, n - 1)]);
    if (g.luu[X(m, n)] > 0.5f)
        str_s[X(m, n)] = dxb[X(m, n)] / dyb[X(m, n)] * (u[X(m, n + 1)] / dxt[X(m, n + 1)] - u[X(m, n)] / dxt[X(m, n)])
                       + dyb[X(m, n)] / dxb[X(m, n)] * (v[X(m + 1, n)] / dyt[X(m + 1, n)] - v[X(m, n)] / dyt[X(m, n)]);
}

// ---- Function/vel_ssh.f90:30-42 ------------------------------------------
__global__ void k_vort(int m0, int m1, int n0, int n1, Dom D, GridDev g,
                       const double *u, const double *v, double *vort)
{
    RANGE_GUARD
    if (g.luu[X(m, n)] > 0.5f) {
        const double *dxt = g.dxt, *dyt = g.dyt, *dxb = g.dxb, *dyb = g.dyb;
        vort[X(m, n)] = (v[X(m + 1, n)] * dyt[X(m + 1, n)] - v[X(m, n)] * dyt[X(m, n)])
                      - (u[X(m, n + 1)] * dxt[X(m, n + 1)] - u[X(m, n)] * dxt[X(m, n)])
                      - ((v[X(m + 1, n)] - v[X(m, n)]) * dyb[X(m, n)] - (u[X(m, n + 1)] - u[X(m, n)]) * dxb[X(m, n)]);
    }
}

// ---- Function/vel_ssh.f90:54-109 -----------------------------------------
__global__ void k_trans(int m0, int m1, int n0, int n1, Dom D, GridDev g,
                        const double *u, const double *v, const double *vort,
                        const double *hu, const double *hv, const double *hh,
                        double *rhsx, double *rhsy)
{
    RANGE_GUARD
    const double *dxh = g.dxh, *dyh = g.dyh;
    if (g.lcu[X(m, n)] > 0.5f) {
        double fx_p = (u[X(m, n)] * dyh[X(m, n)] * hu[X(m, n)] + u[X(m + 1, n)] * dyh[X(m + 1, n)] * hu[X(m + 1, n)]) / 2.0
                      * (u[X(m, n)] + u[X(m + 1, n)]) / 2.0;
        double fx_m = (u[X(m, n)] * dyh[X(m, n)] * hu[X(m, n)] + u[X(m - 1, n)] * dyh[X(m - 1, n)] * hu[X(m - 1, n)]) / 2.0
                      * (u[X(m, n)] + u[X(m - 1, n)]) / 2.0;
        double fy_p = (v[X(m, n)] * dxh[X(m, n)] * hv[X(m, n)] + v[X(m + 1, n)] * dxh[X(m + 1, n)] * hv[X(m + 1, n)]) / 2.0
                      * (u[X(m, n + 1)] + u[X(m, n)]) / 2.0 * (double)g.luu[X(m, n)];
        double fy_m = (v[X(m, n - 1)] * dxh[X(m, n - 1)] * hv[X(m, n - 1)] + v[X(m + 1, n - 1)] * dxh[X(m + 1, n - 1)] * hv[X(m + 1, n - 1)]) / 2.0
                      * (u[X(m, n - 1)] + u[X(m, n)]) / 2.0 * (double)g.luu[X(m, n - 1)];
        rhsx[X(m, n)] = -(fx_p - fx_m + fy_p - fy_m)
                        + (vort[X(m, n)] * hh[X(m, n)] * (v[X(m + 1, n)] + v[X(m, n)])
                           + vort[X(m, n - 1)] * hh[X(m, n - 1)] * (v[X(m + 1, n - 1)] + v[X(m, n - 1)])) / 4.0;
    }
    if (g.lcv[X(m, n)] > 0.5f) {
        double fy_p = (v[X(m, n)] * dxh[X(m, n)] * hv[X(m, n)] + v[X(m, n + 1)] * dxh[X(m, n + 1)] * hv[X(m, n + 1)]) / 2.0
                      * (v[X(m, n)] + v[X(m, n + 1)]) / 2.0;
        double fy_m = (v[X(m, n)] * dxh[X(m, n)] * hv[X(m, n)] + v[X(m, n - 1)] * dxh[X(m, n - 1)] * hv[X(m, n - 1)]) / 2.0
                      * (v[X(m, n)] + v[X(m, n - 1)]) / 2.0;
        double fx_p = (u[X(m, n)] * dyh[X(m, n)] * hu[X(m, n)] + u[X(m, n + 1)] * dyh[X(m, n + 1)] * hu[X(m, n + 1)]) / 2.0
                      * (v[X(m + 1, n)] + v[X(m, n)]) / 2.0;
        double fx_m = (u[X(m - 1, n)] * dyh[X(m - 1, n)] * hu[X(m - 1, n)] + u[X(m - 1, n + 1)] * dyh[X(m - 1, n + 1)] * hu[X(m - 1, n + 1)]) / 2.0
                      * (v[X(m - 1, n)] + v[X(m, n)]) / 2.0;
        rhsy[X(m, n)] = -(fx_p - fx_m + fy_p - fy_m)
                        - (vort[X(m, n)] * hh[X(m, n)] * (u[X(m, n + 1)] + u[X(m, n)])
                           + vort[X(m - 1, n)] * hh[X(m - 1, n)] * (u[X(m - 1, n + 1)] + u[X(m - 1, n)])) / 4.0;
    }
}

// ---- stress divergence, Function/vel_ssh.f90:150-172 ---------------------
__device__ __forceinline__ double dif_xt(const Dom &D, const GridDev &g, const double *mu,
                                         const double *str_t, const double *hq, int m, int n)
{
    double dy1 = g.dy[X(m + 1, n)], dy0 = g.dy[X(m, n)];
    return (dy1 * dy1 * mu[X(m + 1, n)] * hq[X(m + 1, n)] * str_t[X(m + 1, n)]
            - dy0 * dy0 * mu[X(m, n)] * hq[X(m, n)] * str_t[X(m, n)]) / g.dyh[X(m, n)];
}
__device__ __forceinline__ double dif_xs(const Dom &D, const GridDev &g, const double *mu,
                                         const double *str_s, const double *hh, int m, int n)
{
    double muh_p = (mu[X(m, n)] + mu[X(m + 1, n)] + mu[X(m, n + 1)] + mu[X(m + 1, n + 1)]) / 4.0;
    double muh_m = (mu[X(m, n)] + mu[X(m + 1, n)] + mu[X(m, n - 1)] + mu[X(m + 1, n - 1)]) / 4.0;
    double b0 = g.dxb[X(m, n)], b1 = g.dxb[X(m, n - 1)];
    return (b0 * b0 * muh_p * hh[X(m, n)] * str_s[X(m, n)]
            - b1 * b1 * muh_m * hh[X(m, n - 1)] * str_s[X(m, n - 1)]) / g.dxt[X(m, n)];
}
__device__ __forceinline__ double dif_yt(const Dom &D, const GridDev &g, const double *mu,
                                         const double *str_t, const double *hq, int m, int n)
{
    double dx1 = g.dx[X(m, n + 1)], dx0 = g.dx[X(m, n)];
    return (dx1 * dx1 * mu[X(m, n + 1)] * hq[X(m, n + 1)] * str_t[X(m, n + 1)]
            - dx0 * dx0 * mu[X(m, n)] * hq[X(m, n)] * str_t[X(m, n)]) / g.dxh[X(m, n)];
}
__device__ __forceinline__ double dif_ys(const Dom &D, const GridDev &g, const double *mu,
                                         const double *str_s, const double *hh, int m, int n)
{
    double muh_p = (mu[X(m, n)] + mu[X(m + 1, n)] + mu[X(m, n + 1)] + mu[X(m + 1, n + 1)]) / 4.0;
    double muh_m = (mu[X(m, n)] + mu[X(m - 1, n)] + mu[X(m, n + 1)] + mu[X(m - 1, n + 1)]) / 4.0;
    double b0 = g.dyb[X(m, n)], b1 = g.dyb[X(m - 1, n)];
    return (b0 * b0 * muh_p * hh[X(m, n)] * str_s[X(m, n)]
            - b1 * b1 * muh_m * hh[X(m - 1, n)] * str_s[X(m - 1, n)]) / g.dyt[X(m, n)];
}

// Function/vel_ssh.f90:141-179 (mode 0) and :274-312 (mode 1, accumulate)
__global__ void k_diff(int m0, int m1, int n0, int n1, Dom D, GridDev g, const double *mu,
                       const double *str_t, const double *str_s, const double *hq,
                       const double *hh, double *rhsx, double *rhsy, int accumulate)
{
    RANGE_GUARD
    const long long i = X(m, n);
    if (g.lcu[i] > 0.5f) {
        double a = dif_xt(D, g, mu, str_t, hq, m, n), b = dif_xs(D, g, mu, str_s, hh, m, n);
        rhsx[i] = accumulate ? rhsx[i] + a + b : a + b;
    }
    if (g.lcv[i] > 0.5f) {
        double a = dif_yt(D, g, mu, str_t, hq, m, n), b = dif_ys(D, g, mu, str_s, hh, m, n);
        rhsy[i] = accumulate ? rhsy[i] - a + b : -a + b;
    }
}

// Function/vel_ssh.f90:216-257 (normalised harmonic operator of uv_diff4)
__global__ void k_diff4_first(int m0, int m1, int n0, int n1, Dom D, GridDev g, const double *mu,
                              const double *str_t, const double *str_s, const double *hq,
                              const double *hu, const double *hv, const double *hh,
                              double *fx, double *fy)
{
    RANGE_GUARD
    const long long i = X(m, n);
    if (g.lcu[i] > 0.5f) {
        double f = dif_xt(D, g, mu, str_t, hq, m, n) + dif_xs(D, g, mu, str_s, hh, m, n);
        fx[i] = -f / hu[i] / g.dxt[i] / g.dyh[i];
    }
    if (g.lcv[i] > 0.5f) {
        double f = -dif_yt(D, g, mu, str_t, hq, m, n) + dif_ys(D, g, mu, str_s, hh, m, n);
        fy[i] = -f / hv[i] / g.dxh[i] / g.dyt[i];
    }
}

// ---- Function/vel_ssh.f90:487-499 and :707-719 ---------------------------
__global__ void k_continuity(int m0, int m1, int n0, int n1, Dom D, GridDev g, Consts c,
                             double dt, double *sshn, const double *sshp, const double *u,
                             const double *v, const double *hu, const double *hv,
                             const double *wflux)
{
    RANGE_GUARD
    if (g.lu[X(m, n)] > 0.5f) {
        const double *dxh = g.dxh, *dyh = g.dyh;
        double div;
        if (hu)
            div = u[X(m, n)] * hu[X(m, n)] * dyh[X(m, n)] - u[X(m - 1, n)] * hu[X(m - 1, n)] * dyh[X(m - 1, n)]
                  + v[X(m, n)] * hv[X(m, n)] * dxh[X(m, n)] - v[X(m, n - 1)] * hv[X(m, n - 1)] * dxh[X(m, n - 1)];
        else
            div = u[X(m, n)] * dyh[X(m, n)] - u[X(m - 1, n)] * dyh[X(m - 1, n)]
                  + v[X(m, n)] * dxh[X(m, n)] - v[X(m, n - 1)] * dxh[X(m, n - 1)];
        sshn[X(m, n)] = sshp[X(m, n)] + 2.0 * dt * (wflux[X(m, n)] / c.rho * (double)c.ffs
                                                    - div / (g.dx[X(m, n)] * g.dy[X(m, n)]));
    }
}

// ---- Function/vel_ssh.f90:531-573 ------------------------------------------
__global__ void k_momentum(int m0, int m1, int n0, int n1, Dom D, GridDev g, Consts c,
                           double ti, double four_nstep, MomentumArgs a)
{
    RANGE_GUARD
    const long long i = X(m, n);
    const double *dxt = g.dxt, *dyt = g.dyt, *dxh = g.dxh, *dyh = g.dyh;
    const double *dxb = g.dxb, *dyb = g.dyb, *rlh = g.rlh;
    const double grav = c.g;
    if (g.lcu[i] > 0.5f) {
        double bp = a.hun[i] * dxt[i] * dyh[i] / 2.0 / ti;
        double bp0 = a.hup[i] * dxt[i] * dyh[i] / 2.0 / ti;
        double slx = -grav * (a.ssh[X(m + 1, n)] - a.ssh[i]) * dyh[i] * a.hu[i];
        double slxn = -grav * (a.sshn[X(m + 1, n)] - a.sshn[i]) * dyh[i] * a.hun[i];
        double grx = a.rhsx[i] * a.rhs_scale + slx + a.difx[i] + a.advx[i]
                     - (a.rdis[i] + a.rdis[X(m + 1, n)]) / 2.0 * a.up[i] * dxt[i] * dyh[i] * a.hu[i]
                     + (rlh[i] * a.hh[i] * dxb[i] * dyb[i] * (a.v[X(m + 1, n)] + a.v[i])
                        + rlh[X(m, n - 1)] * a.hh[X(m, n - 1)] * dxb[X(m, n - 1)] * dyb[X(m, n - 1)]
                          * (a.v[X(m + 1, n - 1)] + a.v[X(m, n - 1)])) / 4.0;
        double un = (a.up[i] * bp0 + grx) / bp;
        a.un[i] = un;
        a.ubrtr_i[i] = a.ubrtr_i[i] + (a.u[i] * a.hu[i] + un * a.hun[i]) / four_nstep;
        a.gx[i] = a.gx[i] + (slx + slxn) / four_nstep;
    }
    if (g.lcv[i] > 0.5f) {
        double bp = a.hvn[i] * dyt[i] * dxh[i] / 2.0 / ti;
        double bp0 = a.hvp[i] * dyt[i] * dxh[i] / 2.0 / ti;
        double sly = -grav * (a.ssh[X(m, n + 1)] - a.ssh[i]) * dxh[i] * a.hv[i];
        double slyn = -grav * (a.sshn[X(m, n + 1)] - a.sshn[i]) * dxh[i] * a.hvn[i];
        double gry = a.rhsy[i] * a.rhs_scale + sly + a.dify[i] + a.advy[i]
                     - (a.rdis[i] + a.rdis[X(m, n + 1)]) / 2.0 * a.vp[i] * dxh[i] * dyt[i] * a.hv[i]
                     - (rlh[i] * a.hh[i] * dxb[i] * dyb[i] * (a.u[X(m, n + 1)] + a.u[i])
                        + rlh[X(m - 1, n)] * a.hh[X(m - 1, n)] * dxb[X(m - 1, n)] * dyb[X(m - 1, n)]
                          * (a.u[X(m - 1, n + 1)] + a.u[X(m - 1, n)])) / 4.0;
        double vn = (a.vp[i] * bp0 + gry) / bp;
        a.vn[i] = vn;
        a.vbrtr_i[i] = a.vbrtr_i[i] + (a.v[i] * a.hv[i] + vn * a.hvn[i]) / four_nstep;
        a.gy[i] = a.gy[i] + (sly + slyn) / four_nstep;
    }
}

// ---- Function/vel_ssh.f90:589-612 / :738-749 -------------------------------
__global__ void k_asselin3(int m0, int m1, int n0, int n1, Dom D, GridDev g, double ts,
                           double div2, double ns, double *ssh, double *sshp, const double *sshn,
                           double *u, double *up, const double *un, double *v, double *vp,
                           const double *vn)
{
    RANGE_GUARD
    const long long i = X(m, n);
    if (g.lu[i] > 0.5f) { sshp[i] = asselin(ts, ssh[i], sshn[i], sshp[i], div2, ns); ssh[i] = sshn[i]; }
    if (u && g.lcu[i] > 0.5f) { up[i] = asselin(ts, u[i], un[i], up[i], div2, ns); u[i] = un[i]; }
    if (v && g.lcv[i] > 0.5f) { vp[i] = asselin(ts, v[i], vn[i], vp[i], div2, ns); v[i] = vn[i]; }
}

// ---- Control/init_pars.f90:459-481 -----------------------------------------
__global__ void k_r_diss(int m0, int m1, int n0, int n1, Dom D, GridDev g, double r_fric, double *r)
{
    RANGE_GUARD
    if (g.lu[X(m, n)] > 0.5f) {
        const double *h = g.hrest, *dxt = g.dxt, *dyt = g.dyt;
        const float *lcu = g.lcu, *lcv = g.lcv;
        double a = (h[X(m + 1, n)] - h[X(m, n)]) / dxt[X(m, n)];
        double b = (h[X(m, n)] - h[X(m - 1, n)]) / dxt[X(m - 1, n)];
        double hx2 = (a * a * (double)lcu[X(m, n)] + b * b * (double)lcu[X(m - 1, n)])
                     / (double)(lcu[X(m, n)] + lcu[X(m - 1, n)]);
        double d = (h[X(m, n + 1)] - h[X(m, n)]) / dyt[X(m, n)];
        double e = (h[X(m, n)] - h[X(m, n - 1)]) / dyt[X(m, n - 1)];
        double hy2 = (d * d * (double)lcv[X(m, n)] + e * e * (double)lcv[X(m, n - 1)])
                     / (double)(lcv[X(m, n)] + lcv[X(m, n - 1)]);
        r[X(m, n)] = r_fric * sqrt(hx2 + hy2);
    }
}

// ---- Function/fluxes.f90:29-37 + Control/dyncall.f90:115-125 --------------
__global__ void k_wind(int m0, int m1, int n0, int n1, Dom D, GridDev g, double rho,
                       const double *taux, const double *tauy, double *rhsx, double *rhsy)
{
    RANGE_GUARD
    const long long i = X(m, n);
    const double *dx = g.dx, *dy = g.dy;
    if (g.lcu[i] > 0.5f) {
        double ss = (taux[i] * dx[i] * dy[i] + taux[X(m + 1, n)] * dx[X(m + 1, n)] * dy[X(m + 1, n)])
                    / rho / 2.0 / g.dxt[i] / g.dyh[i];
        // dyncall.f90:115-118 with the 3-D, bottom-stress and slpr terms zero
        rhsx[i] = rhsx[i] + ss * g.dxt[i] * g.dyh[i];
    }
    if (g.lcv[i] > 0.5f) {
        double ss = (tauy[i] * dx[i] * dy[i] + tauy[X(m, n + 1)] * dx[X(m, n + 1)] * dy[X(m, n + 1)])
                    / rho / 2.0 / g.dxh[i] / g.dyt[i];
        rhsy[i] = rhsy[i] + ss * g.dyt[i] * g.dxh[i];
    }
}

// ---- Control/dyncall.f90:110-130: the barotropic RHS, one term per launch
// in the reference's left-to-right order, so that every step rounds where
// the Fortran expression rounds (this file: --fmad=false, no reassociation):
// term 0: r - a; 1: r + a; 2: r + (a + b) * area; 3: r - dslpr * b * d / rho
__global__ void k_rhs2d_term(int m0, int m1, int n0, int n1, Dom D, GridDev g, double rho, int term,
                             double *rx, double *ry, const double *ax, const double *ay, const double *bx,
                             const double *by)
{
    RANGE_GUARD
    const long long i = X(m, n);
    if (g.lcu[i] > 0.5f) {
        double r = rx[i];
        if (term == 0) r = r - ax[i];
        else if (term == 1) r = r + ax[i];
        else if (term == 2) r = r + (ax[i] + bx[i]) * g.dxt[i] * g.dyh[i];
        else r = r - (ax[X(m + 1, n)] - ax[i]) * bx[i] * g.dyh[i] / rho;
        rx[i] = r;
    }
    if (g.lcv[i] > 0.5f) {
        double r = ry[i];
        if (term == 0) r = r - ay[i];
        else if (term == 1) r = r + ay[i];
        else if (term == 2) r = r + (ay[i] + by[i]) * g.dyt[i] * g.dxh[i];
        else r = r - (ay[X(m, n + 1)] - ay[i]) * by[i] * g.dxh[i] / rho;
        ry[i] = r;
    }
}

// ---- Control/dyncall.f90:188-201: corrected 2-D velocity and the slpr part
// of the time-mean pressure gradient (interior and its one-point ring)
__global__ void k_velocity2d(int m0, int m1, int n0, int n1, Dom D, GridDev g, double rho, double *uu2d,
                             double *vv2d, double *pgrx, double *pgry, const double *ubrtr_i,
                             const double *vbrtr_i, const double *slpr, const double *hhu, const double *hhv)
{
    RANGE_GUARD
    const long long i = X(m, n);
    if (g.lcu[i] > 0.5f) {
        uu2d[i] = ubrtr_i[i] / hhu[i];
        pgrx[i] = pgrx[i] - (slpr[X(m + 1, n)] - slpr[i]) * hhu[i] * g.dyh[i] / rho;
    }
    if (g.lcv[i] > 0.5f) {
        vv2d[i] = vbrtr_i[i] / hhv[i];
        pgry[i] = pgry[i] - (slpr[X(m, n + 1)] - slpr[i]) * hhv[i] * g.dxh[i] / rho;
    }
}

// ---- Service/grid_construction.f90:59-112 -----------------------------------
__global__ void k_gridcon(int m0, int m1, int n0, int n1, Dom D, const float *lu, float *luu,
                          float *luh, float *llu, float *llv, float *lcu, float *lcv)
{
    RANGE_GUARD
    float a = lu[X(m, n)], b = lu[X(m + 1, n)], cc = lu[X(m, n + 1)], d = lu[X(m + 1, n + 1)];
    if (a + b + cc + d > 0.5f) luh[X(m, n)] = 1.0f;
    if (a * b * cc * d > 0.5f) luu[X(m, n)] = 1.0f;
    if (a + b > 0.5f) llu[X(m, n)] = 1.0f;
    if (a + cc > 0.5f) llv[X(m, n)] = 1.0f;
    if (a * b > 0.5f) lcu[X(m, n)] = 1.0f;
    if (a * cc > 0.5f) lcv[X(m, n)] = 1.0f;
}

// ---- Control/dyncall.f90:452-516 ---------------------------------------------
__global__ void k_guard(int m0, int m1, int n0, int n1, Dom D, GridDev g, const double *ssh,
                        const double *u, const double *v, unsigned long long *nbad)
{
    const int m = m0 + blockIdx.x * BX + threadIdx.x;
    const int n = n0 + blockIdx.y * BY + threadIdx.y;
    unsigned bad = 0;
    if (m <= m1 && n <= n1) {
        const long long i = X(m, n);
        if (g.lu[i] > 0.5f && !(ssh[i] < 10.0 && ssh[i] > -10.0)) bad++;
        if (g.lcu[i] > 0.5f && !(u[i] < 100.0 && u[i] > -100.0)) bad++;
        if (g.lcv[i] > 0.5f && !(v[i] < 100.0 && v[i] > -100.0)) bad++;
    }
    // warp-aggregated count
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(nbad, (unsigned long long)bad);
}

// one block per interior row; fixed-order tree reduction -> deterministic
__global__ void k_diag_rows(Dom D, GridDev g, Consts c, const double *ssh, const double *u,
                            const double *v, const double *hu, const double *hv, double *rows)
{
    const int n = D.ny_start + blockIdx.x;
    const int nrows = D.ny_end - D.ny_start + 1;
    double vol = 0.0, en = 0.0;
    for (int m = D.nx_start + threadIdx.x; m <= D.nx_end; m += blockDim.x) {
        const long long i = X(m, n);
        if (g.lu[i] > 0.5f) {
            double a = g.dx[i] * g.dy[i];
            vol += (g.hrest[i] + ssh[i]) * a;
            en += 0.5 * c.g * ssh[i] * ssh[i] * a;
        }
        if (g.lcu[i] > 0.5f) en += 0.5 * hu[i] * u[i] * u[i] * g.dxt[i] * g.dyh[i];
        if (g.lcv[i] > 0.5f) en += 0.5 * hv[i] * v[i] * v[i] * g.dxh[i] * g.dyt[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        vol += __shfl_down_sync(0xffffffffu, vol, o);
        en += __shfl_down_sync(0xffffffffu, en, o);
    }
    __shared__ double sv[32], se[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sv[w] = vol; se[w] = en; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) { a += sv[k]; b += se[k]; }
        rows[blockIdx.x] = a;
        rows[nrows + blockIdx.x] = b;
    }
}

__global__ void k_diag_final(int nrows, const double *rows, double *out)
{
    // two warps sum the two columns of partials, each lane a fixed stride,
    // then a fixed shuffle tree: independent of timing
    const int col = threadIdx.x >> 5, l = threadIdx.x & 31;
    double s = 0.0;
    for (int k = l; k < nrows; k += 32) s += rows[col * nrows + k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (l == 0) out[col] = s;
}

#undef X
#undef RANGE_GUARD

}  // namespace

// ===========================================================================
void fill(const Dom &d, double *f, double v, cudaStream_t s)
{
    launch2d(k_fill, d.bnd_x1, d.bnd_x2, d.bnd_y1, d.bnd_y2, s, d, f, v);
}

void copy(const Dom &d, double *dst, const double *src, cudaStream_t s)
{
    launch2d(k_copy, d.bnd_x1, d.bnd_x2, d.bnd_y1, d.bnd_y2, s, d, dst, src);
}

void halo(const Dom &d, double *f, cudaStream_t s)
{
    if (d.px) k_cyclize_x<<<(d.nya() + 127) / 128, 128, 0, s>>>(d, f);
    if (d.py) k_cyclize_y<<<(d.nxa() + 127) / 128, 128, 0, s>>>(d, f);
}

void hh_init(const Dom &d, const GridDev &g, const Consts &c,
             double *hq, double *hqp, double *hqn, double *hu, double *hup,
             double *hun, double *hv, double *hvp, double *hvn, double *hh,
             double *hhp, double *hhn, const double *sh, const double *shp,
             cudaStream_t s)
{
    const double ffs = (double)c.ffs;
    launch2d(k_hq_set, d.bnd_x1, d.bnd_x2, d.bnd_y1, d.bnd_y2, s, d, g.hrest, hq, sh, ffs, 1);
    launch2d(k_hq_set, d.bnd_x1, d.bnd_x2, d.bnd_y1, d.bnd_y2, s, d, g.hrest, hqp, shp, ffs, 1);
    launch2d(k_hq_set, d.bnd_x1, d.bnd_x2, d.bnd_y1, d.bnd_y2, s, d, g.hrest, hqn, sh, ffs, 0);
    const int m0 = d.nx_start - 1, m1 = d.nx_end, n0 = d.ny_start - 1, n1 = d.ny_end;
    launch2d(k_hh_interp, m0, m1, n0, n1, s, d, g, (const double *)hq, hu, hv, hh);
    launch2d(k_hh_interp, m0, m1, n0, n1, s, d, g, (const double *)hqp, hup, hvp, hhp);
    launch2d(k_hh_interp, m0, m1, n0, n1, s, d, g, (const double *)hqn, hun, hvn, hhn);
    double *fs[9] = {hu, hup, hun, hv, hvp, hvn, hh, hhp, hhn};
    for (double *f : fs) halo(d, f, s);
}

void hh_update(const Dom &d, const GridDev &g, double *hqn, double *hun,
               double *hvn, double *hhn, const double *sh, cudaStream_t s)
{
    launch2d(k_hq_set, d.bnd_x1, d.bnd_x2, d.bnd_y1, d.bnd_y2, s, d, g.hrest, hqn, sh, 1.0, 1);
    launch2d(k_hh_interp, d.nx_start - 1, d.nx_end, d.ny_start - 1, d.ny_end, s, d, g,
             (const double *)hqn, hun, hvn, hhn);
    halo(d, hun, s);
    halo(d, hvn, s);
    halo(d, hhn, s);
}

void hh_shift(const Dom &d, const GridDev &g, const Consts &c, double *const h[12],
              int nstep, cudaStream_t s)
{
    H12 hp;
    for (int k = 0; k < 12; k++) hp.p[k] = h[k];
    launch2d(k_hh_shift, d.nx_start - 1, d.nx_end + 1, d.ny_start - 1, d.ny_end + 1, s, d, g,
             c.ts, hp, (double)nstep);
}

void stress_components(const Dom &d, const GridDev &g, const double *u,
                       const double *v, double *str_t, double *str_s,
                       cudaStream_t s)
{
    launch2d(k_stress, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, u, v, str_t, str_s);
    halo(d, str_t, s);
    halo(d, str_s, s);
}

void uv_trans(const Dom &d, const GridDev &g, const double *u, const double *v,
              double *vort, const double *hu, const double *hv,
              const double *hh, double *rhsx, double *rhsy, cudaStream_t s)
{
    launch2d(k_vort, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, u, v, vort);
    halo(d, vort, s);
    launch2d(k_trans, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, u, v,
             (const double *)vort, hu, hv, hh, rhsx, rhsy);
}

void uv_diff2(const Dom &d, const GridDev &g, const double *mu,
              const double *str_t, const double *str_s, const double *hq,
              const double *hh, double *rhsx, double *rhsy, cudaStream_t s)
{
    launch2d(k_diff, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, mu, str_t, str_s,
             hq, hh, rhsx, rhsy, 0);
}

void uv_diff4(const Dom &d, const GridDev &g, const double *mu, double *str_t,
              double *str_s, double *fx, double *fy, const double *hq,
              const double *hu, const double *hv, const double *hh,
              double *rhsx, double *rhsy, cudaStream_t s)
{
    fill(d, fx, 0.0, s);
    fill(d, fy, 0.0, s);
    launch2d(k_diff4_first, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, mu,
             (const double *)str_t, (const double *)str_s, hq, hu, hv, hh, fx, fy);
    halo(d, fx, s);
    halo(d, fy, s);
    stress_components(d, g, fx, fy, str_t, str_s, s);
    launch2d(k_diff, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, mu,
             (const double *)str_t, (const double *)str_s, hq, hh, rhsx, rhsy, 1);
}

void continuity(const Dom &d, const GridDev &g, const Consts &c, double dt,
                double *sshn, const double *sshp, const double *u,
                const double *v, const double *hu, const double *hv,
                const double *wflux, cudaStream_t s)
{
    launch2d(k_continuity, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, c, dt, sshn,
             sshp, u, v, hu, hv, wflux);
}

void momentum(const Dom &d, const GridDev &g, const Consts &c, double tau_inner,
              int nstep, const MomentumArgs &a, cudaStream_t s)
{
    launch2d(k_momentum, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, c, tau_inner,
             (double)(4 * nstep), a);
}

void asselin3(const Dom &d, const GridDev &g, const Consts &c, double nstep,
              double *ssh, double *sshp, const double *sshn, double *u,
              double *up, const double *un, double *v, double *vp,
              const double *vn, cudaStream_t s)
{
    // "/2.0d0/dfloat(nstep)" of vel_ssh.f90:594-606; ssh_internal's "/2.0d0"
    // (:743) is the same expression with nstep = 1 (x/1.0 is exact)
    launch2d(k_asselin3, d.nx_start - 1, d.nx_end + 1, d.ny_start - 1, d.ny_end + 1, s, d, g,
             c.ts, 2.0, nstep, ssh, sshp, sshn, u, up, un, v, vp, vn);
}

void r_diss(const Dom &d, const GridDev &g, double r_fric, double *r, cudaStream_t s)
{
    launch2d(k_r_diss, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, r_fric, r);
    halo(d, r, s);
}

void wind_forcing(const Dom &d, const GridDev &g, const Consts &c,
                  const double *taux, const double *tauy, double *rhsx,
                  double *rhsy, cudaStream_t s)
{
    launch2d(k_wind, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, c.rho, taux, tauy,
             rhsx, rhsy);
}

void velocity2d(const Dom &d, const GridDev &g, const Consts &c, double *uu2d, double *vv2d, double *pgrx,
                double *pgry, const double *ubrtr_i, const double *vbrtr_i, const double *slpr, const double *hhu,
                const double *hhv, cudaStream_t s)
{
    launch2d(k_velocity2d, d.nx_start - 1, d.nx_end + 1, d.ny_start - 1, d.ny_end + 1, s, d, g, c.rho, uu2d, vv2d,
             pgrx, pgry, ubrtr_i, vbrtr_i, slpr, hhu, hhv);
}

void rhs2d_term(const Dom &d, const GridDev &g, const Consts &c, int term, double *rx, double *ry,
                const double *ax, const double *ay, const double *bx, const double *by, cudaStream_t s)
{
    launch2d(k_rhs2d_term, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, c.rho, term, rx, ry, ax, ay,
             bx, by);
}

void gridcon(const Dom &d, const float *lu, float *luu, float *luh, float *llu,
             float *llv, float *lcu, float *lcv, cudaStream_t s)
{
    launch2d(k_gridcon, d.nx_start - 1, d.nx_end, d.ny_start - 1, d.ny_end, s, d, lu, luu,
             luh, llu, llv, lcu, lcv);
}

void guard(const Dom &d, const GridDev &g, const double *ssh, const double *u,
           const double *v, unsigned long long *nbad, cudaStream_t s)
{
    launch2d(k_guard, d.nx_start, d.nx_end, d.ny_start, d.ny_end, s, d, g, ssh, u, v, nbad);
}

void diag_rows(const Dom &d, const GridDev &g, const Consts &c,
               const double *ssh, const double *u, const double *v,
               const double *hu, const double *hv, double *rows, cudaStream_t s)
{
    const int nrows = d.ny_end - d.ny_start + 1;
    if (nrows <= 0) return;
    k_diag_rows<<<nrows, 256, 0, s>>>(d, g, c, ssh, u, v, hu, hv, rows);
}

void diag_final(int nrows, const double *rows, double *out, cudaStream_t s)
{
    k_diag_final<<<1, 64, 0, s>>>(nrows, rows, out);
}

}  // namespace general
}  // namespace inmsom
