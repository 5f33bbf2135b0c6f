// Per-water-column kernels (see column.h).  Compiled with --fmad=false; each
// expression keeps the left-to-right order of the Fortran line it cites.
//
// baroclinic_dynamics runs as two kernels:
//  1. k_columns, one thread per interior water column and velocity component
//     (grid z: 0 = u, 1 = v).  The thread builds the tridiagonal system level
//     by level, runs factor8's forward elimination as it goes (x, y of the
//     sweep kept in shared memory), then back-substitutes from the bottom and
//     applies the Robert-Asselin filter to the new velocity at once, writing
//     uu/uup (vv/vvp) to the output arrays.  The inputs stay untouched, so the
//     neighbouring columns' Coriolis and advection reads see the old state.
//  2. k_border, over every point of the arrays outside the interior: the
//     filter on the one-point ring with the new velocity the periodic wrap
//     brings there (zero without a wrap, as the reference's un = 0), a copy
//     elsewhere.
#include "column.h"

namespace inmsom {
namespace column {

namespace {

constexpr int TB = 64;          // threads (water columns) per block of k_columns
constexpr int MAX_NZ = 200;     // 2 * MAX_NZ * TB doubles of shared memory
constexpr int BX = 32, BY = 8;

#define X(m_, n_) ix(D, (m_), (n_))

// Function/vel_ssh.f90:847-983 (V = false: the u block :852-915, true: the v
// block :917-979), factor8 (Service/oc_algorithms.f90:494-524), then the
// filter of :1002-1024 at this point.
template <bool V>
__device__ __forceinline__ void solve_column(const Dom &D, const GridDev &g, const Levels &L,
                                             const BaroclinicArgs &a, double ts, int m, int n, double *xs,
                                             double *ys)
{
    const long long i = X(m, n);
    const long long P = L.plane;
    const int nz = L.nz;
    // the far end of the velocity point (u: m+1, v: n+1) and the partner of
    // the Coriolis average (u: n-1, v: m-1)
    const long long e = V ? D.pitch : 1;
    const long long p = V ? -1 : -D.pitch;
    const double *self = V ? a.vv : a.uu, *selfp = V ? a.vvp : a.uup, *other = V ? a.uu : a.vv;
    double *out = V ? a.vv_out : a.uu_out, *outp = V ? a.vvp_out : a.uup_out;
    const float mask = V ? g.lcv[i] : g.lcu[i];
    if (!(mask > 0.5f)) {
        for (int k = 0; k < nz; k++) {
            const long long o = (long long)k * P + i;
            out[o] = self[o];
            outp[o] = selfp[o];
        }
        return;
    }
    const double f1 = V ? g.dxh[i] : g.dxt[i];   // u: dxt*dyh, v: dxh*dyt
    const double f2 = V ? g.dyt[i] : g.dyh[i];
    const double hn = (V ? a.hhvn : a.hhun)[i];
    const double bp = hn * f1 * f2 / a.tau / 2.0;
    const double bp0 = (V ? a.hhvp : a.hhup)[i] * f1 * f2 / a.tau / 2.0;
    const double hc = (V ? a.hhv : a.hhu)[i];
    const double pg = (V ? a.pgry : a.pgrx)[i];
    const double tsurf = (V ? a.ty_surf : a.tx_surf)[i], tbot = (V ? a.ty_bot : a.tx_bot)[i];
    const double *rhs = V ? a.rhsy : a.rhsx, *rhst = V ? a.rhsy_tran : a.rhsx_tran;
    const double dx0 = g.dx[i], dy0 = g.dy[i], dx1 = g.dx[i + e], dy1 = g.dy[i + e];
    const double cor0 = g.rlh[i] * a.hhh[i] * g.dxb[i] * g.dyb[i];
    const double cor1 = g.rlh[i + p] * a.hhh[i + p] * g.dxb[i + p] * g.dyb[i + p];
    const double drag = (a.rdis[i] + a.rdis[i + e]) / 2.0;

    double dp = 0.0, fz_p = 0.0, xm = 0.0, ym = 0.0;
    double s0 = self[i];                                  // self at level k
    for (int k = 1; k <= nz; k++) {
        const long long o = (long long)(k - 1) * P + i;
        const double dm = dp, fz_m = fz_p;
        const double dzk = L.dz[k - 1];
        double s1 = 0.0;
        if (k < nz) {
            const long long o1 = o + P;
            dp = (a.nu[o1] + a.nu[o1 + e]) / 2.0 / hn / L.hzt[k] * f1 * f2;
            s1 = self[o1];
            fz_p = (a.ww[o1] * dx0 * dy0 + a.ww[o1 + e] * dx1 * dy1) / 2.0 * (s0 + s1) / 2.0;
        } else {
            dp = 0.0;
            fz_p = 0.0;
        }
        const double sp = selfp[o];
        const double cor = (cor0 * (other[o + e] + other[o]) + cor1 * (other[o + p + e] + other[o + p])) / 4.0;
        double eta = bp0 * sp + rhs[o] + rhst[o] + pg - (fz_p - fz_m) / dzk;
        eta = V ? eta - cor : eta + cor;
        eta = eta - drag * sp * f1 * f2 * hc;
        if (k == 1) eta = eta + tsurf / dzk * f1 * f2;
        if (k == nz) eta = eta + tbot / dzk * f1 * f2;
        const double cc = k < nz ? -dp / dzk : 0.0;
        const double bb = k == 1 ? bp + dp / dzk : (k < nz ? bp + (dp + dm) / dzk : bp + dm / dzk);
        double x, y;
        if (k == 1) {
            x = -cc / bb;
            y = eta / bb;
        } else {
            const double aa = -dm / dzk;
            const double scr = 1.0 / (aa * xm + bb);
            x = -cc * scr;
            y = (eta - aa * ym) * scr;
        }
        xs[(k - 1) * TB] = x;
        ys[(k - 1) * TB] = y;
        xm = x;
        ym = y;
        s0 = s1;
    }
    double r = ym;                                        // rksi(nz) = y(nz)
    for (int k = nz; k >= 1; k--) {
        const long long o = (long long)(k - 1) * P + i;
        if (k < nz) r = xs[(k - 1) * TB] * r + ys[(k - 1) * TB];
        const double cu = self[o];
        outp[o] = cu + ts * (r - 2.0 * cu + selfp[o]) / 2.0;
        out[o] = r;
    }
}

__global__ void __launch_bounds__(TB) k_columns(Dom D, GridDev g, Levels L, BaroclinicArgs a, double ts)
{
    extern __shared__ double sm[];
    const int m = D.nx_start + blockIdx.x * TB + threadIdx.x;
    const int n = D.ny_start + blockIdx.y;
    if (m > D.nx_end) return;
    double *xs = sm + threadIdx.x, *ys = sm + (size_t)L.nz * TB + threadIdx.x;
    if (blockIdx.z == 0) solve_column<false>(D, g, L, a, ts, m, n, xs, ys);
    else solve_column<true>(D, g, L, a, ts, m, n, xs, ys);
}

__device__ __forceinline__ int wrap(int i, bool on, int lo, int hi)
{
    if (on) {
        if (i == lo - 1) return hi;
        if (i == hi + 1) return lo;
    }
    return i;
}

// The new velocity the reference's un/vn hold at (m, n) after
// syncborder_real8 (no exchange on one domain) and cyclize8_x/_y
// (Function/vel_ssh.f90:988-998): the interior solve at the wrapped point
// where that point is an interior ocean point, else 0.
__device__ __forceinline__ double new_at(const Dom &D, const float *mask, const double *out, long long lev, int m,
                                         int n)
{
    const int mw = wrap(m, D.px, D.mmm, D.mm), nw = wrap(n, D.py, D.nnn, D.nn);
    if (mw < D.nx_start || mw > D.nx_end || nw < D.ny_start || nw > D.ny_end) return 0.0;
    const long long j = X(mw, nw);
    return mask[j] > 0.5f ? out[lev + j] : 0.0;
}

// Function/vel_ssh.f90:1002-1024 outside the interior, one level per grid row
__global__ void k_border(Dom D, GridDev g, Levels L, BaroclinicArgs a, double ts, int count)
{
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (t0 >= count) return;
    const int nxa = D.bnd_x2 - D.bnd_x1 + 1;
    const int h0 = D.ny_start - D.bnd_y1, h1 = D.bnd_y2 - D.ny_end;
    const int w0 = D.nx_start - D.bnd_x1, w1 = D.bnd_x2 - D.nx_end;
    int m, n, t = t0;
    if (t < h0 * nxa) {
        n = D.bnd_y1 + t / nxa;
        m = D.bnd_x1 + t % nxa;
    } else if ((t -= h0 * nxa) < h1 * nxa) {
        n = D.ny_end + 1 + t / nxa;
        m = D.bnd_x1 + t % nxa;
    } else {
        t -= h1 * nxa;
        n = D.ny_start + t / (w0 + w1);
        const int c = t % (w0 + w1);
        m = c < w0 ? D.bnd_x1 + c : D.nx_end + 1 + (c - w0);
    }
    const long long i = X(m, n);
    const bool ring = m >= D.nx_start - 1 && m <= D.nx_end + 1 && n >= D.ny_start - 1 && n <= D.ny_end + 1;
    const bool fu = ring && g.lcu[i] > 0.5f, fv = ring && g.lcv[i] > 0.5f;
    {
        const long long lev = (long long)blockIdx.y * L.plane, o = lev + i;
        if (fu) {
            const double un = new_at(D, g.lcu, a.uu_out, lev, m, n), cu = a.uu[o];
            a.uup_out[o] = cu + ts * (un - 2.0 * cu + a.uup[o]) / 2.0;
            a.uu_out[o] = un;
        } else {
            a.uu_out[o] = a.uu[o];
            a.uup_out[o] = a.uup[o];
        }
        if (fv) {
            const double vn = new_at(D, g.lcv, a.vv_out, lev, m, n), cv = a.vv[o];
            a.vvp_out[o] = cv + ts * (vn - 2.0 * cv + a.vvp[o]) / 2.0;
            a.vv_out[o] = vn;
        } else {
            a.vv_out[o] = a.vv[o];
            a.vvp_out[o] = a.vvp[o];
        }
    }
}

// Function/vel_ssh.f90:1052-1063 at one interior point, bottom to top
__global__ void k_vertical_velocity(Dom D, GridDev g, Levels L, double rho, int ffs, const double *u,
                                    const double *v, double *w, const double *hu, const double *hv,
                                    const double *wflux)
{
    const int m = D.nx_start + blockIdx.x * BX + threadIdx.x;
    const int n = D.ny_start + blockIdx.y * BY + threadIdx.y;
    if (m > D.nx_end || n > D.ny_end) return;
    const long long i = X(m, n);
    if (!(g.lu[i] > 0.5f)) return;
    const long long iw = X(m - 1, n), is = X(m, n - 1);
    const double dxy = g.dx[i] * g.dy[i];
    const double hu0 = hu[i], dyh0 = g.dyh[i], hu1 = hu[iw], dyh1 = g.dyh[iw];
    const double hv0 = hv[i], dxh0 = g.dxh[i], hv1 = hv[is], dxh1 = g.dxh[is];
    const double src = wflux[i] / rho * (double)ffs;
    const long long P = L.plane;
    double wk = 0.0;
    w[(long long)L.nz * P + i] = 0.0;
    for (int k = L.nz; k >= 1; k--) {
        const long long lev = (long long)(k - 1) * P;
        wk = wk + L.dz[k - 1] / dxy *
                      (u[lev + i] * hu0 * dyh0 - u[lev + iw] * hu1 * dyh1 + v[lev + i] * hv0 * dxh0 -
                       v[lev + is] * hv1 * dxh1 + src);
        w[lev + i] = wk;
    }
}

// Service/oc_algorithms.f90:50-95 and :118-135 on every level (grid y)
__global__ void k_cyclize_x3(Dom D, long long plane, double *f)
{
    const int n = D.bnd_y1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (n > D.bnd_y2) return;
    double *fl = f + (long long)blockIdx.y * plane;
    const double left = fl[X(D.mm, n)], right = fl[X(D.mmm, n)];
    fl[X(D.mmm - 1, n)] = left;
    fl[X(D.mm + 1, n)] = right;
}

__global__ void k_cyclize_y3(Dom D, long long plane, double *f)
{
    const int m = D.bnd_x1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (m > D.bnd_x2) return;
    double *fl = f + (long long)blockIdx.y * plane;
    fl[X(m, D.nnn - 1)] = fl[X(m, D.nn)];
    fl[X(m, D.nn + 1)] = fl[X(m, D.nnn)];
}

void halo3(const Dom &d, double *f, int nlev, long long plane, cudaStream_t s)
{
    if (d.px) k_cyclize_x3<<<dim3((d.nya() + 127) / 128, nlev), 128, 0, s>>>(d, plane, f);
    if (d.py) k_cyclize_y3<<<dim3((d.nxa() + 127) / 128, nlev), 128, 0, s>>>(d, plane, f);
}

#undef X

}  // namespace

int max_levels() { return MAX_NZ; }

bool wrap_inside(const Dom &d)
{
    auto in = [](int i, int lo, int hi) { return i >= lo && i <= hi; };
    return (d.px && (in(d.mmm - 1, d.nx_start, d.nx_end) || in(d.mm + 1, d.nx_start, d.nx_end))) ||
           (d.py && (in(d.nnn - 1, d.ny_start, d.ny_end) || in(d.nn + 1, d.ny_start, d.ny_end)));
}

int baroclinic_dynamics(const Dom &d, const GridDev &g, const Consts &c, const Levels &L,
                        const BaroclinicArgs &a, cudaStream_t s)
{
    if (L.nz < 2 || L.nz > MAX_NZ || wrap_inside(d)) return -1;
    const size_t smem = 2 * (size_t)L.nz * TB * sizeof(double);
    // per device: set on every call (the context's device is current)
    if (cudaFuncSetAttribute(k_columns, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -1;
    const int nxi = d.nx_end - d.nx_start + 1, nyi = d.ny_end - d.ny_start + 1;
    k_columns<<<dim3((nxi + TB - 1) / TB, nyi, 2), TB, smem, s>>>(d, g, L, a, c.ts);
    const int count = d.nxa() * d.nya() - nxi * nyi;
    if (count > 0) k_border<<<dim3((count + 127) / 128, L.nz), 128, 0, s>>>(d, g, L, a, c.ts, count);
    return 0;
}

int vertical_velocity(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const double *u,
                      const double *v, double *w, const double *hu, const double *hv, const double *wflux,
                      cudaStream_t s)
{
    if (L.nz < 1) return -1;
    const int nxi = d.nx_end - d.nx_start + 1, nyi = d.ny_end - d.ny_start + 1;
    k_vertical_velocity<<<dim3((nxi + BX - 1) / BX, (nyi + BY - 1) / BY), dim3(BX, BY), 0, s>>>(
        d, g, L, c.rho, c.ffs, u, v, w, hu, hv, wflux);
    halo3(d, w, L.nz + 1, L.plane, s);
    return 0;
}

}  // namespace column
}  // namespace inmsom
