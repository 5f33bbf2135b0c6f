// Per-water-column kernels (see column.h).  Compiled with --fmad=false; each
// expression keeps the left-to-right order of the Fortran line it cites.
//
// baroclinic_dynamics runs as two kernels:
//  1. k_columns: every interior water column and velocity component is one
//     thread, which builds the tridiagonal system level by level, runs
//     factor8's forward elimination as it goes (x, y of the sweep kept in
//     the output arrays), then back-substitutes from the bottom and applies
//     the Robert-Asselin filter to the new velocity at once, writing uu/uup
//     (vv/vvp) to the output arrays.  The inputs stay untouched, so the
//     neighbouring columns' Coriolis and advection reads see the old state.
//     Every level's rows are staged in shared memory by bulk asynchronous
//     copies (a copy warp runs ahead of the compute warps through a ring of
//     mbarrier slots).
//  2. k_border, over every point of the arrays outside the interior: the
//     filter on the one-point ring with the new velocity the periodic wrap
//     brings there (zero without a wrap, as the reference's un = 0), a copy
//     elsewhere.
//
// tracer_tran_diff runs the same way in three kernels: k_tracer_flux (the
// lateral fluxes on the u and v points), the periodic wraps of those
// fluxes, k_tracer_solve (the vertical diffusion system of every T column
// with the filter) and k_tracer_border.  vertical_velocity, depth_ave and
// the barotropic shift are one thread per column or point.
#include "column.h"

namespace inmsom {
namespace column {

namespace {

constexpr int MAX_NZ = 200;     // levels (dz, hzt in shared memory)
constexpr int BX = 32, BY = 8;

#define X(m_, n_) ix(D, (m_), (n_))

// ---- Function/vel_ssh.f90:847-983: one water column's system --------------
// V = false: the u block (:852-915), true: the v block (:917-979).

// what the column's equations take from 2-D fields, in the Fortran order of
// their products
struct ColConst {
    double f1, f2;            // u: dxt, dyh; v: dxh, dyt
    double hn, bp, bp0, hc, pg, tsurf, tbot;
    double dx0, dy0, dx1, dy1, cor0, cor1, drag;
};

// the values of level k the equations read (nu, ww, s1 at level k + 1)
struct LevelIn {
    double sp, r1, r2, oe, o0, ope, op, nu0, nu1, w0, w1, s1;
};

// the far end of the velocity point (u: m+1, v: n+1) and the partner of the
// Coriolis average (u: n-1, v: m-1), as offsets in a pitched level
template <bool V>
__device__ __forceinline__ long long far_off(const Dom &D) { return V ? D.pitch : 1; }
template <bool V>
__device__ __forceinline__ long long partner_off(const Dom &D) { return V ? -1 : -D.pitch; }

template <bool V>
__device__ __forceinline__ ColConst col_const(const Dom &D, const GridDev &g, const BaroclinicArgs &a, long long i)
{
    const long long e = far_off<V>(D), p = partner_off<V>(D);
    ColConst c;
    c.f1 = V ? g.dxh[i] : g.dxt[i];
    c.f2 = V ? g.dyt[i] : g.dyh[i];
    c.hn = (V ? a.hhvn : a.hhun)[i];
    c.bp = c.hn * c.f1 * c.f2 / a.tau / 2.0;
    c.bp0 = (V ? a.hhvp : a.hhup)[i] * c.f1 * c.f2 / a.tau / 2.0;
    c.hc = (V ? a.hhv : a.hhu)[i];
    c.pg = (V ? a.pgry : a.pgrx)[i];
    c.tsurf = (V ? a.ty_surf : a.tx_surf)[i];
    c.tbot = (V ? a.ty_bot : a.tx_bot)[i];
    c.dx0 = g.dx[i];
    c.dy0 = g.dy[i];
    c.dx1 = g.dx[i + e];
    c.dy1 = g.dy[i + e];
    c.cor0 = g.rlh[i] * a.hhh[i] * g.dxb[i] * g.dyb[i];
    c.cor1 = g.rlh[i + p] * a.hhh[i + p] * g.dxb[i + p] * g.dyb[i + p];
    c.drag = (a.rdis[i] + a.rdis[i + e]) / 2.0;
    return c;
}

// Level k (1-based) of the column: its row of the tridiagonal system
// (:862-911 surface, internal and bottom points) and factor8's forward step
// (Service/oc_algorithms.f90:510-516).  dp, fz_p carry the level above,
// xm, ym the sweep, s0 the velocity at level k.
template <bool V>
__device__ __forceinline__ void level_step(const ColConst &c, const LevelIn &v, int k, int nz, double dzk,
                                           double hztk1, double &dp, double &fz_p, double &xm, double &ym,
                                           double &s0)
{
    const double dm = dp, fz_m = fz_p;
    if (k < nz) {
        dp = (v.nu0 + v.nu1) / 2.0 / c.hn / hztk1 * c.f1 * c.f2;
        fz_p = (v.w0 * c.dx0 * c.dy0 + v.w1 * c.dx1 * c.dy1) / 2.0 * (s0 + v.s1) / 2.0;
    } else {
        dp = 0.0;
        fz_p = 0.0;
    }
    const double cor = (c.cor0 * (v.oe + v.o0) + c.cor1 * (v.ope + v.op)) / 4.0;
    double eta = c.bp0 * v.sp + v.r1 + v.r2 + c.pg - (fz_p - fz_m) / dzk;
    eta = V ? eta - cor : eta + cor;
    eta = eta - c.drag * v.sp * c.f1 * c.f2 * c.hc;
    if (k == 1) eta = eta + c.tsurf / dzk * c.f1 * c.f2;
    if (k == nz) eta = eta + c.tbot / dzk * c.f1 * c.f2;
    const double cc = k < nz ? -dp / dzk : 0.0;
    const double bb = k == 1 ? c.bp + dp / dzk : (k < nz ? c.bp + (dp + dm) / dzk : c.bp + dm / dzk);
    if (k == 1) {
        xm = -cc / bb;
        ym = eta / bb;
    } else {
        const double aa = -dm / dzk;
        const double scr = 1.0 / (aa * xm + bb);
        ym = (eta - aa * ym) * scr;
        xm = -cc * scr;
    }
    s0 = v.s1;
}

// factor8's back substitution (Service/oc_algorithms.f90:517-520) from the
// bottom, with the filter of Function/vel_ssh.f90:1002-1024 at this point:
// uup = uu + ts*(un - 2 uu + uup)/2, uu = un.  The sweep's x(k), y(k) are
// in outp, out at level k, written by this thread in the forward sweep and
// overwritten here with the filtered values (the next level up loaded one
// iteration ahead; no other thread touches these addresses, and the lines
// are still in L2); r starts as y(nz).
__device__ __forceinline__ void back_filter_inplace(int nz, long long P, long long i, double r, double ts,
                                                    const double *self, const double *selfp, double *out,
                                                    double *outp)
{
    long long o = (long long)(nz - 1) * P + i;
    double cu = self[o], cp = selfp[o], xk = 0.0, yk = 0.0;
    for (int k = nz; k >= 1; k--) {
        double cu1 = 0.0, cp1 = 0.0, x1 = 0.0, y1 = 0.0;
        if (k > 1) {
            cu1 = self[o - P];
            cp1 = selfp[o - P];
            x1 = outp[o - P];
            y1 = out[o - P];
        }
        if (k < nz) r = xk * r + yk;
        outp[o] = cu + ts * (r - 2.0 * cu + cp) / 2.0;
        out[o] = r;
        cu = cu1;
        cp = cp1;
        xk = x1;
        yk = y1;
        o -= P;
    }
}

// ---- the column solve ------------------------------------------------------
// A CTA owns CW consecutive columns of one row n for both components: warps
// 0-1 the u columns, warps 2-3 the v columns, warp 4 the copies.  For every
// level j the copy warp brings the fourteen row segments the level's
// equations read (CW + 4 columns each, 16-byte aligned) into a ring slot
// with 1-D bulk asynchronous copies completing on the slot's mbarrier; the
// compute warps read the slot of level k and of level k + 1, then release
// slot k.  The sweep's x, y go to the output arrays, and the back
// substitution re-reads them with uu/uup (vv/vvp) from global memory (L2),
// so shared memory holds only the ring: four CTAs per SM (registers).

constexpr int CW = 64;                   // columns per CTA
constexpr int NCW = 4;                   // compute warps
constexpr int NS = 4;                    // ring slots (levels)
constexpr int NROW = 14;                 // row segments per level
constexpr int RW = CW + 4;               // doubles per staged segment
constexpr int SLOT_D = NROW * RW;        // doubles per slot
constexpr unsigned WAIT_LIMIT = 1u << 20;

// the row segments of a slot: field (level j), row
enum { R_UU0, R_UU1, R_VVM, R_VV0, R_UUP, R_VVP, R_RX, R_RY, R_RXT, R_RYT, R_NU0, R_NU1, R_WW0, R_WW1 };

size_t staged_smem(int nz)
{
    return ((size_t)NS * SLOT_D + 2 * (size_t)nz + 1) * sizeof(double) + 2 * NS * sizeof(uint64_t);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    for (unsigned t = 0; t < WAIT_LIMIT; t++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

template <bool V>
__device__ __forceinline__ LevelIn staged_level(const double *st, const double *sn, int cs, bool last)
{
    LevelIn v;
    if (!V) {
        v.sp = st[R_UUP * RW + cs];
        v.r1 = st[R_RX * RW + cs];
        v.r2 = st[R_RXT * RW + cs];
        v.oe = st[R_VV0 * RW + cs + 1];                   // vv(m+1, n)
        v.o0 = st[R_VV0 * RW + cs];                       // vv(m, n)
        v.ope = st[R_VVM * RW + cs + 1];                  // vv(m+1, n-1)
        v.op = st[R_VVM * RW + cs];                       // vv(m, n-1)
    } else {
        v.sp = st[R_VVP * RW + cs];
        v.r1 = st[R_RY * RW + cs];
        v.r2 = st[R_RYT * RW + cs];
        v.oe = st[R_UU1 * RW + cs];                       // uu(m, n+1)
        v.o0 = st[R_UU0 * RW + cs];                       // uu(m, n)
        v.ope = st[R_UU1 * RW + cs - 1];                  // uu(m-1, n+1)
        v.op = st[R_UU0 * RW + cs - 1];                   // uu(m-1, n)
    }
    if (!last) {
        v.nu0 = sn[R_NU0 * RW + cs];
        v.nu1 = V ? sn[R_NU1 * RW + cs] : sn[R_NU0 * RW + cs + 1];
        v.w0 = sn[R_WW0 * RW + cs];
        v.w1 = V ? sn[R_WW1 * RW + cs] : sn[R_WW0 * RW + cs + 1];
        v.s1 = V ? sn[R_VV0 * RW + cs] : sn[R_UU0 * RW + cs];
    } else {
        v.nu0 = v.nu1 = v.w0 = v.w1 = v.s1 = 0.0;
    }
    return v;
}

template <bool V>
__device__ __forceinline__ bool staged_column(const Dom &D, const GridDev &g, const Levels &L,
                                              const BaroclinicArgs &a, double ts, int m, int n, int cs,
                                              const double *ring, const double *sdz, uint64_t *full,
                                              uint64_t *empty, int lane)
{
    const int nz = L.nz;
    const long long P = L.plane;
    const bool act = m <= D.nx_end;
    const long long i = act ? X(m, n) : 0;
    const bool ocean = act && (V ? g.lcv[i] : g.lcu[i]) > 0.5f;
    const double *self = V ? a.vv : a.uu, *selfp = V ? a.vvp : a.uup;
    double *out = V ? a.vv_out : a.uu_out, *outp = V ? a.vvp_out : a.uup_out;
    ColConst c{};
    if (ocean) c = col_const<V>(D, g, a, i);
    double dp = 0.0, fz_p = 0.0, xm = 0.0, ym = 0.0, s0 = 0.0;
    bool ok = true;
    for (int k = 1; k <= nz && ok; k++) {
        const int sk = (k - 1) % NS, sn = k % NS;
        ok = mbar_wait(&full[sk], (uint32_t)(((k - 1) / NS) & 1));
        if (ok && k < nz) ok = mbar_wait(&full[sn], (uint32_t)((k / NS) & 1));
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        const double *st = ring + (size_t)sk * SLOT_D, *snx = ring + (size_t)sn * SLOT_D;
        const int rself = V ? R_VV0 : R_UU0, rselfp = V ? R_VVP : R_UUP;
        if (ocean) {
            if (k == 1) s0 = st[rself * RW + cs];
            const LevelIn v = staged_level<V>(st, snx, cs, k == nz);
            level_step<V>(c, v, k, nz, sdz[k - 1], k < nz ? sdz[nz + k] : 1.0, dp, fz_p, xm, ym, s0);
            const long long o = (long long)(k - 1) * P + i;
            outp[o] = xm;
            out[o] = ym;
        } else if (act) {
            const long long o = (long long)(k - 1) * P + i;
            out[o] = st[rself * RW + cs];
            outp[o] = st[rselfp * RW + cs];
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[sk]);
    }
    if (ok && ocean) back_filter_inplace(nz, P, i, ym, ts, self, selfp, out, outp);
    return ok;
}

__global__ void __launch_bounds__((NCW + 1) * 32, 4) k_columns(Dom D, GridDev g, Levels L, BaroclinicArgs a, double ts,
                                                               int row0)
{
    extern __shared__ __align__(128) double sm[];
    const int nz = L.nz;
    double *ring = sm;
    double *sdz = ring + (size_t)NS * SLOT_D;             // dz (nz), hzt (nz + 1)
    uint64_t *full = reinterpret_cast<uint64_t *>(sdz + 2 * nz + 1);
    uint64_t *empty = full + NS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = D.nx_start + blockIdx.x * CW, n = row0 + blockIdx.y;

    for (int t = threadIdx.x; t < 2 * nz + 1; t += blockDim.x) sdz[t] = L.dz[t];
    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&full[s])), "r"(1) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[s])), "r"(NCW)
                         : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // the staged segments: device columns c0 .. c0 + cnt - 1, c0 even, from
    // m0 - 1 (or m0 - 2) to at least the last column + 1
    const int cm0 = m0 - D.bnd_x1 + D.xoff;
    const int mlast = min(m0 + CW - 1, D.nx_end);
    const int c0 = (cm0 - 1) & ~1;
    const int cnt = ((mlast - D.bnd_x1 + D.xoff + 2 - c0) + 1) & ~1;

    if (warp == NCW) {
        if (lane != 0) return;
        const long long P = L.plane;
        const long long rb = (long long)(n - D.bnd_y1) * D.pitch + c0;   // row n, column c0
        const long long pt = D.pitch;
        const uint32_t seg = (uint32_t)cnt * 8u;
        int armed = 0;
        bool ok = true;
        for (int j = 1; j <= nz; j++) {
            const int s = (j - 1) % NS;
            if (j > NS && !mbar_wait(&empty[s], (uint32_t)(((j - 1) / NS - 1) & 1))) {
                ok = false;
                break;
            }
            double *slot = ring + (size_t)s * SLOT_D;
            const long long lv = (long long)(j - 1) * P + rb;
            const int nrow = j == 1 ? R_NU0 : NROW;       // nu, ww of level 1 are not read
            mbar_expect(&full[s], seg * (uint32_t)nrow);
            bulk_copy(slot + R_UU0 * RW, a.uu + lv, seg, &full[s]);
            bulk_copy(slot + R_UU1 * RW, a.uu + lv + pt, seg, &full[s]);
            bulk_copy(slot + R_VVM * RW, a.vv + lv - pt, seg, &full[s]);
            bulk_copy(slot + R_VV0 * RW, a.vv + lv, seg, &full[s]);
            bulk_copy(slot + R_UUP * RW, a.uup + lv, seg, &full[s]);
            bulk_copy(slot + R_VVP * RW, a.vvp + lv, seg, &full[s]);
            bulk_copy(slot + R_RX * RW, a.rhsx + lv, seg, &full[s]);
            bulk_copy(slot + R_RY * RW, a.rhsy + lv, seg, &full[s]);
            bulk_copy(slot + R_RXT * RW, a.rhsx_tran + lv, seg, &full[s]);
            bulk_copy(slot + R_RYT * RW, a.rhsy_tran + lv, seg, &full[s]);
            if (j > 1) {
                bulk_copy(slot + R_NU0 * RW, a.nu + lv, seg, &full[s]);
                bulk_copy(slot + R_NU1 * RW, a.nu + lv + pt, seg, &full[s]);
                bulk_copy(slot + R_WW0 * RW, a.ww + lv, seg, &full[s]);
                bulk_copy(slot + R_WW1 * RW, a.ww + lv + pt, seg, &full[s]);
            }
            armed = j;
        }
        if (!ok) atomicOr(a.flag, 1);
        // no copy of this CTA may be in flight when it exits
        for (int j = max(1, armed - NS + 1); j <= armed; j++)
            (void)mbar_wait(&full[(j - 1) % NS], (uint32_t)(((j - 1) / NS) & 1));
        return;
    }
    const bool V = warp >= 2;
    const int col = (warp & 1) * 32 + lane;
    const int m = m0 + col;
    const int cs = (m - D.bnd_x1 + D.xoff) - c0;
    const bool ok = V ? staged_column<true>(D, g, L, a, ts, m, n, cs, ring, sdz, full, empty, lane)
                      : staged_column<false>(D, g, L, a, ts, m, n, cs, ring, sdz, full, empty, lane);
    if (!ok && lane == 0) atomicOr(a.flag, 1);
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

// ---- Function/tem_sal.f90: one tracer's step ---------------------------

// :108-251 at the u (V = false) and v (V = true) points of the interior:
// the lateral advective, diffusive and GM fluxes of every level, the
// vertical parts and coefficients of the isoneutral flux (levels 2..nz;
// levels 1 and nz + 1 are zero), and the depth-integrated diagnostics.
// Staged like k_columns: warps 0-1 the u points of CW columns of row n,
// warps 2-3 the v points, warp 4 copies the twelve row segments of each
// level (ffp, mu, ff on rows n and n+1; uu, vv and the four slopes on row n;
// no slopes for level 1) into a 4-slot mbarrier ring.
constexpr int FNROW = 12;
constexpr int FSLOT_D = FNROW * RW;
constexpr int FNS = 4;                   // ring slots (levels) of the flux kernel
constexpr int FLUX_CTAS = 6;             // resident CTAs per SM its registers are cut for
enum { G_FFP0, G_FFP1, G_MU0, G_MU1, G_FF0, G_FF1, G_UU, G_VV, G_SLRX, G_SLZX, G_SLRY, G_SLZY };

size_t flux_smem(int nz)
{
    return ((size_t)FNS * FSLOT_D + 2 * (size_t)nz + 1) * sizeof(double) + 2 * FNS * sizeof(uint64_t);
}

template <bool V>
__device__ __forceinline__ bool tracer_flux_column(const Dom &D, const GridDev &g, const Levels &L,
                                                   const TracerArgs &a, int m, int n, int cs, const double *ring,
                                                   const double *sdz, uint64_t *full, uint64_t *empty, int lane)
{
    const int nz = L.nz;
    const long long P = L.plane;
    const bool act = m <= D.nx_end;
    const long long i = act ? X(m, n) : 0;
    const bool wet = act && (V ? g.lcv[i] : g.lcu[i]) > 0.5f;
    double *flux = V ? a.flux_y : a.flux_x, *fz = V ? a.flux_zy : a.flux_zx;
    double *coef = V ? a.coef_zy : a.coef_zx, *sfgm = V ? a.sfgm_zy : a.sfgm_zx;
    double *ffo = V ? a.flux_f_y : a.flux_f_x;
    // the far point (u: m+1 on row n, v: m on row n+1) in the staged rows
    const int rf_ffp = V ? G_FFP1 : G_FFP0, rf_mu = V ? G_MU1 : G_MU0, rf_ff = V ? G_FF1 : G_FF0;
    const int cf = V ? cs : cs + 1;
    const int r_slr = V ? G_SLRY : G_SLRX, r_slz = V ? G_SLZY : G_SLZX, r_vel = V ? G_VV : G_UU;
    double hh = 0.0, dside = 0.0, dnorm = 0.0;
    if (wet) {
        hh = (V ? a.hhv : a.hhu)[i];
        dside = V ? g.dxh[i] : g.dyh[i];
        dnorm = V ? g.dyt[i] : g.dxt[i];
    }
    if (act) {
        fz[i] = 0.0;
        coef[i] = 0.0;
        sfgm[i] = 0.0;
    }
    double f1d = 0.0, sg = 0.0;
    double acc1 = 0.0, acc2 = 0.0, acc3 = 0.0, acc4 = 0.0;
    bool ok = true;
    for (int k = 1; k <= nz && ok; k++) {
        const int sk = (k - 1) % FNS, sn = k % FNS;
        ok = mbar_wait(&full[sk], (uint32_t)(((k - 1) / FNS) & 1));
        if (ok && k < nz) ok = mbar_wait(&full[sn], (uint32_t)((k / FNS) & 1));
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        const double *st = ring + (size_t)sk * FSLOT_D, *nx = ring + (size_t)sn * FSLOT_D;
        const long long o = (long long)(k - 1) * P + i;
        if (wet) {
            double f1d1 = 0.0, sg1 = 0.0;
            if (k < nz) {
                const long long o1 = o + P;
                const double dfdz = (nx[G_FFP0 * RW + cs] - st[G_FFP0 * RW + cs] + nx[rf_ffp * RW + cf] -
                                     st[rf_ffp * RW + cf]) / 2.0;
                const double dfdh = (nx[rf_ffp * RW + cf] - nx[G_FFP0 * RW + cs] + st[rf_ffp * RW + cf] -
                                     st[G_FFP0 * RW + cs]) / 2.0;
                const double mu1 = (nx[G_MU0 * RW + cs] + st[G_MU0 * RW + cs] + nx[rf_mu * RW + cf] +
                                    st[rf_mu * RW + cf]) / 4.0 * a.factor_mu * dside / dnorm;
                const double slr = nx[r_slr * RW + cs], slz = nx[r_slz * RW + cs];
                const double slope = a.ar * slr + a.az * slz;
                f1d1 = mu1 * (hh * dfdh * sdz[nz + k] - slope * dfdz);
                fz[o1] = mu1 * slope * dfdh;
                coef[o1] = mu1 * (slope * slope) / hh / sdz[nz + k];
                sg1 = mu1 * (slr - slz) * a.alpha_gm;
                sfgm[o1] = sg1;
            }
            const double dzk = sdz[k - 1];
            double fd;
            if (k == 1) fd = f1d1 / sdz[nz + 1];
            else if (k < nz) fd = (f1d + f1d1) / dzk / 2.0;
            else fd = f1d / sdz[nz + k - 1];
            const double s2 = st[G_FF0 * RW + cs] + st[rf_ff * RW + cf];
            const double fa = -(st[r_vel * RW + cs] * hh * dside * s2 / 2.0);
            const double vg = (sg1 - sg) / dzk;
            const double fg = -(vg * s2 / 2.0);
            flux[o] = fa + fd + fg;
            acc1 = acc1 + dzk * (fa + fd + fg);
            acc2 = acc2 + dzk * fa;
            acc3 = acc3 + dzk * fd;
            acc4 = acc4 + dzk * fg;
            f1d = f1d1;
            sg = sg1;
        } else if (act) {
            flux[o] = 0.0;
            if (k < nz) {
                fz[o + P] = 0.0;
                coef[o + P] = 0.0;
                sfgm[o + P] = 0.0;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[sk]);
    }
    if (ok && act) {
        const long long ot = (long long)nz * P + i;        // level nz + 1
        fz[ot] = 0.0;
        coef[ot] = 0.0;
        sfgm[ot] = 0.0;
        ffo[i] = acc1;
        ffo[P + i] = acc2;
        ffo[2 * P + i] = acc3;
        ffo[3 * P + i] = acc4;
    }
    return ok;
}

__global__ void __launch_bounds__((NCW + 1) * 32, FLUX_CTAS) k_tracer_flux(Dom D, GridDev g, Levels L, TracerArgs a, int row0)
{
    extern __shared__ __align__(128) double sm[];
    const int nz = L.nz;
    double *ring = sm;
    double *sdz = ring + (size_t)FNS * FSLOT_D;            // dz (nz), hzt (nz + 1)
    uint64_t *full = reinterpret_cast<uint64_t *>(sdz + 2 * nz + 1);
    uint64_t *empty = full + FNS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = D.nx_start + blockIdx.x * CW, n = row0 + blockIdx.y;
    for (int t = threadIdx.x; t < 2 * nz + 1; t += blockDim.x) sdz[t] = L.dz[t];
    if (threadIdx.x == 0) {
        for (int s = 0; s < FNS; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&full[s])), "r"(1) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[s])), "r"(NCW)
                         : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int cm0 = m0 - D.bnd_x1 + D.xoff;
    const int mlast = min(m0 + CW - 1, D.nx_end);
    const int c0 = (cm0 - 1) & ~1;
    const int cnt = ((mlast - D.bnd_x1 + D.xoff + 2 - c0) + 1) & ~1;
    if (warp == NCW) {
        if (lane != 0) return;
        const long long P = L.plane;
        const long long rb = (long long)(n - D.bnd_y1) * D.pitch + c0, pt = D.pitch;
        const uint32_t seg = (uint32_t)cnt * 8u;
        int armed = 0;
        bool ok = true;
        for (int j = 1; j <= nz; j++) {
            const int s = (j - 1) % FNS;
            if (j > FNS && !mbar_wait(&empty[s], (uint32_t)(((j - 1) / FNS - 1) & 1))) {
                ok = false;
                break;
            }
            double *slot = ring + (size_t)s * FSLOT_D;
            const long long lv = (long long)(j - 1) * P + rb;
            mbar_expect(&full[s], seg * (uint32_t)(j == 1 ? G_SLRX : FNROW));
            bulk_copy(slot + G_FFP0 * RW, a.ffp + lv, seg, &full[s]);
            bulk_copy(slot + G_FFP1 * RW, a.ffp + lv + pt, seg, &full[s]);
            bulk_copy(slot + G_MU0 * RW, a.mu + lv, seg, &full[s]);
            bulk_copy(slot + G_MU1 * RW, a.mu + lv + pt, seg, &full[s]);
            bulk_copy(slot + G_FF0 * RW, a.ff + lv, seg, &full[s]);
            bulk_copy(slot + G_FF1 * RW, a.ff + lv + pt, seg, &full[s]);
            bulk_copy(slot + G_UU * RW, a.uu + lv, seg, &full[s]);
            bulk_copy(slot + G_VV * RW, a.vv + lv, seg, &full[s]);
            if (j > 1) {
                bulk_copy(slot + G_SLRX * RW, a.slrx + lv, seg, &full[s]);
                bulk_copy(slot + G_SLZX * RW, a.slzx + lv, seg, &full[s]);
                bulk_copy(slot + G_SLRY * RW, a.slry + lv, seg, &full[s]);
                bulk_copy(slot + G_SLZY * RW, a.slzy + lv, seg, &full[s]);
            }
            armed = j;
        }
        if (!ok) atomicOr(a.flag, 1);
        for (int j = max(1, armed - FNS + 1); j <= armed; j++)
            (void)mbar_wait(&full[(j - 1) % FNS], (uint32_t)(((j - 1) / FNS) & 1));
        return;
    }
    const bool V = warp >= 2;
    const int m = m0 + (warp & 1) * 32 + lane;
    const int cs = (m - D.bnd_x1 + D.xoff) - c0;
    const bool ok = V ? tracer_flux_column<true>(D, g, L, a, m, n, cs, ring, sdz, full, empty, lane)
                      : tracer_flux_column<false>(D, g, L, a, m, n, cs, ring, sdz, full, empty, lane);
    if (!ok && lane == 0) atomicOr(a.flag, 1);
}

// :277-392 at the T points of the interior (the vertical diffusion system,
// factor8), then the filter of :405-419 there.  Staged like k_columns: a CTA
// owns CW columns of row n (warps 0-1) and a copy warp (2) brings, for
// every level j, the nineteen row segments the equations of levels j - 1
// and j read into a 3-slot mbarrier ring; stage nz + 1 holds nu only.  The
// sweep's x, y go to ffp_out, ff_out (back_filter_inplace).
constexpr int TNS = 3;                    // ring slots of the tracer solve
constexpr int TNROW = 19;
constexpr int TSLOT_D = TNROW * RW;
enum {
    Q_FF, Q_FFPM, Q_FFP0, Q_FFPP, Q_FLX, Q_FLY0, Q_FLYM, Q_SRC, Q_NU,          // levels 1..nz (nu: 1..nz+1)
    Q_WW, Q_FZX, Q_FZY0, Q_FZYM, Q_COX, Q_COY0, Q_COYM, Q_SGX, Q_SGY0, Q_SGYM  // levels 2..nz
};

size_t tracer_smem(int nz)
{
    return ((size_t)TNS * TSLOT_D + 2 * (size_t)nz + 1) * sizeof(double) + 2 * TNS * sizeof(uint64_t);
}

__global__ void __launch_bounds__(3 * 32) k_tracer_solve(Dom D, GridDev g, Levels L, TracerArgs a, double ts, int row0)
{
    extern __shared__ __align__(128) double sm[];
    const int nz = L.nz;
    double *ring = sm;
    double *sdz = ring + (size_t)TNS * TSLOT_D;           // dz (nz), hzt (nz + 1)
    uint64_t *full = reinterpret_cast<uint64_t *>(sdz + 2 * nz + 1);
    uint64_t *empty = full + TNS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = D.nx_start + blockIdx.x * CW, n = row0 + blockIdx.y;
    for (int t = threadIdx.x; t < 2 * nz + 1; t += blockDim.x) sdz[t] = L.dz[t];
    if (threadIdx.x == 0) {
        for (int s = 0; s < TNS; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&full[s])), "r"(1) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[s])), "r"(2) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int cm0 = m0 - D.bnd_x1 + D.xoff;
    const int mlast = min(m0 + CW - 1, D.nx_end);
    const int c0 = (cm0 - 1) & ~1;
    const int cnt = ((mlast - D.bnd_x1 + D.xoff + 2 - c0) + 1) & ~1;
    const long long P = L.plane;

    if (warp == 2) {
        if (lane != 0) return;
        const long long rb = (long long)(n - D.bnd_y1) * D.pitch + c0, pt = D.pitch;
        const uint32_t seg = (uint32_t)cnt * 8u;
        int armed = 0;
        bool ok = true;
        for (int j = 1; j <= nz + 1; j++) {
            const int s = (j - 1) % TNS;
            if (j > TNS && !mbar_wait(&empty[s], (uint32_t)(((j - 1) / TNS - 1) & 1))) {
                ok = false;
                break;
            }
            double *slot = ring + (size_t)s * TSLOT_D;
            const long long lv = (long long)(j - 1) * P + rb;
            const int nrow = j == nz + 1 ? 1 : (j == 1 ? Q_NU + 1 : TNROW);
            mbar_expect(&full[s], seg * (uint32_t)nrow);
            bulk_copy(slot + Q_NU * RW, a.nu + lv, seg, &full[s]);
            if (j <= nz) {
                bulk_copy(slot + Q_FF * RW, a.ff + lv, seg, &full[s]);
                bulk_copy(slot + Q_FFPM * RW, a.ffp + lv - pt, seg, &full[s]);
                bulk_copy(slot + Q_FFP0 * RW, a.ffp + lv, seg, &full[s]);
                bulk_copy(slot + Q_FFPP * RW, a.ffp + lv + pt, seg, &full[s]);
                bulk_copy(slot + Q_FLX * RW, a.flux_x + lv, seg, &full[s]);
                bulk_copy(slot + Q_FLY0 * RW, a.flux_y + lv, seg, &full[s]);
                bulk_copy(slot + Q_FLYM * RW, a.flux_y + lv - pt, seg, &full[s]);
                bulk_copy(slot + Q_SRC * RW, a.src + lv, seg, &full[s]);
            }
            if (j > 1 && j <= nz) {
                bulk_copy(slot + Q_WW * RW, a.ww + lv, seg, &full[s]);
                bulk_copy(slot + Q_FZX * RW, a.flux_zx + lv, seg, &full[s]);
                bulk_copy(slot + Q_FZY0 * RW, a.flux_zy + lv, seg, &full[s]);
                bulk_copy(slot + Q_FZYM * RW, a.flux_zy + lv - pt, seg, &full[s]);
                bulk_copy(slot + Q_COX * RW, a.coef_zx + lv, seg, &full[s]);
                bulk_copy(slot + Q_COY0 * RW, a.coef_zy + lv, seg, &full[s]);
                bulk_copy(slot + Q_COYM * RW, a.coef_zy + lv - pt, seg, &full[s]);
                bulk_copy(slot + Q_SGX * RW, a.sfgm_zx + lv, seg, &full[s]);
                bulk_copy(slot + Q_SGY0 * RW, a.sfgm_zy + lv, seg, &full[s]);
                bulk_copy(slot + Q_SGYM * RW, a.sfgm_zy + lv - pt, seg, &full[s]);
            }
            armed = j;
        }
        if (!ok) atomicOr(a.flag, 1);
        for (int j = max(1, armed - TNS + 1); j <= armed; j++)
            (void)mbar_wait(&full[(j - 1) % TNS], (uint32_t)(((j - 1) / TNS) & 1));
        return;
    }

    const int m = m0 + warp * 32 + lane;
    const bool act = m <= D.nx_end;
    const long long i = act ? X(m, n) : 0;
    const bool ocean = act && g.lu[i] > 0.5f;
    const int cs = (m - D.bnd_x1 + D.xoff) - c0;
    double dx = 0.0, dy = 0.0, hn = 0.0, bp = 0.0, bp0 = 0.0, cu = 0.0, cv = 0.0, hq = 0.0, swb = 0.0;
    double ftop = 0.0, fbot = 0.0;
    int igt = 0, igb = 0;
    if (ocean) {
        dx = g.dx[i];
        dy = g.dy[i];
        hn = a.hhqn[i];
        bp = hn * dx * dy / a.tau / 2.0;
        bp0 = a.hhqp[i] * dx * dy / a.tau / 2.0;
        cu = (double)fmaxf(g.lcu[i] + g.lcu[i - 1], 1e-10f);
        cv = (double)fmaxf(g.lcv[i] + g.lcv[i - D.pitch], 1e-10f);
        hq = g.hrest[i];
        swb = a.swbal[i];
        ftop = a.ff_top[i];
        fbot = a.ff_bot[i];
        igt = a.ig_top[i];
        igb = a.ig_bot[i];
    }
    double fz_p = 0.0, dp = 0.0, xm = 0.0, ym = 0.0;
    bool ok = true;
    for (int k = 1; k <= nz && ok; k++) {
        const int sk = (k - 1) % TNS, sn = k % TNS;
        ok = mbar_wait(&full[sk], (uint32_t)(((k - 1) / TNS) & 1)) && mbar_wait(&full[sn], (uint32_t)((k / TNS) & 1));
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        const double *st = ring + (size_t)sk * TSLOT_D, *nx = ring + (size_t)sn * TSLOT_D;
        const int q = k - 1;
        const long long o = (long long)q * P + i;
        if (ocean) {
            const double dzk = sdz[q];
            const double fz_m = fz_p;
            if (k < nz) {
                const double vel_gm = -(nx[Q_SGX * RW + cs] - nx[Q_SGX * RW + cs - 1] + nx[Q_SGY0 * RW + cs] -
                                        nx[Q_SGYM * RW + cs]);
                fz_p = -((nx[Q_FZX * RW + cs] + nx[Q_FZX * RW + cs - 1]) / cu) -
                       (nx[Q_FZY0 * RW + cs] + nx[Q_FZYM * RW + cs]) / cv +
                       (nx[Q_COX * RW + cs] * (nx[Q_FFP0 * RW + cs + 1] - st[Q_FFP0 * RW + cs + 1]) +
                        nx[Q_COX * RW + cs - 1] * (nx[Q_FFP0 * RW + cs - 1] - st[Q_FFP0 * RW + cs - 1])) /
                           cu / 2.0 +
                       (nx[Q_COY0 * RW + cs] * (nx[Q_FFPP * RW + cs] - st[Q_FFPP * RW + cs]) +
                        nx[Q_COYM * RW + cs] * (nx[Q_FFPM * RW + cs] - st[Q_FFPM * RW + cs])) /
                           cv / 2.0 -
                       (nx[Q_WW * RW + cs] * dx * dy + vel_gm) * (st[Q_FF * RW + cs] + nx[Q_FF * RW + cs]) / 2.0;
            } else {
                fz_p = 0.0;
            }
            const double nu_p = nx[Q_NU * RW + cs] * a.factor_nu;
            const double dm = k == 1 ? st[Q_NU * RW + cs] * a.factor_nu * dx * dy / hn / sdz[nz] : dp;
            if (k < nz)
                dp = (nx[Q_COX * RW + cs] + nx[Q_COX * RW + cs - 1]) / cu / 2.0 +
                     (nx[Q_COY0 * RW + cs] + nx[Q_COYM * RW + cs]) / cv / 2.0 + nu_p * dx * dy / hn / sdz[nz + k];
            else
                dp = nu_p * dx * dy / hn / sdz[nz + k];
            const double rhs = st[Q_FLX * RW + cs] - st[Q_FLX * RW + cs - 1] + st[Q_FLY0 * RW + cs] -
                               st[Q_FLYM * RW + cs] + (fz_p - fz_m) / dzk +
                               st[Q_SRC * RW + cs] * hq * swb * a.src_factor * dx * dy;
            const double base = st[Q_FFP0 * RW + cs];
            double cc, aa = 0.0, bb, eta;
            if (k == 1) {
                cc = -dp / dzk;
                if (igt == 1) {
                    bb = bp + (dp + dm) / dzk;
                    eta = bp0 * base + rhs + dm * ftop / dzk;
                } else {
                    bb = bp + dp / dzk;
                    eta = bp0 * base + rhs + ftop / dzk * dx * dy;
                }
            } else if (k < nz) {
                cc = -dp / dzk;
                aa = -dm / dzk;
                bb = bp + (dp + dm) / dzk;
                eta = bp0 * base + rhs;
            } else {
                cc = 0.0;
                aa = -dm / dzk;
                if (igb == 1) {
                    bb = bp + (dp + dm) / dzk;
                    eta = bp0 * base + rhs + dp * fbot / dzk;
                } else {
                    bb = bp + dm / dzk;
                    eta = bp0 * base + rhs + fbot / dzk * dx * dy;
                }
            }
            if (k == 1) {
                xm = -cc / bb;
                ym = eta / bb;
            } else {
                const double scr = 1.0 / (aa * xm + bb);
                ym = (eta - aa * ym) * scr;
                xm = -cc * scr;
            }
            a.ffp_out[o] = xm;
            a.ff_out[o] = ym;
        } else if (act) {
            a.ff_out[o] = st[Q_FF * RW + cs];
            a.ffp_out[o] = st[Q_FFP0 * RW + cs];
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[sk]);
    }
    if (!ok) {
        if (lane == 0) atomicOr(a.flag, 1);
        return;
    }
    // the copy warp's last stage (nz + 1, slot nz % TNS) was waited on above
    if (ocean) back_filter_inplace(nz, P, i, ym, ts, a.ff, a.ffp, a.ff_out, a.ffp_out);
}

// :405-419 outside the interior (the ring with the wrapped new tracer,
// copies elsewhere), one level per grid row
__global__ void k_tracer_border(Dom D, GridDev g, Levels L, TracerArgs a, double ts, int count)
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
    const long long lev = (long long)blockIdx.y * L.plane, o = lev + i;
    if (ring && g.lu[i] > 0.5f) {
        const double fnew = new_at(D, g.lu, a.ff_out, lev, m, n), cf = a.ff[o];
        a.ffp_out[o] = cf + ts * (fnew - 2.0 * cf + a.ffp[o]) / 2.0;
        a.ff_out[o] = fnew;
    } else {
        a.ff_out[o] = a.ff[o];
        a.ffp_out[o] = a.ffp[o];
    }
}

// Function/depth.f90:231-250 at one point
__global__ void k_depth_ave(Dom D, Levels L, double *u, double *utr, const float *mask, int kbcl)
{
    const int m = D.bnd_x1 + 1 + blockIdx.x * BX + threadIdx.x;
    const int n = D.bnd_y1 + 1 + blockIdx.y * BY + threadIdx.y;
    if (m > D.bnd_x2 - 1 || n > D.bnd_y2 - 1) return;
    const long long i = X(m, n);
    if (!(mask[i] > 0.5f)) return;
    double ff0 = 0.0;
    for (int k = 0; k < L.nz; k++) ff0 = ff0 + u[(long long)k * L.plane + i] * L.dz[k];
    utr[i] = ff0;
    const double kb = (double)kbcl;
    for (int k = 0; k < L.nz; k++) {
        const long long o = (long long)k * L.plane + i;
        u[o] = u[o] - kb * ff0;
    }
}

// Control/dyncall.f90:170-183 / :215-229 at one point of the interior and its ring
__global__ void k_shift_barotropic(Dom D, GridDev g, Levels L, double *uu, double *vv, const double *uu2d,
                                   const double *vv2d, int sign)
{
    const int m = D.nx_start - 1 + blockIdx.x * BX + threadIdx.x;
    const int n = D.ny_start - 1 + blockIdx.y * BY + threadIdx.y;
    if (m > D.nx_end + 1 || n > D.ny_end + 1) return;
    const long long i = X(m, n);
    if (g.lcu[i] > 0.5f) {
        const double s = uu2d[i];
        for (int k = 0; k < L.nz; k++) {
            const long long o = (long long)k * L.plane + i;
            uu[o] = sign < 0 ? uu[o] - s : uu[o] + s;
        }
    }
    if (g.lcv[i] > 0.5f) {
        const double s = vv2d[i];
        for (int k = 0; k < L.nz; k++) {
            const long long o = (long long)k * L.plane + i;
            vv[o] = sign < 0 ? vv[o] - s : vv[o] + s;
        }
    }
}

// Function/mixing.f90:129-153 at one point of the interior, level blockIdx.z
__global__ void k_stress3(Dom D, GridDev g, Levels L, const double *u, const double *v, double *str_t,
                          double *str_s)
{
    const int m = D.nx_start + blockIdx.x * BX + threadIdx.x;
    const int n = D.ny_start + blockIdx.y * BY + threadIdx.y;
    if (m > D.nx_end || n > D.ny_end) return;
    const long long o = (long long)blockIdx.z * L.plane;
    const double *uk = u + o, *vk = v + o;
    const double *dx = g.dx, *dy = g.dy, *dxh = g.dxh, *dyh = g.dyh;
    const double *dxt = g.dxt, *dyt = g.dyt, *dxb = g.dxb, *dyb = g.dyb;
    if (g.lu[X(m, n)] > 0.5f)
        str_t[o + X(m, n)] =
            dy[X(m, n)] / dx[X(m, n)] * (uk[X(m, n)] / dyh[X(m, n)] - uk[X(m - 1, n)] / dyh[X(m - 1, n)]) -
            dx[X(m, n)] / dy[X(m, n)] * (vk[X(m, n)] / dxh[X(m, n)] - vk[X(m, n - 1)] / dxh[X(m, n - 1)]);
    if (g.luu[X(m, n)] > 0.5f)
        str_s[o + X(m, n)] =
            dxb[X(m, n)] / dyb[X(m, n)] * (uk[X(m, n + 1)] / dxt[X(m, n + 1)] - uk[X(m, n)] / dxt[X(m, n)]) +
            dyb[X(m, n)] / dxb[X(m, n)] * (vk[X(m + 1, n)] / dyt[X(m + 1, n)] - vk[X(m, n)] / dyt[X(m, n)]);
}

// Function/mixing.f90:186-199 at one point of the interior, level
// blockIdx.z; kp = vonkarman/Pi
__global__ void k_smagorinsky3(Dom D, GridDev g, Levels L, double visc2, double dift, double kp,
                               const double *str_t, const double *str_s, double *amts, double *amuv)
{
    const int m = D.nx_start + blockIdx.x * BX + threadIdx.x;
    const int n = D.ny_start + blockIdx.y * BY + threadIdx.y;
    if (m > D.nx_end || n > D.ny_end) return;
    if (!(g.lu[X(m, n)] > 0.5f)) return;
    const long long o = (long long)blockIdx.z * L.plane;
    const double *sk = str_s + o;
    const double s0 = sk[X(m, n)], s1 = sk[X(m - 1, n)], s2 = sk[X(m, n - 1)], s3 = sk[X(m - 1, n - 1)];
    const double str_s2 = (s0 * s0 + s1 * s1 + s2 * s2 + s3 * s3) / 4.0;
    const double st = str_t[o + X(m, n)];
    const double mu_smag = kp * kp * g.dx[X(m, n)] * g.dy[X(m, n)] * sqrt(st * st + str_s2);
    amuv[o + X(m, n)] = visc2 + mu_smag;
    amts[o + X(m, n)] = dift + mu_smag * 0.1;   // prandtl = 0.1d0 (:177)
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

int baroclinic_rows(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const BaroclinicArgs &a,
                    int n0, int n1, cudaStream_t s)
{
    // the staged segments need an even row pitch and level stride
    if (L.nz < 2 || L.nz > MAX_NZ || wrap_inside(d) || d.pitch % 2 || L.plane % 2 || !a.flag) return -1;
    if (n0 < d.ny_start || n1 > d.ny_end || n0 > n1) return -1;
    const int nxi = d.nx_end - d.nx_start + 1;
    const size_t smem = staged_smem(L.nz);
    // per device: set on every call (the context's device is current)
    if (cudaFuncSetAttribute(k_columns, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -1;
    k_columns<<<dim3((nxi + CW - 1) / CW, n1 - n0 + 1), (NCW + 1) * 32, smem, s>>>(d, g, L, a, c.ts, n0);
    return 0;
}

int baroclinic_border(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const BaroclinicArgs &a,
                      cudaStream_t s)
{
    const int nxi = d.nx_end - d.nx_start + 1, nyi = d.ny_end - d.ny_start + 1;
    const int count = d.nxa() * d.nya() - nxi * nyi;
    if (count > 0) k_border<<<dim3((count + 127) / 128, L.nz), 128, 0, s>>>(d, g, L, a, c.ts, count);
    return 0;
}

int baroclinic_dynamics(const Dom &d, const GridDev &g, const Consts &c, const Levels &L,
                        const BaroclinicArgs &a, cudaStream_t s)
{
    if (baroclinic_rows(d, g, c, L, a, d.ny_start, d.ny_end, s)) return -1;
    return baroclinic_border(d, g, c, L, a, s);
}

int tracer_rows(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const TracerArgs &a, int n0, int n1,
                cudaStream_t s)
{
    // the staged kernels' 16-byte segments need an even row pitch and level stride
    if (L.nz < 2 || L.nz > MAX_NZ || wrap_inside(d) || d.pitch % 2 || L.plane % 2 || !a.flag) return -1;
    if (n0 < d.ny_start || n1 > d.ny_end || n0 > n1) return -1;
    // the y-fluxes' periodic wrap needs every row's fluxes first
    if (d.py && (n0 != d.ny_start || n1 != d.ny_end)) return -1;
    const int nxi = d.nx_end - d.nx_start + 1, rows = n1 - n0 + 1;
    const size_t fsm = flux_smem(L.nz);
    if (cudaFuncSetAttribute(k_tracer_flux, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm) != cudaSuccess)
        return -1;
    k_tracer_flux<<<dim3((nxi + CW - 1) / CW, rows), (NCW + 1) * 32, fsm, s>>>(d, g, L, a, n0);
    // the x-fluxes wrap in x, the y-fluxes in y (Function/tem_sal.f90:264-274); the x wrap
    // copies whole columns, so a band's wrap also rewrites the earlier bands' (final) rows
    if (d.px) {
        k_cyclize_x3<<<dim3((d.nya() + 127) / 128, L.nz), 128, 0, s>>>(d, L.plane, a.flux_x);
        for (double *f : {a.flux_zx, a.coef_zx, a.sfgm_zx})
            k_cyclize_x3<<<dim3((d.nya() + 127) / 128, L.nz + 1), 128, 0, s>>>(d, L.plane, f);
    }
    if (d.py) {
        k_cyclize_y3<<<dim3((d.nxa() + 127) / 128, L.nz), 128, 0, s>>>(d, L.plane, a.flux_y);
        for (double *f : {a.flux_zy, a.coef_zy, a.sfgm_zy})
            k_cyclize_y3<<<dim3((d.nxa() + 127) / 128, L.nz + 1), 128, 0, s>>>(d, L.plane, f);
    }
    const size_t smem = tracer_smem(L.nz);
    if (cudaFuncSetAttribute(k_tracer_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -1;
    k_tracer_solve<<<dim3((nxi + CW - 1) / CW, rows), 3 * 32, smem, s>>>(d, g, L, a, c.ts, n0);
    return 0;
}

int tracer_border(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const TracerArgs &a,
                  cudaStream_t s)
{
    const int nxi = d.nx_end - d.nx_start + 1, nyi = d.ny_end - d.ny_start + 1;
    const int count = d.nxa() * d.nya() - nxi * nyi;
    if (count > 0) k_tracer_border<<<dim3((count + 127) / 128, L.nz), 128, 0, s>>>(d, g, L, a, c.ts, count);
    return 0;
}

int tracer_tran_diff(const Dom &d, const GridDev &g, const Consts &c, const Levels &L, const TracerArgs &a,
                     cudaStream_t s)
{
    if (tracer_rows(d, g, c, L, a, d.ny_start, d.ny_end, s)) return -1;
    return tracer_border(d, g, c, L, a, s);
}

int depth_ave(const Dom &d, const Levels &L, double *u, double *utr, const float *mask, int kbcl, cudaStream_t s)
{
    if (L.nz < 1) return -1;
    const int w = d.nxa() - 2, h = d.nya() - 2;
    if (w < 1 || h < 1) return 0;
    k_depth_ave<<<dim3((w + BX - 1) / BX, (h + BY - 1) / BY), dim3(BX, BY), 0, s>>>(d, L, u, utr, mask, kbcl);
    return 0;
}

int stress_components(const Dom &d, const GridDev &g, const Levels &L, const double *u, const double *v,
                      double *str_t, double *str_s, cudaStream_t s)
{
    if (L.nz < 1 || L.nz > 65535) return -1;
    const int nxi = d.nx_end - d.nx_start + 1, nyi = d.ny_end - d.ny_start + 1;
    k_stress3<<<dim3((nxi + BX - 1) / BX, (nyi + BY - 1) / BY, L.nz), dim3(BX, BY), 0, s>>>(d, g, L, u, v, str_t,
                                                                                            str_s);
    halo3(d, str_t, L.nz, L.plane, s);
    halo3(d, str_s, L.nz, L.plane, s);
    return 0;
}

int smagorinsky_coeff(const Dom &d, const GridDev &g, const Levels &L, double visc2, double dift, double kp,
                      const double *str_t, const double *str_s, double *amts, double *amuv, cudaStream_t s)
{
    if (L.nz < 1 || L.nz > 65535) return -1;
    const int nxi = d.nx_end - d.nx_start + 1, nyi = d.ny_end - d.ny_start + 1;
    k_smagorinsky3<<<dim3((nxi + BX - 1) / BX, (nyi + BY - 1) / BY, L.nz), dim3(BX, BY), 0, s>>>(
        d, g, L, visc2, dift, kp, str_t, str_s, amts, amuv);
    halo3(d, amuv, L.nz, L.plane, s);
    halo3(d, amts, L.nz, L.plane, s);
    return 0;
}

int shift_barotropic(const Dom &d, const GridDev &g, const Levels &L, double *uu, double *vv, const double *uu2d,
                     const double *vv2d, int sign, cudaStream_t s)
{
    if (L.nz < 1) return -1;
    const int w = d.nx_end - d.nx_start + 3, h = d.ny_end - d.ny_start + 3;
    k_shift_barotropic<<<dim3((w + BX - 1) / BX, (h + BY - 1) / BY), dim3(BX, BY), 0, s>>>(d, g, L, uu, vv, uu2d,
                                                                                            vv2d, sign);
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
