// Fused streaming kernel of the barotropic step (see fused.h).
//
// Work decomposition.  A CTA is one warp; lane l owns device column
// k = g0+2+l of a 32-column strip starting at device column g0+2
// (g0 = 30*strip, even).  Strip columns 1..30 are written, so strips overlap
// by two columns.  The CTA marches down a chunk of rows [r0, r1); iteration
// j of its row loop computes
//   stage 1,  row j  : u/v-point depths of the current level, the transports
//                      U = u*hu and V = v*hv, and loads the forcing of row j;
//   stage 2,  row j-1: new SSH (continuity), advective fluxes on T and h
//                      points, Coriolis-plus-metric-vorticity products,
//                      tension and shear stresses times viscosity and depth;
//   stage 3u, row j-1: u momentum and the SSH update (time-mean sums,
//                      Robert-Asselin filter and time shift, stores);
//   stage 3v, row j-2: the same for v (it needs stage 2 of the row above).
// A value needed from a neighbouring column comes from the neighbouring lane
// by a warp shuffle; values of earlier rows stay in registers, in three
// instances of each per-row struct that the three-fold unrolled row loop
// renames instead of copying.  There is no CTA barrier, and the per-column
// arithmetic is branch-free (masked selects, predicated stores) except for
// warp-wide skips of rows without ocean.
//
// Input rows j-2..j+1 of the state, the rest depth (and, in the general
// variant, the 2-D forcing fields and the row's metric coefficients) plus the
// row's T-mask bits sit in a ring of RING shared-memory slots.  Lane 0 refills
// the slot of row j-2 with row j-2+RING by 1-D bulk TMA copies
// (cp.async.bulk, no multicast) completing on that slot's mbarrier.  Every
// wait is bounded: on timeout the CTA sets a status bit, drains its own
// copies (bounded) and returns.
//
// Two variants: UNI for square uniform grids (every metric array equal to
// one spacing d; all metric factors fold into a few constants and only the
// Coriolis parameter varies by row) with spatially uniform viscosity, drag
// and water flux; GEN for metrics that vary along y and 2-D forcing fields.
#include "fused.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace inmsom {
namespace fused {

namespace {

constexpr int NL = 32;            // lanes = threads per CTA = strip columns
constexpr int OUTW = NL - 2;      // written columns per strip
constexpr int SEG = NL + 4;       // ring segment: strip columns -2 .. 33
constexpr int RING = 6;           // ring slots (4 rows in use + 2 in flight)
constexpr int COEF_D = (int)(sizeof(RowCoef) / sizeof(double));
constexpr unsigned WAIT_LIMIT = 1u << 20;

// state order, as the *_e arguments: u, up, v, vp, ssh, sshp
enum { S_U, S_UP, S_V, S_VP, S_SSH, S_SSHP };
// ring fields
enum { R_U, R_V, R_SSH, R_UP, R_VP, R_SSHP, R_H, R_NUNI, R_MU = R_NUNI, R_RD, R_WF, R_NGEN };

struct Params {
    const double *src[6];
    double *dst[6];
    const double *H, *rhsx, *rhsy, *mu, *rdis, *wflux;
    double *acc[4];
    const uint32_t *bits;
    const RowCoef *rows;
    const double *cor;
    long long pitch;
    int bm_words;
    int chunk_rows;
    int r_first, r_last;   // interior device rows
    int c_first, c_last;   // interior device columns
    double two_ti, gam, c4, rhs_scale, mu0, rd0, wq0, inv_rho;
    double d, inv_d, d4, gd, d2, inv_d2;   // UNI metric constants
    int vort_zero;
    unsigned *flags;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

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
    for (unsigned i = 0; i < WAIT_LIMIT; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 1-D bulk copy global -> this CTA's shared memory, completion on *bar
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

template <bool GEN>
struct Layout {
    static constexpr int NF = GEN ? R_NGEN : R_NUNI;
    static constexpr int NCOEF = GEN ? COEF_D : 0;
    static constexpr int SLOT_D = NF * SEG + NCOEF + 4;   // doubles per slot (4 = 8 mask words)
    static constexpr size_t bytes = (size_t)RING * SLOT_D * sizeof(double) + RING * sizeof(uint64_t);
    static constexpr uint32_t row_tx = (uint32_t)(SLOT_D * sizeof(double));
    static constexpr int min_ctas = GEN ? 10 : 12;
};

__device__ __forceinline__ double sel(int m, double x) { return m ? x : 0.0; }

// 1 / (number of ocean T points) for the mask-weighted depth averages
__device__ __forceinline__ double rcount(int n)
{
    return n == 4 ? 0.25 : (n == 3 ? 1.0 / 3.0 : (n == 2 ? 0.5 : (n == 1 ? 1.0 : 0.0)));
}

// 1/x by two Newton-Raphson steps r <- r + r*(1 - x*r) (quadratic
// convergence) from the single-precision reciprocal: about 1 ulp of double
// for a positive normal x inside the float range, such as a water depth.
__device__ __forceinline__ double rcp_nr(double x)
{
    double r = (double)__frcp_rn((float)x);
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

#define SHFL_UP(x) __shfl_up_sync(0xffffffffu, (x), 1)
#define SHFL_DN(x) __shfl_down_sync(0xffffffffu, (x), 1)

// per-row values carried between the stages of the row pipeline
struct S1 {          // stage 1 of a row
    double U, V;             // U = u*hu, V = v*hv
    double Ul, Vr;           // U(k-1), V(k+1) from the neighbouring lanes
    double hu, hv;           // current-level u/v depths
    double rx, ry;           // forcing RHSx, RHSy of the row
};
struct HQ {          // H + ssh of a row at k, k+1
    double a, b;
};
struct S2 {          // stage 2 of a row
    double sn;               // new SSH
    double FY, QU, SS, GX, GXl, GY, QV, QVl, ST, SSl;
};

// MODE = acc + 3*write: acc 0 none, 1 first substep (write), 2 accumulate;
// write 1 stores the new state
template <bool GEN, int MODE>
__global__ void __launch_bounds__(NL, Layout<GEN>::min_ctas) k_substep(const __grid_constant__ Params p)
{
    using L = Layout<GEN>;
    constexpr int NF = L::NF;
    constexpr int ACC = MODE % 3;
    constexpr bool WRITE = MODE / 3 != 0;
    extern __shared__ __align__(128) double smem[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + RING * L::SLOT_D);

    const int l = threadIdx.x;
    const int g0 = blockIdx.x * OUTW;          // device column of segment offset 0
    const int k = g0 + 2 + l;                  // this lane's column
    const int r0 = p.r_first + blockIdx.y * p.chunk_rows;
    const int r1 = min(r0 + p.chunk_rows, p.r_last + 1);   // exclusive
    if (r0 >= r1) return;
    const int row_lo = r0 - 2, row_hi = r1 + 1;             // rows kept in the ring
    const int wbase = (g0 >> 7) << 2;                       // first mask word of the window
    const int bsh = k - wbase * 32;                         // bit of k in the window
    const int po = l + 2;                                   // segment offset of k

    auto slotp = [&](int s) { return smem + (size_t)s * L::SLOT_D; };
    auto slot_of = [&](int row) { return (row - row_lo) % RING; };
    auto issue = [&](int row) {
        const int s = slot_of(row);
        double *dd = slotp(s);
        uint64_t *bar = &mbar[s];
        mbar_expect_tx(bar, L::row_tx);
        const long long off = (long long)row * p.pitch + g0;
        const uint32_t nb = SEG * sizeof(double);
        bulk_load(dd + R_U * SEG, p.src[S_U] + off, nb, bar);
        bulk_load(dd + R_V * SEG, p.src[S_V] + off, nb, bar);
        bulk_load(dd + R_SSH * SEG, p.src[S_SSH] + off, nb, bar);
        bulk_load(dd + R_UP * SEG, p.src[S_UP] + off, nb, bar);
        bulk_load(dd + R_VP * SEG, p.src[S_VP] + off, nb, bar);
        bulk_load(dd + R_SSHP * SEG, p.src[S_SSHP] + off, nb, bar);
        bulk_load(dd + R_H * SEG, p.H + off, nb, bar);
        if constexpr (GEN) {
            bulk_load(dd + R_MU * SEG, p.mu + off, nb, bar);
            bulk_load(dd + R_RD * SEG, p.rdis + off, nb, bar);
            bulk_load(dd + R_WF * SEG, p.wflux + off, nb, bar);
            bulk_load(dd + NF * SEG, p.rows + row, sizeof(RowCoef), bar);
        }
        bulk_load(dd + NF * SEG + L::NCOEF, p.bits + (size_t)row * p.bm_words + wbase, 32, bar);
    };
    auto at = [&](int s, int f, int dk) { return slotp(s)[f * SEG + po + dk]; };
    auto mask2 = [&](int s) -> uint32_t {   // bits: lu(k), lu(k+1)
        const uint32_t *w = reinterpret_cast<const uint32_t *>(slotp(s) + NF * SEG + L::NCOEF);
        return __funnelshift_r(w[bsh >> 5], w[(bsh >> 5) + 1], bsh & 31) & 3u;
    };
    auto coef = [&](int s) { return reinterpret_cast<const RowCoef *>(slotp(s) + NF * SEG); };
    // metric coefficient of the row in slot s: GEN from the ring, UNI folded
#define CG(s, x) coef(s)->x
#define C_KU(s) (GEN ? CG(s, ku) : 1.0)
#define C_KU2(s) (GEN ? CG(s, ku2) : 0.5)
#define C_WV0(s) (GEN ? CG(s, wv0) : 1.0)
#define C_WV1(s) (GEN ? CG(s, wv1) : 1.0)
#define C_D4(s, x) (GEN ? CG(s, x) : p.d4)
#define C_GD(s, x) (GEN ? CG(s, x) : p.gd)
#define C_D2(s, x) (GEN ? CG(s, x) : p.d2)
#define C_INVD2(s, x) (GEN ? CG(s, x) : p.inv_d2)

    if (l == 0) {
        for (int s = 0; s < RING; s++) mbar_init(&mbar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    int issued = row_lo - 1;
    if (l == 0)
        for (int row = row_lo; row < row_lo + RING && row <= row_hi; row++) issue(row), issued = row;

    const bool out = l >= 1 && l <= NL - 2 && k >= p.c_first && k <= p.c_last;
    const double gam = p.gam, two_ti = p.two_ti, rs = p.rhs_scale;

    // T-mask bits, 2 per row: row j+1 in bits 0-1, j in 2-3, j-1 in 4-5, j-2 in 6-7
    uint32_t mk = 0;
    uint32_t bad = 0;   // guard: a new value out of range or NaN
    int waited = row_lo - 1;
    bool ok = true;
    auto wait_upto = [&](int need) {
        while (waited < need && ok) {
            const int row = waited + 1;
            if (!mbar_wait(&mbar[slot_of(row)], (uint32_t)(((row - row_lo) / RING) & 1))) { ok = false; break; }
            waited = row;
            mk = (mk << 2) | mask2(slot_of(row));
        }
        ok = __all_sync(0xffffffffu, ok);
    };

    auto step = [&](const int j, S1 &s1n, const S1 &s1c, const S1 &s1p, HQ &hqn, const HQ &hqc,
                    const HQ &hqp, S2 &s2n, const S2 &s2o) {
        wait_upto(min(j + 1, row_hi));
        if (j + 1 > row_hi) mk <<= 2;   // keep the row alignment of mk
        if (!ok) return;
        const int s_m2 = slot_of(j - 2), s_m1 = slot_of(j - 1), s_0 = slot_of(j), s_p1 = slot_of(j + 1);

        // ---------------- stage 1: row j ---------------------------------
        if (j <= r1) {
            const uint32_t mj = (mk >> 2) & 3u, mn = mk & 3u;
            hqn.a = at(s_p1, R_H, 0) + at(s_p1, R_SSH, 0);
            hqn.b = at(s_p1, R_H, 1) + at(s_p1, R_SSH, 1);
            const int a = mj & 1, b = (mj >> 1) & 1, c = mn & 1;
            // Function/depth.f90:127-139 mask-weighted averages to u and v points
            const double hu = (sel(a, hqc.a) + sel(b, hqc.b)) * (a & b ? C_KU2(s_0) : (a | b ? C_KU(s_0) : 0.0));
            const double hv = (sel(a, hqc.a * C_WV0(s_0)) + sel(c, hqn.a * C_WV1(s_0))) *
                              (a & c ? 0.5 : (a | c ? 1.0 : 0.0));
            s1n.hu = hu;
            s1n.hv = hv;
            s1n.U = at(s_0, R_U, 0) * hu;
            s1n.V = at(s_0, R_V, 0) * hv;
            const long long gi = (long long)j * p.pitch + k;
            s1n.rx = p.rhsx[gi];
            s1n.ry = p.rhsy[gi];
        }
        s1n.Ul = SHFL_UP(s1n.U);
        s1n.Vr = SHFL_DN(s1n.V);

        // ---------------- stage 2: row rho = j-1 -------------------------
        double FX = 0.0, u_r = 0.0, up_r = 0.0;
        if (j >= r0 && j <= r1 + 1) {
            const uint32_t mr = (mk >> 4) & 3u, mu_ = (mk >> 2) & 3u;   // rows rho, rho+1
            const int sr = s_m1, sm = s_m2, su = s_0;
            const int lc = mr & 1, lr = (mr >> 1) & 1, lu = mu_ & 1, lur = (mu_ >> 1) & 1;
            const int luu = lc & lr & lu & lur;
            u_r = at(sr, R_U, 0);
            up_r = at(sr, R_UP, 0);
            const double u_l = at(sr, R_U, -1), u_u = at(su, R_U, 0);
            const double v_r = at(sr, R_V, 0), v_rr = at(sr, R_V, 1), v_m = at(sm, R_V, 0);
            const double up_l = at(sr, R_UP, -1), up_u = at(su, R_UP, 0);
            const double vp_r = at(sr, R_VP, 0), vp_rr = at(sr, R_VP, 1), vp_m = at(sm, R_VP, 0);
            double mu_t = p.mu0, mu_h = p.mu0, wq = p.wq0;
            if constexpr (GEN) {
                mu_t = at(sr, R_MU, 0);
                mu_h = (mu_t + at(sr, R_MU, 1) + at(su, R_MU, 0) + at(su, R_MU, 1)) * 0.25;
                wq = at(sr, R_WF, 0) * p.inv_rho;
            }
            // vel_ssh.f90:491-494 continuity over 2*tau_inner
            const double div = GEN ? (s1c.U - s1c.Ul) * CG(sr, c_u) + s1c.V * CG(sr, c_v0) - s1p.V * CG(sr, c_v1)
                                   : ((s1c.U - s1c.Ul) + (s1c.V - s1p.V)) * p.inv_d;
            s2n.sn = sel(lc, at(sr, R_SSHP, 0) + two_ti * (wq - div));
            // vel_ssh.f90:63-73, :88-98 advective fluxes on T and h faces
            FX = (s1c.Ul + s1c.U) * (u_l + u_r) * C_D4(sr, fx);
            s2n.FY = sel(luu, (s1c.V + s1c.Vr) * (u_r + u_u) * C_D4(sr, fy));
            s2n.GX = (GEN ? s1c.U * CG(sr, gx0) + s1n.U * CG(sr, gx1) : (s1c.U + s1n.U) * p.d4) * (v_r + v_rr);
            s2n.GY = (GEN ? s1p.V * CG(sr, gy0) + s1c.V * CG(sr, gy1) : (s1p.V + s1c.V) * p.d4) * (v_m + v_r);
            // depth.f90:141-147 depth on the h point
            const double sa = sel(lc, hqp.a) + sel(lr, hqp.b);
            const double sb = sel(lu, hqc.a) + sel(lur, hqc.b);
            const double hh = (GEN ? sa * CG(sr, wh0) + sb * CG(sr, wh1) : sa + sb) * rcount(lc + lr + lu + lur);
            // vel_ssh.f90:35-37 metric vorticity (zero on uniform grids) + Coriolis
            double cor;
            if constexpr (GEN) {
                cor = CG(sr, cor);
                if (!p.vort_zero)
                    cor += sel(luu, (v_rr - v_r) * CG(sr, vt0) - u_u * CG(sr, vt1) + u_r * CG(sr, vt2));
            } else {
                cor = p.cor[j - 1];
            }
            const double Wh = hh * cor;
            s2n.QU = Wh * (v_r + v_rr);
            s2n.QV = Wh * (u_r + u_u);
            // mixing.f90:134-148 stresses from the previous level
            const double str_t = GEN ? sel(lc, CG(sr, t1) * (up_r - up_l) - (CG(sr, t2) * vp_r - CG(sr, t3) * vp_m))
                                     : sel(lc, ((up_r - up_l) - (vp_r - vp_m)) * p.inv_d);
            const double str_s = GEN ? sel(luu, CG(sr, s1) * up_u - CG(sr, s2) * up_r + CG(sr, s3) * (vp_rr - vp_r))
                                     : sel(luu, ((up_u - up_r) + (vp_rr - vp_r)) * p.inv_d);
            s2n.ST = mu_t * hqp.a * str_t;
            s2n.SS = mu_h * hh * str_s;
        }
        const double FXr = SHFL_DN(FX);
        const double STr = SHFL_DN(s2n.ST);
        const double SNr = SHFL_DN(s2n.sn);
        s2n.GXl = SHFL_UP(s2n.GX);
        s2n.QVl = SHFL_UP(s2n.QV);
        s2n.SSl = SHFL_UP(s2n.SS);

        // ---------------- stage 3u: row rho = j-1 (u and SSH) -----------
        const uint32_t mr = (mk >> 4) & 3u;
        if (j >= r0 + 1 && j <= r1 && __any_sync(0xffffffffu, out && (mr & 1u))) {
            const int sr = s_m1;
            const int lc = mr & 1, lr = (mr >> 1) & 1;
            const bool wu = out && (lc & lr), wt = out && lc;
            const double e0 = at(sr, R_SSH, 0), e1 = at(sr, R_SSH, 1);
            const double sp0 = at(sr, R_SSHP, 0), sp1 = at(sr, R_SSHP, 1);
            const double h0 = at(sr, R_H, 0), h1 = at(sr, R_H, 1);
            const double sn0 = s2n.sn;
            // vel_ssh.f90:536-551
            const double hu = s1c.hu;
            const double hup = ((h0 + sp0) + (h1 + sp1)) * C_KU2(sr);
            const double hun = ((h0 + sn0) + (h1 + SNr)) * C_KU2(sr);
            const double slx = -(e1 - e0) * C_GD(sr, gdyh) * hu;
            const double slxn = -(SNr - sn0) * C_GD(sr, gdyh) * hun;
            const double adv = -((FXr - FX) + (s2n.FY - s2o.FY));
            const double dif = GEN ? (STr - s2n.ST) * CG(sr, dux) + (s2n.SS * CG(sr, dus0) - s2o.SS * CG(sr, dus1))
                                   : ((STr - s2n.ST) + (s2n.SS - s2o.SS)) * p.d;
            double rd = p.rd0;
            if constexpr (GEN) rd = (at(sr, R_RD, 0) + at(sr, R_RD, 1)) * 0.5;
            const double grx = s1c.rx * rs + slx + dif + adv - rd * up_r * C_D2(sr, au) * hu
                               + (s2n.QU + s2o.QU) * 0.25;
            const double un = (up_r * hup + grx * (two_ti * C_INVD2(sr, rau))) * rcp_nr(hun);
            bad |= (uint32_t)(wu && !(un < 100.0 && un > -100.0));
            bad |= (uint32_t)(wt && !(sn0 < 10.0 && sn0 > -10.0));
            const long long idx = (long long)(j - 1) * p.pitch + k;
            if (ACC && wu) {
                double a = (u_r * hu + un * hun) * p.c4, b = (slx + slxn) * p.c4;
                if (ACC == 2) { a += p.acc[0][idx]; b += p.acc[2][idx]; }
                p.acc[0][idx] = a;
                p.acc[2][idx] = b;
            }
            if (WRITE && wu) {
                p.dst[S_UP][idx] = u_r + gam * (un - 2.0 * u_r + up_r);
                p.dst[S_U][idx] = un;
            }
            if (WRITE && wt) {   // vel_ssh.f90:593-596
                p.dst[S_SSHP][idx] = e0 + gam * (sn0 - 2.0 * e0 + sp0);
                p.dst[S_SSH][idx] = sn0;
            }
        }

        // ---------------- stage 3v: row R = j-2 (v) ----------------------
        const uint32_t mR = (mk >> 6) & 3u, mU = (mk >> 4) & 3u;   // rows R, R+1
        if (j >= r0 + 2 && j <= r1 + 1 && __any_sync(0xffffffffu, out && (mR & mU & 1u))) {
            const int sR = s_m2, sU = s_m1;
            const bool wv = out && (mR & mU & 1u);
            const double e0 = at(sR, R_SSH, 0), e1 = at(sU, R_SSH, 0);
            const double sp0 = at(sR, R_SSHP, 0), sp1 = at(sU, R_SSHP, 0);
            const double h0 = at(sR, R_H, 0), h1 = at(sU, R_H, 0);
            const double v0 = at(sR, R_V, 0), vp0 = at(sR, R_VP, 0);
            const double sn0 = s2o.sn, sn1 = s2n.sn;
            // vel_ssh.f90:554-569
            const double hv = s1p.hv;
            const double hvp = (GEN ? (h0 + sp0) * CG(sR, wv0) + (h1 + sp1) * CG(sR, wv1) : (h0 + sp0) + (h1 + sp1)) * 0.5;
            const double hvn = (GEN ? (h0 + sn0) * CG(sR, wv0) + (h1 + sn1) * CG(sR, wv1) : (h0 + sn0) + (h1 + sn1)) * 0.5;
            const double sly = -(e1 - e0) * C_GD(sR, gdxh) * hv;
            const double slyn = -(sn1 - sn0) * C_GD(sR, gdxh) * hvn;
            const double adv = -((s2o.GX - s2o.GXl) + (s2n.GY - s2o.GY));
            const double dif = GEN ? -(s2n.ST * CG(sR, dvt1) - s2o.ST * CG(sR, dvt0)) + (s2o.SS - s2o.SSl) * CG(sR, dvs)
                                   : (-(s2n.ST - s2o.ST) + (s2o.SS - s2o.SSl)) * p.d;
            double rd = p.rd0;
            if constexpr (GEN) rd = (at(sR, R_RD, 0) + at(sU, R_RD, 0)) * 0.5;
            const double gry = s1p.ry * rs + sly + dif + adv - rd * vp0 * C_D2(sR, av) * hv
                               - (s2o.QV + s2o.QVl) * 0.25;
            const double vn = (vp0 * hvp + gry * (two_ti * C_INVD2(sR, rav))) * rcp_nr(hvn);
            bad |= (uint32_t)(wv && !(vn < 100.0 && vn > -100.0));
            const long long idx = (long long)(j - 2) * p.pitch + k;
            if (ACC && wv) {
                double a = (v0 * hv + vn * hvn) * p.c4, b = (sly + slyn) * p.c4;
                if (ACC == 2) { a += p.acc[1][idx]; b += p.acc[3][idx]; }
                p.acc[1][idx] = a;
                p.acc[3][idx] = b;
            }
            if (WRITE && wv) {
                p.dst[S_VP][idx] = v0 + gam * (vn - 2.0 * v0 + vp0);
                p.dst[S_V][idx] = vn;
            }
        }
        // row j-2 was last read above: once every lane is past it, its slot
        // takes row j-2+RING
        __syncwarp();
        if (l == 0) {
            const int dead = j - 2;
            if (dead >= row_lo && dead + RING <= row_hi) issue(dead + RING), issued = dead + RING;
        }
    };

    // H + ssh of row r0-1, the stage-1 "current" row of the first step
    HQ HA{}, HB{}, HC{};
    wait_upto(row_lo + 1);
    if (ok) {
        const int s = slot_of(r0 - 1);
        HC.a = at(s, R_H, 0) + at(s, R_SSH, 0);
        HC.b = at(s, R_H, 1) + at(s, R_SSH, 1);
    }
    // three instances of each carried struct, renamed (not copied) by the
    // three-fold unrolled loop
    S1 A{}, B{}, C{};
    S2 X{}, Y{}, Z{};
    for (int j = r0 - 1; j <= r1 + 1 && ok; j += 3) {
        step(j, A, C, B, HA, HC, HB, X, Z);
        step(j + 1, B, A, C, HB, HA, HC, Y, X);
        step(j + 2, C, B, A, HC, HB, HA, Z, Y);
    }
    if (__any_sync(0xffffffffu, bad != 0) && l == 0) atomicOr(p.flags, FLAG_GUARD);
    if (!ok && l == 0) {
        atomicOr(p.flags, FLAG_TIMEOUT);
        // drain this CTA's copies still in flight (bounded) before exiting
        for (int row = max(waited + 1, row_lo); row <= issued; row++)
            (void)mbar_wait(&mbar[slot_of(row)], (uint32_t)(((row - row_lo) / RING) & 1));
    }
#undef CG
#undef C_KU
#undef C_KU2
#undef C_WV0
#undef C_WV1
#undef C_D4
#undef C_GD
#undef C_D2
#undef C_INVD2
}

// min/max over the ocean points of three fields, for the uniform-forcing test
__global__ void k_minmax3(Dom D, const float *lu, const double *a, const double *b, const double *c3, double *out)
{
    __shared__ double sh[6][256];
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int w = D.nx_end - D.nx_start + 3, h = D.ny_end - D.ny_start + 3;
    const long long tot = (long long)w * h;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot; k += (long long)gridDim.x * blockDim.x) {
        const int m = D.nx_start - 1 + (int)(k % w), n = D.ny_start - 1 + (int)(k / w);
        const long long i = ix(D, m, n);
        if (!(lu[i] > 0.5f)) continue;   // the step reads these fields at ocean points only
        const double v[3] = {a[i], b[i], c3[i]};
        for (int q = 0; q < 3; q++) {
            // a NaN makes the field non-uniform
            mn[q] = (v[q] < mn[q] || v[q] != v[q]) ? v[q] : mn[q];
            mx[q] = (v[q] > mx[q] || v[q] != v[q]) ? v[q] : mx[q];
        }
    }
    for (int q = 0; q < 3; q++) { sh[q][threadIdx.x] = mn[q]; sh[3 + q][threadIdx.x] = mx[q]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)blockDim.x; k++)
            for (int q = 0; q < 3; q++) {
                double x = sh[q][k], y = sh[3 + q][k];
                mn[q] = (x < mn[q] || x != x) ? x : mn[q];
                mx[q] = (y > mx[q] || y != y) ? y : mx[q];
            }
        for (int q = 0; q < 3; q++) { out[blockIdx.x * 6 + q] = mn[q]; out[blockIdx.x * 6 + 3 + q] = mx[q]; }
    }
}

constexpr int MINMAX_BLOCKS = 592;

struct Forcing {
    bool uniform;
    double mu0, rd0, wq0;
};

int forcing_mode(Plan &p, const Dom &d, const Consts &c, double *forc[6], cudaStream_t s, Forcing &f)
{
    // forc order: RHSx RHSy wflux mu mu4 rdis
    k_minmax3<<<MINMAX_BLOCKS, 256, 0, s>>>(d, p.lu, forc[3], forc[5], forc[2], p.d_uniform);
    std::vector<double> h((size_t)MINMAX_BLOCKS * 6);
    if (cudaMemcpyAsync(h.data(), p.d_uniform, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return 1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return 1;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool nan = false;
    for (int b = 0; b < MINMAX_BLOCKS; b++)
        for (int q = 0; q < 3; q++) {
            double x = h[b * 6 + q], y = h[b * 6 + 3 + q];
            nan |= x != x || y != y;
            mn[q] = std::min(mn[q], x);
            mx[q] = std::max(mx[q], y);
        }
    f.uniform = !nan && mn[0] == mx[0] && mn[1] == mx[1] && mn[2] == mx[2];
    if (mn[0] > mx[0]) mn[0] = mn[1] = mn[2] = 0.0;   // no ocean at all
    f.mu0 = mn[0];
    f.rd0 = mn[1];
    f.wq0 = mn[2] / c.rho * (double)c.ffs;
    return 0;
}

Params base_params(const Plan &p, const Dom &d, const Consts &c, double *forc[6], const Forcing &f, int gen)
{
    Params q{};
    q.H = p.hrest;
    q.rhsx = forc[0];
    q.rhsy = forc[1];
    q.wflux = forc[2];
    q.mu = forc[3];
    q.rdis = forc[5];
    q.bits = p.bits;
    q.rows = p.rows;
    q.cor = p.cor;
    q.pitch = d.pitch;
    q.bm_words = p.bm_words;
    q.r_first = d.ny_start - d.bnd_y1;
    q.r_last = d.ny_end - d.bnd_y1;
    q.c_first = d.nx_start - d.bnd_x1 + d.xoff;
    q.c_last = d.nx_end - d.bnd_x1 + d.xoff;
    q.mu0 = f.mu0;
    q.rd0 = f.rd0;
    q.wq0 = f.wq0;
    q.inv_rho = 1.0 / c.rho;   // wflux/RefDen as wflux*(1/RefDen): within rounding
    q.rhs_scale = 1.0;
    q.vort_zero = p.vort_zero ? 1 : 0;
    q.flags = p.d_flags;
    q.d = p.d;
    q.inv_d = p.d != 0.0 ? 1.0 / p.d : 0.0;
    q.d4 = p.d / 4.0;
    q.gd = c.g * p.d;
    q.d2 = p.d * p.d;
    q.inv_d2 = p.d != 0.0 ? 1.0 / (p.d * p.d) : 0.0;
    q.chunk_rows = p.chunk_rows[gen];
    return q;
}

template <bool GEN, int MODE>
void launch_t(const Plan &p, const Params &q, cudaStream_t s)
{
    dim3 grid(p.nstrips, p.nchunks[GEN ? 1 : 0]);
    k_substep<GEN, MODE><<<grid, NL, Layout<GEN>::bytes, s>>>(q);
}

// mode = acc + 3*write (acc: 0 none, 1 write, 2 accumulate)
template <bool GEN>
void launch_g(const Plan &p, const Params &q, int mode, cudaStream_t s)
{
    switch (mode) {
    case 3: launch_t<GEN, 3>(p, q, s); break;
    case 4: launch_t<GEN, 4>(p, q, s); break;
    case 5: launch_t<GEN, 5>(p, q, s); break;
    default: launch_t<GEN, 2>(p, q, s); break;
    }
}

void launch(Plan &p, const Params &q, int gen, int mode, cudaStream_t s)
{
    p.last_variant = gen;
    if (gen) launch_g<true>(p, q, mode, s);
    else launch_g<false>(p, q, mode, s);
}

int sync_buffers(Plan &p, const Dom &d, double *state[6], cudaStream_t s)
{
    const size_t bytes = (size_t)d.pitch * d.nya() * sizeof(double);
    for (int b = 0; b < 2; b++)
        for (int k = 0; k < 6; k++)
            if (cudaMemcpyAsync(p.buf[b][k], state[k], bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                return 1;
    p.buffers_synced = true;
    return 0;
}

int read_flags(Plan &p, cudaStream_t s, unsigned *out)
{
    unsigned h = 0;
    if (cudaMemcpyAsync(&h, p.d_flags, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess) return 1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return 1;
    *out = h;
    return 0;
}

template <bool GEN, int MODE>
int set_smem1()
{
    return cudaFuncSetAttribute(k_substep<GEN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)Layout<GEN>::bytes) != cudaSuccess;
}

int set_smem()
{
    return set_smem1<false, 2>() | set_smem1<false, 3>() | set_smem1<false, 4>() | set_smem1<false, 5>() |
           set_smem1<true, 2>() | set_smem1<true, 3>() | set_smem1<true, 4>() | set_smem1<true, 5>();
}

}  // namespace

// ===========================================================================
Plan make_plan(const inmsom_bounds &b)
{
    Plan p;
    p.ncol = NL;
    p.outw = OUTW;
    const int nx = b.nx_end - b.nx_start + 1;
    p.nstrips = (nx + p.outw - 1) / p.outw;
    const long long g0_last = (long long)(p.nstrips - 1) * p.outw;
    p.min_pitch = g0_last + SEG;
    return p;
}

const char *check_eligible(const Plan &p, const Dom &d, const Consts &c, const float *const masks[7],
                           const double *const grid[10])
{
    (void)p;
    if (d.bnd_x1 != d.nx_start - 2 || d.bnd_x2 != d.nx_end + 2 || d.bnd_y1 != d.ny_start - 2 ||
        d.bnd_y2 != d.ny_end + 2)
        return "array bounds are not the interior plus a 2-point halo";
    if (d.px || d.py) return "periodic wrap";
    if (c.ffs != 1) return "full_free_surface != 1";
    if (d.xoff != XOFF) return "device layout without the fused column offset";
    const int nxa = d.nxa(), nya = d.nya();
    auto at = [&](const float *a, int m, int n) { return a[(size_t)(n - d.bnd_y1) * nxa + (m - d.bnd_x1)]; };
    const float *lu = masks[0];
    for (int n = d.bnd_y1; n <= d.bnd_y2; n++)
        for (int m = d.bnd_x1; m <= d.bnd_x2; m++) {
            float v = at(lu, m, n);
            if (v != 0.0f && v != 1.0f) return "lu is not 0/1";
            bool interior = m >= d.nx_start && m <= d.nx_end && n >= d.ny_start && n <= d.ny_end;
            if (!interior && v != 0.0f) return "ocean points in the halo ring";
        }
    // derived masks must be gridcon(lu) (Service/grid_construction.f90:59-112)
    std::vector<float> ref[6];
    for (auto &r : ref) r.assign((size_t)nxa * nya, 0.0f);
    for (int n = d.ny_start - 1; n <= d.ny_end; n++)
        for (int m = d.nx_start - 1; m <= d.nx_end; m++) {
            size_t i = (size_t)(n - d.bnd_y1) * nxa + (m - d.bnd_x1);
            float a = at(lu, m, n), b2 = at(lu, m + 1, n), cc = at(lu, m, n + 1), dd = at(lu, m + 1, n + 1);
            if (a * b2 * cc * dd > 0.5f) ref[0][i] = 1.0f;   // luu
            if (a + b2 + cc + dd > 0.5f) ref[1][i] = 1.0f;   // luh
            if (a * b2 > 0.5f) ref[2][i] = 1.0f;             // lcu
            if (a * cc > 0.5f) ref[3][i] = 1.0f;             // lcv
            if (a + b2 > 0.5f) ref[4][i] = 1.0f;             // llu
            if (a + cc > 0.5f) ref[5][i] = 1.0f;             // llv
        }
    for (int k = 0; k < 6; k++)
        if (std::memcmp(ref[k].data(), masks[k + 1], ref[k].size() * sizeof(float)) != 0)
            return "derived masks differ from gridcon(lu)";
    // metrics and Coriolis constant along rows over the points the step reads
    for (int k = 0; k < 9; k++)
        for (int n = d.ny_start - 1; n <= d.ny_end + 1; n++) {
            const double *g = grid[k] + (size_t)(n - d.bnd_y1) * nxa;
            const double v0 = g[d.nx_start - d.bnd_x1];
            if (!std::isfinite(v0) || (k < 8 && v0 == 0.0)) return "zero or non-finite metric";
            for (int m = d.nx_start - 1; m <= d.nx_end + 1; m++)
                if (g[m - d.bnd_x1] != v0) return "metrics or Coriolis vary along a row";
        }
    const double *hr = grid[9];
    for (size_t i = 0; i < (size_t)nxa * nya; i++)
        if (!std::isfinite(hr[i])) return "non-finite rest depth";
    return nullptr;
}

int setup(Plan &p, const Dom &d, const Consts &c, const float *const masks[7], const double *const grid[10],
          const double *d_hrest, const float *d_lu, cudaStream_t s)
{
    const int nxa = d.nxa(), nya = d.nya();
    auto row_of = [&](int k, int n) {
        n = std::min(std::max(n, d.ny_start - 1), d.ny_end + 1);
        return grid[k][(size_t)(n - d.bnd_y1) * nxa + (d.nx_start - d.bnd_x1)];
    };
    enum { DX, DY, DXT, DYT, DXH, DYH, DXB, DYB, RLH };
    std::vector<RowCoef> rows(nya);
    bool vz = true;
    for (int r = 0; r < nya; r++) {
        const int n = r + d.bnd_y1;
        auto g = [&](int k, int dn) { return row_of(k, n + dn); };
        RowCoef &q = rows[r];
        q = RowCoef{};
        const double area = g(DX, 0) * g(DY, 0), area1 = g(DX, 1) * g(DY, 1);
        q.ku = area / (g(DXT, 0) * g(DYH, 0));
        q.ku2 = 0.5 * q.ku;
        q.wv0 = area / (g(DXH, 0) * g(DYT, 0));
        q.wv1 = area1 / (g(DXH, 0) * g(DYT, 0));
        q.wh0 = area / (g(DXB, 0) * g(DYB, 0));
        q.wh1 = area1 / (g(DXB, 0) * g(DYB, 0));
        q.c_u = g(DYH, 0) / area;
        q.c_v0 = g(DXH, 0) / area;
        q.c_v1 = g(DXH, -1) / area;
        q.fx = g(DYH, 0) / 4.0;
        q.fy = g(DXH, 0) / 4.0;
        q.gx0 = g(DYH, 0) / 4.0;
        q.gx1 = g(DYH, 1) / 4.0;
        q.gy0 = g(DXH, -1) / 4.0;
        q.gy1 = g(DXH, 0) / 4.0;
        q.cor = g(RLH, 0) * g(DXB, 0) * g(DYB, 0);
        q.vt0 = g(DYT, 0) - g(DYB, 0);
        q.vt1 = g(DXT, 1) - g(DXB, 0);
        q.vt2 = g(DXT, 0) - g(DXB, 0);
        if (n >= d.ny_start - 1 && n <= d.ny_end && (q.vt0 != 0.0 || q.vt1 != 0.0 || q.vt2 != 0.0)) vz = false;
        q.t1 = g(DY, 0) / (g(DX, 0) * g(DYH, 0));
        q.t2 = g(DX, 0) / (g(DY, 0) * g(DXH, 0));
        q.t3 = g(DX, 0) / (g(DY, 0) * g(DXH, -1));
        q.s1 = g(DXB, 0) / (g(DYB, 0) * g(DXT, 1));
        q.s2 = g(DXB, 0) / (g(DYB, 0) * g(DXT, 0));
        q.s3 = g(DYB, 0) / (g(DXB, 0) * g(DYT, 0));
        q.dux = g(DY, 0) * g(DY, 0) / g(DYH, 0);
        q.dus0 = g(DXB, 0) * g(DXB, 0) / g(DXT, 0);
        q.dus1 = g(DXB, -1) * g(DXB, -1) / g(DXT, 0);
        q.dvt0 = g(DX, 0) * g(DX, 0) / g(DXH, 0);
        q.dvt1 = g(DX, 1) * g(DX, 1) / g(DXH, 0);
        q.dvs = g(DYB, 0) * g(DYB, 0) / g(DYT, 0);
        q.gdyh = c.g * g(DYH, 0);
        q.gdxh = c.g * g(DXH, 0);
        q.au = g(DXT, 0) * g(DYH, 0);
        q.av = g(DYT, 0) * g(DXH, 0);
        q.rau = 1.0 / q.au;
        q.rav = 1.0 / q.av;
    }
    p.vort_zero = vz;
    // square uniform grid: every metric array equal to one spacing over the
    // points the step reads -> the UNI variant with folded coefficients
    p.uni = true;
    p.d = row_of(DX, d.ny_start);
    for (int k = 0; k < 8 && p.uni; k++)
        for (int n = d.ny_start - 1; n <= d.ny_end + 1 && p.uni; n++)
            if (row_of(k, n) != p.d) p.uni = false;
    std::vector<double> cor(nya);
    for (int r = 0; r < nya; r++) cor[r] = row_of(RLH, r + d.bnd_y1) * p.d * p.d;
    // 1-bit T mask indexed by device column, rows padded so that every CTA
    // window (8 words from a 4-word boundary) lies inside the row
    p.bm_words = (int)(((d.pitch + 31) / 32 + 8 + 3) / 4 * 4);
    std::vector<uint32_t> bits((size_t)p.bm_words * nya, 0u);
    const float *lu = masks[0];
    for (int r = 0; r < nya; r++)
        for (int col = 0; col < nxa; col++)
            if (lu[(size_t)r * nxa + col] > 0.5f) {
                const int dc = col + d.xoff;
                bits[(size_t)r * p.bm_words + dc / 32] |= 1u << (dc % 32);
            }

    if (cudaMalloc(&p.rows, rows.size() * sizeof(RowCoef)) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(p.rows, rows.data(), rows.size() * sizeof(RowCoef), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return 1;
    if (cudaMalloc(&p.cor, cor.size() * sizeof(double)) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(p.cor, cor.data(), cor.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return 1;
    if (cudaMalloc(&p.bits, bits.size() * sizeof(uint32_t)) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(p.bits, bits.data(), bits.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return 1;
    const size_t fb = (size_t)d.pitch * nya * sizeof(double);
    for (int b = 0; b < 2; b++)
        for (int k = 0; k < 6; k++) {
            if (cudaMalloc(&p.buf[b][k], fb) != cudaSuccess) return 1;
            if (cudaMemsetAsync(p.buf[b][k], 0, fb, s) != cudaSuccess) return 1;
        }
    if (cudaMalloc(&p.d_uniform, (size_t)MINMAX_BLOCKS * 6 * sizeof(double)) != cudaSuccess) return 1;
    if (cudaMalloc(&p.d_flags, sizeof(unsigned)) != cudaSuccess) return 1;
    if (cudaMemsetAsync(p.d_flags, 0, sizeof(unsigned), s) != cudaSuccess) return 1;
    p.hrest = d_hrest;
    p.lu = d_lu;
    p.buffers_synced = false;
    if (set_smem()) return 1;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    p.nsm = nsm;
    int occ[2] = {1, 1};
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], k_substep<false, 3>, NL, Layout<false>::bytes) !=
            cudaSuccess || occ[0] < 1)
        occ[0] = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], k_substep<true, 3>, NL, Layout<true>::bytes) !=
            cudaSuccess || occ[1] < 1)
        occ[1] = 1;
    // one wave: strips x chunks <= SMs x resident CTAs, chunks as tall as
    // that allows; each chunk re-reads and recomputes three rows of warm-up,
    // so keep chunks at least 16 rows tall
    const int ny = d.ny_end - d.ny_start + 1;
    for (int v = 0; v < 2; v++) {
        int nchunks = std::max(1, nsm * occ[v] / p.nstrips);
        nchunks = std::min(nchunks, std::max(1, (ny + 15) / 16));
        p.chunk_rows[v] = (ny + nchunks - 1) / nchunks;
        p.nchunks[v] = (ny + p.chunk_rows[v] - 1) / p.chunk_rows[v];
    }
    return 0;
}

int dynamics(Plan &p, const Dom &d, const Consts &c, double tau, int nstep, double *state[6], double *acc[4],
             double *forc[6], cudaStream_t s)
{
    Forcing f;
    if (forcing_mode(p, d, c, forc, s, f)) return 1;
    if (!p.buffers_synced && sync_buffers(p, d, state, s)) return 1;
    if (cudaMemsetAsync(p.d_flags, 0, sizeof(unsigned), s) != cudaSuccess) return 1;
    const size_t fb = (size_t)d.pitch * d.nya() * sizeof(double);
    for (int k = 0; k < 4; k++)
        if (cudaMemsetAsync(acc[k], 0, fb, s) != cudaSuccess) return 1;   // vel_ssh.f90:479-482
    const int gen = (p.uni && f.uniform) ? 0 : 1;
    Params q = base_params(p, d, c, forc, f, gen);
    const double ti = tau / (double)nstep;
    q.two_ti = 2.0 * ti;
    q.gam = c.ts / 2.0 / (double)nstep;
    q.c4 = 1.0 / (double)(4 * nstep);
    for (int k = 0; k < 4; k++) q.acc[k] = acc[k];
    // substeps 1..nstep ping-pong between state[] and buf[0]; the state
    // after substep nstep (vel_ssh.f90:638-648) is then swapped into state[]
    for (int step = 1; step <= nstep; step++) {
        const bool odd = step & 1;
        for (int k = 0; k < 6; k++) {
            q.src[k] = odd ? state[k] : p.buf[0][k];
            q.dst[k] = odd ? p.buf[0][k] : state[k];
        }
        launch(p, q, gen, step == 1 ? 4 : 5, s);
        if (cudaGetLastError() != cudaSuccess) return 1;
    }
    if (nstep & 1)
        for (int k = 0; k < 6; k++) std::swap(state[k], p.buf[0][k]);
    // substeps nstep+1..2*nstep feed only the time means: state[] -> buf[0],
    // then buf[0] <-> buf[1]; the last one writes no state
    for (int k2 = 1; k2 <= nstep; k2++) {
        for (int k = 0; k < 6; k++) {
            q.src[k] = k2 == 1 ? state[k] : ((k2 & 1) ? p.buf[1][k] : p.buf[0][k]);
            q.dst[k] = (k2 & 1) ? p.buf[0][k] : p.buf[1][k];
        }
        launch(p, q, gen, k2 < nstep ? 5 : 2, s);
        if (cudaGetLastError() != cudaSuccess) return 1;
    }
    unsigned flags = 0;
    if (read_flags(p, s, &flags)) return 1;
    p.last_flags = flags;
    return 0;
}

int run_substeps(Plan &p, const Dom &d, const Consts &c, int nsub, double dt, const double *rhs_scale,
                 double *state[6], double *forc[6], cudaStream_t s)
{
    Forcing f;
    if (forcing_mode(p, d, c, forc, s, f)) return 1;
    if (!p.buffers_synced && sync_buffers(p, d, state, s)) return 1;
    if (cudaMemsetAsync(p.d_flags, 0, sizeof(unsigned), s) != cudaSuccess) return 1;
    const int gen = (p.uni && f.uniform) ? 0 : 1;
    Params q = base_params(p, d, c, forc, f, gen);
    q.two_ti = 2.0 * dt;
    q.gam = c.ts / 2.0;   // nstep = 1
    q.c4 = 0.25;
    for (int k = 0; k < 4; k++) q.acc[k] = nullptr;
    for (int step = 0; step < nsub; step++) {
        for (int k = 0; k < 6; k++) {
            q.src[k] = (step & 1) ? p.buf[0][k] : state[k];
            q.dst[k] = (step & 1) ? state[k] : p.buf[0][k];
        }
        q.rhs_scale = rhs_scale ? rhs_scale[step] : 1.0;
        launch(p, q, gen, 3, s);
        if (cudaGetLastError() != cudaSuccess) return 1;
    }
    if (nsub & 1)
        for (int k = 0; k < 6; k++) std::swap(state[k], p.buf[0][k]);
    unsigned flags = 0;
    if (read_flags(p, s, &flags)) return 1;
    p.last_flags = flags;
    return 0;
}

void free_plan(Plan &p)
{
    cudaFree(p.rows);
    cudaFree(p.cor);
    cudaFree(p.bits);
    for (auto &b : p.buf)
        for (auto &x : b) cudaFree(x);
    cudaFree(p.d_uniform);
    cudaFree(p.d_flags);
    p = Plan{};
}

}  // namespace fused
}  // namespace inmsom
