// Fused streaming kernel of the barotropic step (see fused.h).
//
// Work decomposition.  A CTA is one warp.  Lane l owns the two adjacent
// device columns k0 = g0+2+2l and k0+1 of a 64-column strip starting at
// device column g0+2 (g0 = 62*strip, even); strip columns 1..62 are written,
// so strips overlap by two columns.  The CTA marches down a chunk of output
// rows [r0, r1).  Iteration j computes, for its columns,
//   stage 1, row j   : u/v-point depths of the current level and the
//                      transports U = u*hu, V = v*hv;
//   stage 2, row j-1 : new SSH (continuity), advective fluxes on T and h
//                      points, Coriolis-plus-metric-vorticity products,
//                      tension and shear stresses times viscosity and depth;
//   stage 3u, row j-1: u momentum, SSH update, their time-mean sums,
//                      Robert-Asselin filter and time shift, stores;
//   stage 3v, row j-2: the same for v (it needs stage 2 of the row above).
// A value a stage needs from the neighbouring column is the other column
// of the same lane or comes from the neighbouring lane by a warp shuffle;
// values of earlier rows of the same column stay in registers, in three
// instances of each per-row struct that the three-fold unrolled row loop
// renames instead of copying.  There is no CTA-wide barrier, and the
// per-column work is branch-free (predicated stores) except for warp-wide
// skips of rows without ocean.
//
// Input rows j-2..j+1 of the input fields (a 68-column segment per field
// and row, 16-byte aligned), the row's coefficients and the row's T-mask
// bits sit in a ring of RING shared-memory slots.  Lane 0 refills the slot
// of row j-2 with row j-2+RING by 1-D bulk TMA copies (cp.async.bulk, no
// multicast) completing on that slot's mbarrier.  Every wait is bounded: on
// timeout the CTA sets a status bit, drains its own copies (bounded) and
// returns.
#include "fused.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace inmsom {
namespace fused {

namespace {

constexpr int NL = 32;            // lanes = threads per CTA
constexpr int NCOL = 2 * NL;      // strip columns
constexpr int OUTW = NCOL - 2;    // written columns per strip
constexpr int SEG = NCOL + 4;     // ring segment: strip columns -2 .. 65
constexpr int RING = 6;           // ring slots (4 rows in use + 2 in flight)
constexpr int CTAS_PER_SM = 7;
constexpr int COEF_D = (int)(sizeof(RowCoef) / sizeof(double));
constexpr unsigned WAIT_LIMIT = 1u << 20;

// state order, as the *_e arguments: u, up, v, vp, ssh, sshp
enum { S_U, S_UP, S_V, S_VP, S_SSH, S_SSHP };
// ring fields
enum { R_U, R_V, R_SSH, R_UP, R_VP, R_SSHP, R_H, R_RX, R_RY, R_NBASE, R_MU = R_NBASE, R_RD, R_WF, R_N2D };

struct Params {
    const double *src[6];
    double *dst[6];
    const double *H, *rhsx, *rhsy, *mu, *rdis, *wflux;
    double *acc[4];
    const uint32_t *bits;
    const RowCoef *rows;
    RowCoef rc;            // row-invariant coefficients (used when !ROWVAR)
    long long pitch;
    int bm_words;
    int chunk_rows;
    int r_first, r_last;   // interior device rows
    int c_first, c_last;   // interior device columns
    double two_ti, gam, c4, rhs_scale, mu0, rd0, wq0, inv_rho;
    int acc_mode;          // 0 none, 1 write, 2 accumulate
    int write_state;
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

template <bool F2D>
struct Layout {
    static constexpr int NF = F2D ? R_N2D : R_NBASE;
    static constexpr int SLOT_D = NF * SEG + COEF_D + 4;   // doubles per slot
    static constexpr size_t bytes = (size_t)RING * SLOT_D * sizeof(double) + RING * sizeof(uint64_t);
    static constexpr uint32_t row_tx = (uint32_t)((NF * SEG + COEF_D + 4) * sizeof(double));
};

__device__ __forceinline__ double sel(int m, double x) { return m ? x : 0.0; }

// 1 / (number of ocean T points) for the mask-weighted depth averages
__device__ __forceinline__ double rcount(int n)
{
    return n == 4 ? 0.25 : (n == 3 ? 1.0 / 3.0 : (n == 2 ? 0.5 : (n == 1 ? 1.0 : 0.0)));
}

#define SHFL_UP(x) __shfl_up_sync(0xffffffffu, (x), 1)
#define SHFL_DN(x) __shfl_down_sync(0xffffffffu, (x), 1)

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

// per-row values carried between the stages of the row pipeline
struct S1 {          // stage 1 of a row: transports and current-level depths
    double U0, U1, V0, V1;   // U = u*hu at k0, k0+1; V = v*hv
    double Ul, Vr;           // U(k0-1), V(k0+2) from the neighbouring lanes
    double hu0, hu1, hv0, hv1;
};
struct HQ {          // H + ssh of a row at k0, k0+1, k0+2
    double a, b, c;
};
struct S2 {          // stage 2 of a row
    double sn0, sn1;         // new SSH
    double FY0, FY1, QU0, QU1, SS0, SS1;
    double GX0, GX1, GXl, GY0, GY1, QV0, QV1, QVl, ST0, ST1, SSl;
};

template <bool F2D, bool ROWVAR>
__global__ void __launch_bounds__(NL, CTAS_PER_SM) k_substep(const __grid_constant__ Params p)
{
    using L = Layout<F2D>;
    constexpr int NF = L::NF;
    extern __shared__ __align__(128) double smem[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + RING * L::SLOT_D);

    const int l = threadIdx.x;
    const int g0 = blockIdx.x * OUTW;          // device column of segment offset 0
    const int k0 = g0 + 2 + 2 * l;             // this lane's columns k0, k0+1
    const int r0 = p.r_first + blockIdx.y * p.chunk_rows;
    const int r1 = min(r0 + p.chunk_rows, p.r_last + 1);   // exclusive
    if (r0 >= r1) return;
    const int row_lo = r0 - 2, row_hi = r1 + 1;             // rows kept in the ring
    const int wbase = (g0 >> 7) << 2;                       // first mask word of the window
    const int bsh = k0 - wbase * 32;                        // bit of k0 in the window
    const int po = 2 * l + 2;                               // segment offset of k0

    auto slotp = [&](int s) { return smem + (size_t)s * L::SLOT_D; };
    auto slot_of = [&](int row) { return (row - row_lo) % RING; };
    auto issue = [&](int row) {
        const int s = slot_of(row);
        double *d = slotp(s);
        uint64_t *bar = &mbar[s];
        mbar_expect_tx(bar, L::row_tx);
        const long long off = (long long)row * p.pitch + g0;
        const uint32_t nb = SEG * sizeof(double);
        bulk_load(d + R_U * SEG, p.src[S_U] + off, nb, bar);
        bulk_load(d + R_V * SEG, p.src[S_V] + off, nb, bar);
        bulk_load(d + R_SSH * SEG, p.src[S_SSH] + off, nb, bar);
        bulk_load(d + R_UP * SEG, p.src[S_UP] + off, nb, bar);
        bulk_load(d + R_VP * SEG, p.src[S_VP] + off, nb, bar);
        bulk_load(d + R_SSHP * SEG, p.src[S_SSHP] + off, nb, bar);
        bulk_load(d + R_H * SEG, p.H + off, nb, bar);
        bulk_load(d + R_RX * SEG, p.rhsx + off, nb, bar);
        bulk_load(d + R_RY * SEG, p.rhsy + off, nb, bar);
        if constexpr (F2D) {
            bulk_load(d + R_MU * SEG, p.mu + off, nb, bar);
            bulk_load(d + R_RD * SEG, p.rdis + off, nb, bar);
            bulk_load(d + R_WF * SEG, p.wflux + off, nb, bar);
        }
        bulk_load(d + NF * SEG, p.rows + row, sizeof(RowCoef), bar);
        bulk_load(d + NF * SEG + COEF_D, p.bits + (size_t)row * p.bm_words + wbase, 32, bar);
    };
    // field f of a slot: own pair (k0, k0+1), left neighbour (k0-1), right (k0+2)
    auto pair = [&](int s, int f) {
        return *reinterpret_cast<const double2 *>(slotp(s) + f * SEG + po);
    };
    auto leftv = [&](int s, int f) { return slotp(s)[f * SEG + po - 1]; };
    auto rightv = [&](int s, int f) { return slotp(s)[f * SEG + po + 2]; };
    auto coef = [&](int s) { return reinterpret_cast<const RowCoef *>(slotp(s) + NF * SEG); };
    auto mask3 = [&](int s) -> uint32_t {   // bits: lu(k0), lu(k0+1), lu(k0+2)
        const uint32_t *w = reinterpret_cast<const uint32_t *>(slotp(s) + NF * SEG + COEF_D);
        return __funnelshift_r(w[bsh >> 5], w[(bsh >> 5) + 1], bsh & 31) & 7u;
    };
#define CF(s, x) (ROWVAR ? coef(s)->x : p.rc.x)

    if (l == 0) {
        for (int s = 0; s < RING; s++) mbar_init(&mbar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    int issued = row_lo - 1;
    if (l == 0)
        for (int row = row_lo; row < row_lo + RING && row <= row_hi; row++) issue(row), issued = row;

    const bool out0 = l >= 1 && k0 >= p.c_first && k0 <= p.c_last;
    const bool out1 = l <= NL - 2 && k0 + 1 >= p.c_first && k0 + 1 <= p.c_last;
    const double gam = p.gam, two_ti = p.two_ti, rs = p.rhs_scale;

    // T-mask bits, 3 per row: row j+1 in bits 0-2, j in 3-5, j-1 in 6-8, j-2 in 9-11
    uint32_t mk = 0;
    uint32_t bad = 0;   // guard: a new value out of range or NaN
    int waited = row_lo - 1;
    bool ok = true;

    // One row step of the pipeline, for iteration j (see the file comment):
    //   stage 1 row j      -> s1n (and H+ssh of row j+1 -> hqn)
    //   stage 2 row j-1    -> s2n, from s1c = S1(j-1), s1p = S1(j-2), s1n,
    //                         hqp = H+ssh(j-1), hqc = H+ssh(j)
    //   stage 3u row j-1   u momentum and the SSH update, from s2n, s2o
    //   stage 3v row j-2   v momentum, from s2o = S2(j-2), s2n, s1p
    auto step = [&](const int j, S1 &s1n, const S1 &s1c, const S1 &s1p, HQ &hqn, const HQ &hqc,
                    const HQ &hqp, S2 &s2n, const S2 &s2o) {
        // --- rows up to j+1 must have landed ------------------------------
        const int need = min(j + 1, row_hi);
        while (waited < need && ok) {
            const int row = waited + 1;
            const uint32_t par = (uint32_t)(((row - row_lo) / RING) & 1);
            if (!mbar_wait(&mbar[slot_of(row)], par)) { ok = false; break; }
            waited = row;
            mk = (mk << 3) | mask3(slot_of(row));
        }
        if (j + 1 > row_hi) mk <<= 3;   // keep the row alignment of mk
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) return;
        const int s_m2 = slot_of(j - 2), s_m1 = slot_of(j - 1), s_0 = slot_of(j), s_p1 = slot_of(j + 1);

        // ---------------- stage 1: row j ---------------------------------
        if (j <= r1) {
            const uint32_t mj = (mk >> 3) & 7u, mn = mk & 7u;
            {   // H + ssh of row j+1 at k0, k0+1, k0+2
                const double2 h = pair(s_p1, R_H), e = pair(s_p1, R_SSH);
                hqn.a = h.x + e.x;
                hqn.b = h.y + e.y;
                hqn.c = rightv(s_p1, R_H) + rightv(s_p1, R_SSH);
            }
            const double ku = CF(s_0, ku), ku2 = CF(s_0, ku2), wv0 = CF(s_0, wv0), wv1 = CF(s_0, wv1);
            const double2 u = pair(s_0, R_U), v = pair(s_0, R_V);
            const double hq0[3] = {hqc.a, hqc.b, hqc.c}, hq1[2] = {hqn.a, hqn.b};
            double hu[2], hv[2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                // Function/depth.f90:127-139 mask-weighted averages to u and v points
                const int a = (mj >> e) & 1, b = (mj >> (e + 1)) & 1, c = (mn >> e) & 1;
                hu[e] = (sel(a, hq0[e]) + sel(b, hq0[e + 1])) * (a & b ? ku2 : (a | b ? ku : 0.0));
                hv[e] = (sel(a, hq0[e] * wv0) + sel(c, hq1[e] * wv1)) * (a & c ? 0.5 : (a | c ? 1.0 : 0.0));
            }
            s1n.hu0 = hu[0]; s1n.hu1 = hu[1]; s1n.hv0 = hv[0]; s1n.hv1 = hv[1];
            s1n.U0 = u.x * hu[0];
            s1n.U1 = u.y * hu[1];
            s1n.V0 = v.x * hv[0];
            s1n.V1 = v.y * hv[1];
        }
        s1n.Ul = SHFL_UP(s1n.U1);
        s1n.Vr = SHFL_DN(s1n.V0);

        // ---------------- stage 2: row rho = j-1 -------------------------
        const bool st2 = j >= r0 && j <= r1 + 1;
        double FX0 = 0, FX1 = 0, FXr = 0, ST_r = 0, SNr = 0;
        if (st2) {
            const uint32_t mr = (mk >> 6) & 7u, mu_ = (mk >> 3) & 7u;   // rows rho, rho+1
            const int sr = s_m1, sm = s_m2, su = s_0;
            const double2 u_r = pair(sr, R_U), u_u = pair(su, R_U), v_r = pair(sr, R_V);
            const double2 v_m = pair(sm, R_V), up_r = pair(sr, R_UP), up_u = pair(su, R_UP);
            const double2 vp_r = pair(sr, R_VP), vp_m = pair(sm, R_VP), sp_r = pair(sr, R_SSHP);
            const double ur[3] = {leftv(sr, R_U), u_r.x, u_r.y};     // u at k0-1, k0, k0+1
            const double vr[3] = {v_r.x, v_r.y, rightv(sr, R_V)};    // v at k0, k0+1, k0+2
            const double vpr[3] = {vp_r.x, vp_r.y, rightv(sr, R_VP)};
            const double upr[3] = {leftv(sr, R_UP), up_r.x, up_r.y};
            const double uu[2] = {u_u.x, u_u.y}, vm[2] = {v_m.x, v_m.y};
            const double upu[2] = {up_u.x, up_u.y}, vpm[2] = {vp_m.x, vp_m.y};
            const double spr[2] = {sp_r.x, sp_r.y};
            const double Ur[3] = {s1c.Ul, s1c.U0, s1c.U1};           // U(rho) at k0-1, k0, k0+1
            const double Vr[3] = {s1c.V0, s1c.V1, s1c.Vr};           // V(rho) at k0, k0+1, k0+2
            const double Un[2] = {s1n.U0, s1n.U1};                   // U(rho+1)
            const double Vm[2] = {s1p.V0, s1p.V1};                   // V(rho-1)
            const double hqr[3] = {hqp.a, hqp.b, hqp.c}, hqu[3] = {hqc.a, hqc.b, hqc.c};
            double mur[3] = {p.mu0, p.mu0, p.mu0}, muu[3] = {p.mu0, p.mu0, p.mu0}, wf[2] = {p.wq0, p.wq0};
            if constexpr (F2D) {
                const double2 a = pair(sr, R_MU), b = pair(su, R_MU), w = pair(sr, R_WF);
                mur[0] = a.x; mur[1] = a.y; mur[2] = rightv(sr, R_MU);
                muu[0] = b.x; muu[1] = b.y; muu[2] = rightv(su, R_MU);
                wf[0] = w.x * p.inv_rho; wf[1] = w.y * p.inv_rho;
            }
            const double c_u = CF(sr, c_u), c_v0 = CF(sr, c_v0), c_v1 = CF(sr, c_v1);
            const double fx = CF(sr, fx), fy = CF(sr, fy), gx0 = CF(sr, gx0), gx1 = CF(sr, gx1);
            const double gy0 = CF(sr, gy0), gy1 = CF(sr, gy1), wh0 = CF(sr, wh0), wh1 = CF(sr, wh1);
            const double t1 = CF(sr, t1), t2 = CF(sr, t2), t3 = CF(sr, t3);
            const double s1 = CF(sr, s1), s2 = CF(sr, s2), s3 = CF(sr, s3);
            const double cor = coef(sr)->cor;
            double sn[2], FX[2], FY[2], GX[2], GY[2], QU[2], QV[2], ST[2], SS[2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int lc = (mr >> e) & 1, lr = (mr >> (e + 1)) & 1;
                const int lu = (mu_ >> e) & 1, lur = (mu_ >> (e + 1)) & 1;
                const int luu = lc & lr & lu & lur;
                // vel_ssh.f90:491-494 continuity over 2*tau_inner
                const double div = (Ur[e + 1] - Ur[e]) * c_u + Vr[e] * c_v0 - Vm[e] * c_v1;
                sn[e] = sel(lc, spr[e] + two_ti * (wf[e] - div));
                // vel_ssh.f90:63-73, :88-98 advective fluxes on T and h faces
                FX[e] = (Ur[e] + Ur[e + 1]) * (ur[e] + ur[e + 1]) * fx;
                FY[e] = sel(luu, (Vr[e] + Vr[e + 1]) * (ur[e + 1] + uu[e]) * fy);
                GX[e] = (Ur[e + 1] * gx0 + Un[e] * gx1) * (vr[e] + vr[e + 1]);
                GY[e] = (Vm[e] * gy0 + Vr[e] * gy1) * (vm[e] + vr[e]);
                // depth.f90:141-147 depth on the h point
                const double sa = sel(lc, hqr[e]) + sel(lr, hqr[e + 1]);
                const double sb = sel(lu, hqu[e]) + sel(lur, hqu[e + 1]);
                const double hh = (sa * wh0 + sb * wh1) * rcount(lc + lr + lu + lur);
                // vel_ssh.f90:35-37 metric vorticity (zero on uniform grids) + Coriolis
                double vort = 0.0;
                if (!p.vort_zero)
                    vort = sel(luu, (vr[e + 1] - vr[e]) * CF(sr, vt0) - uu[e] * CF(sr, vt1) + ur[e + 1] * CF(sr, vt2));
                const double Wh = hh * (cor + vort);
                QU[e] = Wh * (vr[e] + vr[e + 1]);
                QV[e] = Wh * (ur[e + 1] + uu[e]);
                // mixing.f90:134-148 stresses from the previous level
                const double str_t = sel(lc, t1 * (upr[e + 1] - upr[e]) - (t2 * vpr[e] - t3 * vpm[e]));
                const double str_s = sel(luu, s1 * upu[e] - s2 * upr[e + 1] + s3 * (vpr[e + 1] - vpr[e]));
                double mu_h = p.mu0;
                if constexpr (F2D) mu_h = (mur[e] + mur[e + 1] + muu[e] + muu[e + 1]) * 0.25;
                ST[e] = mur[e] * hqr[e] * str_t;
                SS[e] = mu_h * hh * str_s;
            }
            s2n.sn0 = sn[0]; s2n.sn1 = sn[1];
            s2n.FY0 = FY[0]; s2n.FY1 = FY[1]; s2n.QU0 = QU[0]; s2n.QU1 = QU[1];
            s2n.SS0 = SS[0]; s2n.SS1 = SS[1]; s2n.GX0 = GX[0]; s2n.GX1 = GX[1];
            s2n.GY0 = GY[0]; s2n.GY1 = GY[1]; s2n.QV0 = QV[0]; s2n.QV1 = QV[1];
            s2n.ST0 = ST[0]; s2n.ST1 = ST[1];
            FX0 = FX[0]; FX1 = FX[1];
        }
        FXr = SHFL_DN(FX0);
        ST_r = SHFL_DN(s2n.ST0);
        SNr = SHFL_DN(s2n.sn0);
        s2n.GXl = SHFL_UP(s2n.GX1);
        s2n.QVl = SHFL_UP(s2n.QV1);
        s2n.SSl = SHFL_UP(s2n.SS1);

        // ---------------- stage 3u: row rho = j-1 (u and SSH) -----------
        const int rho = j - 1;
        const uint32_t mr = (mk >> 6) & 7u;
        const bool wr3u = j >= r0 + 1 && j <= r1 && __any_sync(0xffffffffu, (out0 || out1) && (mr & 3u));
        if (wr3u) {
            const int sr = s_m1;
            const double2 e_r = pair(sr, R_SSH), sp_r = pair(sr, R_SSHP), h_r = pair(sr, R_H);
            const double e3[3] = {e_r.x, e_r.y, rightv(sr, R_SSH)};
            const double sp3[3] = {sp_r.x, sp_r.y, rightv(sr, R_SSHP)};
            const double h3[3] = {h_r.x, h_r.y, rightv(sr, R_H)};
            const double2 u_r = pair(sr, R_U), up_r = pair(sr, R_UP), rx = pair(sr, R_RX);
            const double u0[2] = {u_r.x, u_r.y}, up0[2] = {up_r.x, up_r.y}, rxv[2] = {rx.x, rx.y};
            const double sn3[3] = {s2n.sn0, s2n.sn1, SNr};
            const double FX3[3] = {FX0, FX1, FXr};
            const double ST3[3] = {s2n.ST0, s2n.ST1, ST_r};
            const double FYd[2] = {s2n.FY0 - s2o.FY0, s2n.FY1 - s2o.FY1};
            const double QUs[2] = {s2n.QU0 + s2o.QU0, s2n.QU1 + s2o.QU1};
            const double SSn[2] = {s2n.SS0, s2n.SS1}, SSo[2] = {s2o.SS0, s2o.SS1};
            const double hu_c[2] = {s1c.hu0, s1c.hu1};
            double rd3[3] = {p.rd0, p.rd0, p.rd0};
            if constexpr (F2D) {
                const double2 a = pair(sr, R_RD);
                rd3[0] = a.x; rd3[1] = a.y; rd3[2] = rightv(sr, R_RD);
            }
            const double ku2 = CF(sr, ku2), gdyh = CF(sr, gdyh), dux = CF(sr, dux);
            const double dus0 = CF(sr, dus0), dus1 = CF(sr, dus1), au = CF(sr, au);
            const double cu = two_ti * CF(sr, rau);
            const long long rowb = (long long)rho * p.pitch + k0;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const bool oute = e == 0 ? out0 : out1;
                const int lc = (mr >> e) & 1, lr = (mr >> (e + 1)) & 1;
                const bool wu = oute && (lc & lr), wt = oute && lc;
                // vel_ssh.f90:536-551
                const double hu = hu_c[e];
                const double hup = ((h3[e] + sp3[e]) + (h3[e + 1] + sp3[e + 1])) * ku2;
                const double hun = ((h3[e] + sn3[e]) + (h3[e + 1] + sn3[e + 1])) * ku2;
                const double slx = -(e3[e + 1] - e3[e]) * gdyh * hu;
                const double slxn = -(sn3[e + 1] - sn3[e]) * gdyh * hun;
                const double adv = -((FX3[e + 1] - FX3[e]) + FYd[e]);
                const double dif = (ST3[e + 1] - ST3[e]) * dux + (SSn[e] * dus0 - SSo[e] * dus1);
                const double rd = F2D ? (rd3[e] + rd3[e + 1]) * 0.5 : p.rd0;
                const double grx = rxv[e] * rs + slx + dif + adv - rd * up0[e] * au * hu + QUs[e] * 0.25;
                const double un = (up0[e] * hup + grx * cu) * rcp_nr(hun);
                bad |= (uint32_t)(wu && !(un < 100.0 && un > -100.0));
                bad |= (uint32_t)(wt && !(sn3[e] < 10.0 && sn3[e] > -10.0));
                const long long idx = rowb + e;
                if (p.acc_mode && wu) {
                    double a = (u0[e] * hu + un * hun) * p.c4, b = (slx + slxn) * p.c4;
                    if (p.acc_mode == 2) { a += p.acc[0][idx]; b += p.acc[2][idx]; }
                    p.acc[0][idx] = a;
                    p.acc[2][idx] = b;
                }
                if (p.write_state) {
                    if (wu) {
                        p.dst[S_UP][idx] = u0[e] + gam * (un - 2.0 * u0[e] + up0[e]);
                        p.dst[S_U][idx] = un;
                    }
                    if (wt) {   // vel_ssh.f90:593-596
                        p.dst[S_SSHP][idx] = e3[e] + gam * (sn3[e] - 2.0 * e3[e] + sp3[e]);
                        p.dst[S_SSH][idx] = sn3[e];
                    }
                }
            }
        }

        // ---------------- stage 3v: row R = j-2 (v) ----------------------
        const int R = j - 2;
        const uint32_t mR = (mk >> 9) & 7u, mU = (mk >> 6) & 7u;   // rows R, R+1
        const bool wr3v = j >= r0 + 2 && j <= r1 + 1 &&
                          __any_sync(0xffffffffu, (out0 && (mR & mU & 1u)) || (out1 && (mR & mU & 2u)));
        if (wr3v) {
            const int sR = s_m2, sU = s_m1;
            const double2 eR = pair(sR, R_SSH), spR = pair(sR, R_SSHP), hR = pair(sR, R_H);
            const double2 eU = pair(sU, R_SSH), spU = pair(sU, R_SSHP), hU = pair(sU, R_H);
            const double2 v_R = pair(sR, R_V), vp_R = pair(sR, R_VP), ry = pair(sR, R_RY);
            const double e0[2] = {eR.x, eR.y}, sp0[2] = {spR.x, spR.y}, h0[2] = {hR.x, hR.y};
            const double e1[2] = {eU.x, eU.y}, sp1[2] = {spU.x, spU.y}, h1[2] = {hU.x, hU.y};
            const double v0[2] = {v_R.x, v_R.y}, vp0[2] = {vp_R.x, vp_R.y}, ryv[2] = {ry.x, ry.y};
            const double sn0[2] = {s2o.sn0, s2o.sn1}, sn1[2] = {s2n.sn0, s2n.sn1};
            const double GX3[3] = {s2o.GXl, s2o.GX0, s2o.GX1};
            const double QV3[3] = {s2o.QVl, s2o.QV0, s2o.QV1};
            const double SS3[3] = {s2o.SSl, s2o.SS0, s2o.SS1};
            const double GYd[2] = {s2n.GY0 - s2o.GY0, s2n.GY1 - s2o.GY1};
            const double STo[2] = {s2o.ST0, s2o.ST1}, STn[2] = {s2n.ST0, s2n.ST1};
            const double hv_c[2] = {s1p.hv0, s1p.hv1};
            double rdR[2] = {p.rd0, p.rd0}, rdU[2] = {p.rd0, p.rd0};
            if constexpr (F2D) {
                const double2 a = pair(sR, R_RD), b = pair(sU, R_RD);
                rdR[0] = a.x; rdR[1] = a.y; rdU[0] = b.x; rdU[1] = b.y;
            }
            const double wv0 = CF(sR, wv0), wv1 = CF(sR, wv1), gdxh = CF(sR, gdxh);
            const double dvt0 = CF(sR, dvt0), dvt1 = CF(sR, dvt1), dvs = CF(sR, dvs), av = CF(sR, av);
            const double cv = two_ti * CF(sR, rav);
            const long long rowb = (long long)R * p.pitch + k0;
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const bool oute = e == 0 ? out0 : out1;
                const bool wv = oute && ((mR >> e) & (mU >> e) & 1u);
                // vel_ssh.f90:554-569
                const double hv = hv_c[e];
                const double hvp = ((h0[e] + sp0[e]) * wv0 + (h1[e] + sp1[e]) * wv1) * 0.5;
                const double hvn = ((h0[e] + sn0[e]) * wv0 + (h1[e] + sn1[e]) * wv1) * 0.5;
                const double sly = -(e1[e] - e0[e]) * gdxh * hv;
                const double slyn = -(sn1[e] - sn0[e]) * gdxh * hvn;
                const double adv = -((GX3[e + 1] - GX3[e]) + GYd[e]);
                const double dif = -(STn[e] * dvt1 - STo[e] * dvt0) + (SS3[e + 1] - SS3[e]) * dvs;
                const double rd = F2D ? (rdR[e] + rdU[e]) * 0.5 : p.rd0;
                const double gry = ryv[e] * rs + sly + dif + adv - rd * vp0[e] * av * hv
                                   - (QV3[e + 1] + QV3[e]) * 0.25;
                const double vn = (vp0[e] * hvp + gry * cv) * rcp_nr(hvn);
                bad |= (uint32_t)(wv && !(vn < 100.0 && vn > -100.0));
                const long long idx = rowb + e;
                if (p.acc_mode && wv) {
                    double a = (v0[e] * hv + vn * hvn) * p.c4, b = (sly + slyn) * p.c4;
                    if (p.acc_mode == 2) { a += p.acc[1][idx]; b += p.acc[3][idx]; }
                    p.acc[1][idx] = a;
                    p.acc[3][idx] = b;
                }
                if (p.write_state && wv) {
                    p.dst[S_VP][idx] = v0[e] + gam * (vn - 2.0 * v0[e] + vp0[e]);
                    p.dst[S_V][idx] = vn;
                }
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

    // three instances of each carried struct, renamed (not copied) by the
    // three-fold unrolled loop
    S1 A{}, B{}, C{};
    HQ HA{}, HB{}, HC{};
    S2 X{}, Y{}, Z{};
    {   // H + ssh of row r0-1 (the stage-1 "current" row of the first step)
        const int need = row_lo + 1;
        while (waited < need && ok) {
            const int row = waited + 1;
            if (!mbar_wait(&mbar[slot_of(row)], (uint32_t)(((row - row_lo) / RING) & 1))) { ok = false; break; }
            waited = row;
            mk = (mk << 3) | mask3(slot_of(row));
        }
        ok = __all_sync(0xffffffffu, ok);
        if (ok) {
            const int s = slot_of(r0 - 1);
            const double2 h = pair(s, R_H), e = pair(s, R_SSH);
            HC.a = h.x + e.x;
            HC.b = h.y + e.y;
            HC.c = rightv(s, R_H) + rightv(s, R_SSH);
        }
    }
    // mk now holds rows r0-2 (bits 3-5) and r0-1 (bits 0-2); the first step
    // pushes row r0 so that row j+1 = r0 sits in bits 0-2
    for (int j = r0 - 1; j <= r1 + 1 && ok; j += 3) {
        step(j, A, C, B, HA, HC, HB, X, Z);
        step(j + 1, B, A, C, HB, HA, HC, Y, X);
        step(j + 2, C, B, A, HC, HB, HA, Z, Y);
    }
#undef CF
    if (__any_sync(0xffffffffu, bad != 0) && l == 0) atomicOr(p.flags, FLAG_GUARD);
    if (!ok && l == 0) {
        atomicOr(p.flags, FLAG_TIMEOUT);
        // drain this CTA's copies still in flight (bounded) before exiting
        for (int row = max(waited + 1, row_lo); row <= issued; row++)
            (void)mbar_wait(&mbar[slot_of(row)], (uint32_t)(((row - row_lo) / RING) & 1));
    }
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

Params base_params(const Plan &p, const Dom &d, const Consts &c, double *forc[6], const Forcing &f)
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
    q.rc = p.rc;
    q.pitch = d.pitch;
    q.bm_words = p.bm_words;
    q.chunk_rows = p.chunk_rows;
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
    return q;
}

template <bool F2D, bool RV>
void launch_t(const Plan &p, const Params &q, cudaStream_t s)
{
    dim3 grid(p.nstrips, p.nchunks);
    k_substep<F2D, RV><<<grid, NL, Layout<F2D>::bytes, s>>>(q);
}

void launch(const Plan &p, const Params &q, bool f2d, cudaStream_t s)
{
    if (f2d) {
        if (p.rowvar) launch_t<true, true>(p, q, s); else launch_t<true, false>(p, q, s);
    } else {
        if (p.rowvar) launch_t<false, true>(p, q, s); else launch_t<false, false>(p, q, s);
    }
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

template <bool F2D, bool RV>
int set_smem()
{
    return cudaFuncSetAttribute(k_substep<F2D, RV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)Layout<F2D>::bytes) != cudaSuccess;
}

}  // namespace

// ===========================================================================
Plan make_plan(const inmsom_bounds &b)
{
    Plan p;
    p.ncol = NCOL;
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
    // rows identical except for cor -> the coefficients go in the kernel
    // parameters and only cor is read per row
    p.rowvar = false;
    for (int r = 1; r < nya && !p.rowvar; r++) {
        RowCoef a = rows[r], b = rows[0];
        a.cor = b.cor = 0.0;
        p.rowvar = std::memcmp(&a, &b, sizeof(RowCoef)) != 0;
    }
    p.rc = rows[d.ny_start - d.bnd_y1];
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
    if (set_smem<false, false>() || set_smem<false, true>() || set_smem<true, false>() || set_smem<true, true>())
        return 1;
    int dev = 0, nsm = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_substep<false, false>, NL,
                                                      Layout<false>::bytes) != cudaSuccess || occ < 1)
        occ = 1;
    p.nsm = nsm;
    // one wave: strips x chunks <= SMs x resident CTAs, chunks as tall as
    // that allows; each chunk re-reads and recomputes three rows of warm-up,
    // so keep chunks at least 16 rows tall
    const int ny = d.ny_end - d.ny_start + 1;
    const int slots = nsm * occ;
    int nchunks = std::max(1, slots / p.nstrips);
    nchunks = std::min(nchunks, std::max(1, (ny + 15) / 16));
    p.chunk_rows = (ny + nchunks - 1) / nchunks;
    p.nchunks = (ny + p.chunk_rows - 1) / p.chunk_rows;
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
    Params q = base_params(p, d, c, forc, f);
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
        q.acc_mode = step == 1 ? 1 : 2;
        q.write_state = 1;
        launch(p, q, !f.uniform, s);
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
        q.acc_mode = 2;
        q.write_state = k2 < nstep ? 1 : 0;
        launch(p, q, !f.uniform, s);
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
    Params q = base_params(p, d, c, forc, f);
    q.two_ti = 2.0 * dt;
    q.gam = c.ts / 2.0;   // nstep = 1
    q.c4 = 0.25;
    q.acc_mode = 0;
    q.write_state = 1;
    for (int k = 0; k < 4; k++) q.acc[k] = nullptr;
    for (int step = 0; step < nsub; step++) {
        for (int k = 0; k < 6; k++) {
            q.src[k] = (step & 1) ? p.buf[0][k] : state[k];
            q.dst[k] = (step & 1) ? state[k] : p.buf[0][k];
        }
        q.rhs_scale = rhs_scale ? rhs_scale[step] : 1.0;
        launch(p, q, !f.uniform, s);
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
    cudaFree(p.bits);
    for (auto &b : p.buf)
        for (auto &x : b) cudaFree(x);
    cudaFree(p.d_uniform);
    cudaFree(p.d_flags);
    p = Plan{};
}

}  // namespace fused
}  // namespace inmsom
