// Fused streaming kernel of the barotropic step (see fused.h).
//
// Work decomposition.  A CTA of W threads owns device columns
// [cs, cs+W) (thread t <-> column cs+t) and writes the W-2 columns of
// threads 1..W-2; strips overlap by two columns.  It marches down a chunk of
// output rows [r0, r1).  Iteration j computes, for the CTA's columns,
//   stage 1, row j   : u/v-point depths of the current level and the
//                      transports U = u*hu, V = v*hv;
//   stage 2, row j-1 : new SSH (continuity), advective fluxes on T and h
//                      points, Coriolis-plus-metric-vorticity products,
//                      tension and shear stresses times viscosity and depth;
//   stage 3, row j-2 : u and v momentum, time-mean sums, Robert-Asselin
//                      filter and time shift, stores.
// Values a stage needs from the neighbouring column pass through a
// double-buffered shared exchange row; values it needs from earlier rows of
// its own column stay in registers.  So one __syncthreads per row suffices.
//
// Input rows j-2..j+1 of the ten input fields sit in a ring of RING
// shared-memory slots; thread 0 refills the slot of row j-2 with row
// j-2+RING by 1-D bulk TMA copies (cp.async.bulk, no multicast) completing
// on that slot's mbarrier.  Every wait is bounded: on timeout the CTA sets
// a status bit, drains its own copies (bounded) and returns.
#include "fused.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace inmsom {
namespace fused {

namespace {

constexpr int W = 128;          // threads per CTA = columns per strip
constexpr int SEG = W + 2;      // columns per ring row segment: cs-1 .. cs+W
constexpr int RING = 6;         // ring slots (4 rows in use + 2 in flight)
constexpr int NXCH = 8;         // doubles per thread in the exchange row
constexpr unsigned WAIT_LIMIT = 1u << 20;

// state order, as the *_e arguments: u, up, v, vp, ssh, sshp
enum { S_U, S_UP, S_V, S_VP, S_SSH, S_SSHP };
// ring fields
enum { R_U, R_V, R_SSH, R_UP, R_VP, R_SSHP, R_H, R_RX, R_RY, R_NBASE, R_MU = R_NBASE, R_RD, R_WF, R_N2D };
// exchange row slots
enum { X_U, X_V, X_FX, X_ST, X_SSHN, X_GX, X_QV, X_SS };

struct Params {
    const double *src[6];
    double *dst[6];
    const double *H, *rhsx, *rhsy, *mu, *rdis, *wflux;
    double *acc[4];
    const uint32_t *bits;
    const RowCoef *rows;
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
struct Smem {
    static constexpr int NF = F2D ? R_N2D : R_NBASE;
    static constexpr size_t ring_bytes = (size_t)RING * NF * SEG * sizeof(double);
    static constexpr size_t bits_bytes = (size_t)RING * 8 * sizeof(uint32_t);
    static constexpr size_t xch_bytes = (size_t)2 * NXCH * W * sizeof(double);
    static constexpr size_t bar_bytes = (size_t)RING * sizeof(uint64_t);
    static constexpr size_t total = ring_bytes + bits_bytes + xch_bytes + bar_bytes;
    static constexpr uint32_t row_tx = (uint32_t)(NF * SEG * sizeof(double) + 8 * sizeof(uint32_t));
};

template <bool F2D>
__global__ void __launch_bounds__(W, 3) k_substep(const Params p)
{
    using L = Smem<F2D>;
    constexpr int NF = L::NF;
    extern __shared__ __align__(128) unsigned char smem[];
    double *ring = reinterpret_cast<double *>(smem);
    uint32_t *rbits = reinterpret_cast<uint32_t *>(smem + L::ring_bytes);
    double *xch = reinterpret_cast<double *>(smem + L::ring_bytes + L::bits_bytes);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + L::ring_bytes + L::bits_bytes + L::xch_bytes);

    const int t = threadIdx.x;
    const int cs = 1 + blockIdx.x * (W - 2);   // device column of thread 0
    const int c = cs + t;
    const int r0 = p.r_first + blockIdx.y * p.chunk_rows;
    const int r1 = min(r0 + p.chunk_rows, p.r_last + 1);   // exclusive
    if (r0 >= r1) return;
    const int row_lo = r0 - 2, row_hi = r1 + 1;             // rows kept in the ring
    const int wbase = ((cs - 1) >> 7) << 2;                 // first mask word of the window
    const int bbase = wbase * 32;                           // its first column
    const long long seg0 = cs - 1;

    auto slot_of = [&](int row) { return (row - row_lo) % RING; };
    auto fld = [&](int slot, int f) -> const double * { return ring + ((size_t)slot * NF + f) * SEG; };
    auto bit = [&](int slot, int col) -> int {
        const int k = col - bbase;
        return (int)((rbits[slot * 8 + (k >> 5)] >> (k & 31)) & 1u);
    };
    auto issue = [&](int row) {
        const int s = slot_of(row);
        uint64_t *bar = &mbar[s];
        mbar_expect_tx(bar, L::row_tx);
        const long long off = (long long)row * p.pitch + seg0;
        double *d = ring + (size_t)s * NF * SEG;
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
        bulk_load(rbits + s * 8, p.bits + (size_t)row * p.bm_words + wbase, 32, bar);
    };

    if (t == 0) {
        for (int s = 0; s < RING; s++) mbar_init(&mbar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued = row_lo - 1;   // (meaningful in thread 0 only)
    if (t == 0)
        for (int row = row_lo; row < row_lo + RING && row <= row_hi; row++) issue(row), issued = row;

    const int tm = max(t - 1, 0), tp = min(t + 1, W - 1);
    const bool out_col = t >= 1 && t <= W - 2 && c >= p.c_first && c <= p.c_last;

    // stage-1 results of earlier rows (own column)
    double U_cur = 0, V_cur = 0, V_prev = 0;
    // stage-2 results of earlier rows (own column)
    double sshn_p = 0, FX_p = 0, GX_p = 0, QV_p = 0, ST_p = 0, SS_p = 0, SS_pp = 0;
    double FY_p = 0, FY_pp = 0, QU_p = 0, QU_pp = 0, GY_p = 0;

    int waited = row_lo - 1;
    bool abort = false;
    for (int j = r0 - 1; j <= r1 + 1; j++) {
        const int need = min(j + 1, row_hi);
        bool ok = true;
        while (waited < need) {
            const int row = waited + 1;
            const uint32_t par = (uint32_t)(((row - row_lo) / RING) & 1);
            if (!mbar_wait(&mbar[slot_of(row)], par)) { ok = false; break; }
            waited = row;
        }
        const double *xr = xch + (size_t)((j + 1) & 1) * NXCH * W;   // written at j-1
        double *xw = xch + (size_t)(j & 1) * NXCH * W;

        double U_new = 0, V_new = 0;
        double sshn_c = 0, FX_c = 0, GX_c = 0, QV_c = 0, ST_c = 0, SS_c = 0, FY_c = 0, QU_c = 0, GY_c = 0;
        if (ok) {
            // ---------------- stage 1: row j ---------------------------------
            if (j <= r1) {
                const int sj = slot_of(j), sn = slot_of(j + 1);
                const RowCoef &rc = p.rows[j];
                const double *Hj = fld(sj, R_H), *Ej = fld(sj, R_SSH);
                const int l0 = bit(sj, c), l1 = bit(sj, c + 1), ln = bit(sn, c);
                const double hq0 = Hj[t + 1] + Ej[t + 1];
                const double hq1 = Hj[t + 2] + Ej[t + 2];
                const double hqn = fld(sn, R_H)[t + 1] + fld(sn, R_SSH)[t + 1];
                // Function/depth.f90:127-139: mask-weighted averages onto u and v points
                const double su = (l0 ? hq0 : 0.0) + (l1 ? hq1 : 0.0);
                const double hu = su * (l0 + l1 == 2 ? rc.ku2 : (l0 + l1 == 1 ? rc.ku : 0.0));
                const double sv = (l0 ? hq0 * rc.wv0 : 0.0) + (ln ? hqn * rc.wv1 : 0.0);
                const double hv = sv * (l0 + ln == 2 ? 0.5 : (l0 + ln == 1 ? 1.0 : 0.0));
                U_new = fld(sj, R_U)[t + 1] * hu;
                V_new = fld(sj, R_V)[t + 1] * hv;
                xw[X_U * W + t] = U_new;
                xw[X_V * W + t] = V_new;
            }
            // ---------------- stage 2: row rho = j-1 -------------------------
            if (j >= r0) {
                const int rho = j - 1;
                const int sr = slot_of(rho), sm = slot_of(rho - 1), su_ = slot_of(rho + 1);
                const RowCoef &rc = p.rows[rho];
                const double *u_r = fld(sr, R_U), *v_r = fld(sr, R_V), *e_r = fld(sr, R_SSH);
                const double *h_r = fld(sr, R_H), *up_r = fld(sr, R_UP), *vp_r = fld(sr, R_VP);
                const double *u_u = fld(su_, R_U), *e_u = fld(su_, R_SSH), *h_u = fld(su_, R_H);
                const int lc = bit(sr, c), lr = bit(sr, c + 1), lu_ = bit(su_, c), lur = bit(su_, c + 1);
                const int luu = lc & lr & lu_ & lur;
                const double U_l = xr[X_U * W + tm];    // U(c-1, rho)
                const double V_r = xr[X_V * W + tp];    // V(c+1, rho)
                // vel_ssh.f90:491-494 continuity (leap-frog over 2*tau_inner)
                const double wq = F2D ? fld(sr, R_WF)[t + 1] * p.inv_rho : p.wq0;
                const double div = (U_cur - U_l) * rc.c_u + V_cur * rc.c_v0 - V_prev * rc.c_v1;
                sshn_c = lc ? fld(sr, R_SSHP)[t + 1] + p.two_ti * (wq - div) : 0.0;
                // vel_ssh.f90:63-73 and :88-98: advective fluxes through T and h faces
                FX_c = (U_l + U_cur) * (u_r[t] + u_r[t + 1]) * rc.fx;
                FY_c = luu ? (V_cur + V_r) * (u_r[t + 1] + u_u[t + 1]) * rc.fy : 0.0;
                GX_c = (U_cur * rc.gx0 + U_new * rc.gx1) * (v_r[t + 1] + v_r[t + 2]);
                GY_c = (V_prev * rc.gy0 + V_cur * rc.gy1) * (fld(sm, R_V)[t + 1] + v_r[t + 1]);
                // depth on the h point, depth.f90:141-147
                const double a0 = h_r[t + 1] + e_r[t + 1], a1 = h_r[t + 2] + e_r[t + 2];
                const double b0 = h_u[t + 1] + e_u[t + 1], b1 = h_u[t + 2] + e_u[t + 2];
                const double s0 = (lc ? a0 : 0.0) + (lr ? a1 : 0.0);
                const double s1 = (lu_ ? b0 : 0.0) + (lur ? b1 : 0.0);
                const int nl = lc + lr + lu_ + lur;
                const double rl = nl == 4 ? 0.25 : (nl == 3 ? 1.0 / 3.0 : (nl == 2 ? 0.5 : (nl == 1 ? 1.0 : 0.0)));
                const double hh = (s0 * rc.wh0 + s1 * rc.wh1) * rl;
                // vel_ssh.f90:35-37 metric vorticity (zero on uniform grids) + Coriolis
                double vort = 0.0;
                if (!p.vort_zero && luu)
                    vort = (v_r[t + 2] - v_r[t + 1]) * rc.vt0 - u_u[t + 1] * rc.vt1 + u_r[t + 1] * rc.vt2;
                const double Wh = hh * (rc.cor + vort);
                QU_c = Wh * (v_r[t + 1] + v_r[t + 2]);
                QV_c = Wh * (u_r[t + 1] + u_u[t + 1]);
                // mixing.f90:134-148 stresses from the previous level
                const double str_t =
                    lc ? rc.t1 * (up_r[t + 1] - up_r[t]) - (rc.t2 * vp_r[t + 1] - rc.t3 * fld(sm, R_VP)[t + 1])
                       : 0.0;
                const double str_s =
                    luu ? rc.s1 * fld(su_, R_UP)[t + 1] - rc.s2 * up_r[t + 1] + rc.s3 * (vp_r[t + 2] - vp_r[t + 1])
                        : 0.0;
                double mu_t = p.mu0, mu_h = p.mu0;
                if constexpr (F2D) {
                    const double *m_r = fld(sr, R_MU), *m_u = fld(su_, R_MU);
                    mu_t = m_r[t + 1];
                    mu_h = (m_r[t + 1] + m_r[t + 2] + m_u[t + 1] + m_u[t + 2]) * 0.25;
                }
                ST_c = mu_t * a0 * str_t;
                SS_c = mu_h * hh * str_s;
                xw[X_FX * W + t] = FX_c;
                xw[X_ST * W + t] = ST_c;
                xw[X_SSHN * W + t] = sshn_c;
                xw[X_GX * W + t] = GX_c;
                xw[X_QV * W + t] = QV_c;
                xw[X_SS * W + t] = SS_c;
            }
            // ---------------- stage 3: row R = j-2 ---------------------------
            if (j >= r0 + 2 && out_col) {
                const int R = j - 2;
                const int sR = slot_of(R), sU = slot_of(R + 1);
                const RowCoef &rc = p.rows[R];
                const int lc = bit(sR, c), lr = bit(sR, c + 1), lup = bit(sU, c);
                const double *e_R = fld(sR, R_SSH), *h_R = fld(sR, R_H), *ep_R = fld(sR, R_SSHP);
                const double ssh0 = e_R[t + 1], sshp0 = ep_R[t + 1], H0 = h_R[t + 1];
                const double sshn0 = sshn_p;
                const long long idx = (long long)R * p.pitch + c;
                if (lc & lr) {   // vel_ssh.f90:536-551
                    const double ssh1 = e_R[t + 2], sshp1 = ep_R[t + 2], H1 = h_R[t + 2];
                    const double sshn1 = xr[X_SSHN * W + t + 1];
                    const double u0 = fld(sR, R_U)[t + 1], up0 = fld(sR, R_UP)[t + 1];
                    const double hu = ((H0 + ssh0) + (H1 + ssh1)) * rc.ku2;
                    const double hup = ((H0 + sshp0) + (H1 + sshp1)) * rc.ku2;
                    const double hun = ((H0 + sshn0) + (H1 + sshn1)) * rc.ku2;
                    const double slx = -(ssh1 - ssh0) * rc.gdyh * hu;
                    const double slxn = -(sshn1 - sshn0) * rc.gdyh * hun;
                    const double adv = -((xr[X_FX * W + t + 1] - FX_p) + (FY_p - FY_pp));
                    const double dif = (xr[X_ST * W + t + 1] - ST_p) * rc.dux + (SS_p * rc.dus0 - SS_pp * rc.dus1);
                    double rd = p.rd0;
                    if constexpr (F2D) rd = (fld(sR, R_RD)[t + 1] + fld(sR, R_RD)[t + 2]) * 0.5;
                    const double grx = fld(sR, R_RX)[t + 1] * p.rhs_scale + slx + dif + adv
                                       - rd * up0 * rc.au * hu + (QU_p + QU_pp) * 0.25;
                    const double un = (up0 * hup + grx * p.two_ti * rc.rau) / hun;
                    if (!(un < 100.0 && un > -100.0)) atomicOr(p.flags, FLAG_GUARD);
                    if (p.acc_mode) {
                        double a = (u0 * hu + un * hun) * p.c4, b = (slx + slxn) * p.c4;
                        if (p.acc_mode == 2) { a += p.acc[0][idx]; b += p.acc[2][idx]; }
                        p.acc[0][idx] = a;
                        p.acc[2][idx] = b;
                    }
                    if (p.write_state) {
                        p.dst[S_UP][idx] = u0 + p.gam * (un - 2.0 * u0 + up0);
                        p.dst[S_U][idx] = un;
                    }
                }
                if (lc & lup) {   // vel_ssh.f90:554-569
                    const double sshU = fld(sU, R_SSH)[t + 1], sshpU = fld(sU, R_SSHP)[t + 1];
                    const double HU = fld(sU, R_H)[t + 1];
                    const double sshnU = sshn_c;
                    const double v0 = fld(sR, R_V)[t + 1], vp0 = fld(sR, R_VP)[t + 1];
                    const double hv = ((H0 + ssh0) * rc.wv0 + (HU + sshU) * rc.wv1) * 0.5;
                    const double hvp = ((H0 + sshp0) * rc.wv0 + (HU + sshpU) * rc.wv1) * 0.5;
                    const double hvn = ((H0 + sshn0) * rc.wv0 + (HU + sshnU) * rc.wv1) * 0.5;
                    const double sly = -(sshU - ssh0) * rc.gdxh * hv;
                    const double slyn = -(sshnU - sshn0) * rc.gdxh * hvn;
                    const double adv = -((GX_p - xr[X_GX * W + t - 1]) + (GY_c - GY_p));
                    const double dif = -(ST_c * rc.dvt1 - ST_p * rc.dvt0) + (SS_p - xr[X_SS * W + t - 1]) * rc.dvs;
                    double rd = p.rd0;
                    if constexpr (F2D) rd = (fld(sR, R_RD)[t + 1] + fld(sU, R_RD)[t + 1]) * 0.5;
                    const double gry = fld(sR, R_RY)[t + 1] * p.rhs_scale + sly + dif + adv
                                       - rd * vp0 * rc.av * hv - (QV_p + xr[X_QV * W + t - 1]) * 0.25;
                    const double vn = (vp0 * hvp + gry * p.two_ti * rc.rav) / hvn;
                    if (!(vn < 100.0 && vn > -100.0)) atomicOr(p.flags, FLAG_GUARD);
                    if (p.acc_mode) {
                        double a = (v0 * hv + vn * hvn) * p.c4, b = (sly + slyn) * p.c4;
                        if (p.acc_mode == 2) { a += p.acc[1][idx]; b += p.acc[3][idx]; }
                        p.acc[1][idx] = a;
                        p.acc[3][idx] = b;
                    }
                    if (p.write_state) {
                        p.dst[S_VP][idx] = v0 + p.gam * (vn - 2.0 * v0 + vp0);
                        p.dst[S_V][idx] = vn;
                    }
                }
                if (lc) {   // vel_ssh.f90:593-596
                    if (!(sshn0 < 10.0 && sshn0 > -10.0)) atomicOr(p.flags, FLAG_GUARD);
                    if (p.write_state) {
                        p.dst[S_SSHP][idx] = ssh0 + p.gam * (sshn0 - 2.0 * ssh0 + sshp0);
                        p.dst[S_SSH][idx] = sshn0;
                    }
                }
            }
        }
        // rotate the register pipelines
        V_prev = V_cur;
        V_cur = V_new;
        U_cur = U_new;
        FY_pp = FY_p; FY_p = FY_c;
        QU_pp = QU_p; QU_p = QU_c;
        SS_pp = SS_p; SS_p = SS_c;
        sshn_p = sshn_c; GY_p = GY_c; ST_p = ST_c; FX_p = FX_c; GX_p = GX_c; QV_p = QV_c;

        if (__syncthreads_or(!ok)) { abort = true; break; }
        if (t == 0) {
            const int dead = j - 2;   // last use of row j-2 was stage 3 above
            if (dead >= row_lo && dead + RING <= row_hi) issue(dead + RING), issued = dead + RING;
        }
    }
    if (abort && t == 0) {
        atomicOr(p.flags, FLAG_TIMEOUT);
        // drain this CTA's copies still in flight (bounded) before exiting
        for (int row = max(waited + 1, row_lo); row <= issued; row++)
            (void)mbar_wait(&mbar[slot_of(row)], (uint32_t)(((row - row_lo) / RING) & 1));
    }
}

// min/max over [m0,m1]x[n0,n1] of three fields, for the uniform-forcing test
__global__ void k_minmax3(Dom D, const float *lu, const double *a, const double *b, const double *c3,
                          double *out)
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

constexpr int MINMAX_BLOCKS = 64;

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
    q.pitch = d.pitch;
    q.bm_words = p.bm_words;
    q.chunk_rows = p.chunk_rows;
    q.r_first = d.ny_start - d.bnd_y1;
    q.r_last = d.ny_end - d.bnd_y1;
    q.c_first = d.nx_start - d.bnd_x1;
    q.c_last = d.nx_end - d.bnd_x1;
    q.mu0 = f.mu0;
    q.rd0 = f.rd0;
    q.wq0 = f.wq0;
    q.inv_rho = 1.0 / c.rho;   // wflux/RefDen as wflux*(1/RefDen): within rounding
    q.rhs_scale = 1.0;
    q.vort_zero = p.vort_zero ? 1 : 0;
    q.flags = p.d_flags;
    return q;
}

void launch(const Plan &p, const Params &q, bool f2d, cudaStream_t s)
{
    dim3 grid(p.nstrips, p.nchunks);
    if (f2d)
        k_substep<true><<<grid, W, Smem<true>::total, s>>>(q);
    else
        k_substep<false><<<grid, W, Smem<false>::total, s>>>(q);
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

}  // namespace

// ===========================================================================
Plan make_plan(const inmsom_bounds &b)
{
    Plan p;
    p.W = W;
    p.outw = W - 2;
    const int nx = b.nx_end - b.nx_start + 1;
    p.nstrips = (nx + p.outw - 1) / p.outw;
    const long long cs_last = 1 + (long long)(p.nstrips - 1) * p.outw;
    p.min_pitch = cs_last + W + 1;
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
    (void)c;
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
    // 1-bit T mask, rows padded so that every CTA window (8 words from a
    // 4-word boundary) is inside the row
    p.bm_words = (int)(((d.pitch + 31) / 32 + 8 + 3) / 4 * 4);
    std::vector<uint32_t> bits((size_t)p.bm_words * nya, 0u);
    const float *lu = masks[0];
    for (int r = 0; r < nya; r++)
        for (int col = 0; col < nxa; col++)
            if (lu[(size_t)r * nxa + col] > 0.5f) bits[(size_t)r * p.bm_words + col / 32] |= 1u << (col % 32);

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

    if (cudaFuncSetAttribute(k_substep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Smem<false>::total) != cudaSuccess)
        return 1;
    if (cudaFuncSetAttribute(k_substep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Smem<true>::total) != cudaSuccess)
        return 1;
    int dev = 0, nsm = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_substep<false>, W, Smem<false>::total) != cudaSuccess ||
        occ < 1)
        occ = 1;
    p.nsm = nsm;
    // one wave: strips x chunks <= SMs x resident CTAs, chunks as tall as that allows
    const int ny = d.ny_end - d.ny_start + 1;
    const int slots = nsm * occ;
    int nchunks = std::max(1, slots / p.nstrips);
    // each chunk re-reads and recomputes three rows of warm-up: keep chunks
    // at least 16 rows tall
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
