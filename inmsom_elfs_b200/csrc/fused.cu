// Fused streaming kernel of the barotropic step (see fused.h).
//
// Work decomposition.  A CTA is one warp; lane l owns device column
// k = g0+2+l of a 32-column strip starting at device column g0+2
// (g0 = 30*strip, even).  Strip columns 1..30 are written, so strips overlap
// by two columns.  The CTA marches down a chunk of rows (a work item; the
// chunks of a strip are cut so that all items cost about the same and the
// single wave of CTAs finishes together); iteration j of its row loop
// computes
//   stage 1,  row j  : u/v-point depths of the current level, the transports
//                      U = u*hu and V = v*hv, and the row's forcing, pressure
//                      gradient and drag terms of the u and v equations;
//   stage 2,  row j-1: new SSH (continuity), advective fluxes on T and h
//                      points, Coriolis-plus-metric-vorticity products,
//                      tension and shear stresses times viscosity and depth;
//   stage 3u, row j-1: u momentum and the SSH update (time-mean sums,
//                      Robert-Asselin filter and time shift, stores);
//   stage 3v, row j-2: the same for v (it needs stage 2 of the row above).
// Each row's contributions to a later stage are folded into a few partial
// sums as soon as they are known, so only two instances of the carried
// values exist; the two-fold unrolled row loop renames them.  A value needed
// from a neighbouring column comes from the neighbouring lane by a warp
// shuffle.  There is no CTA barrier, and the per-column arithmetic is
// branch-free (masked selects, predicated stores) except for warp-wide skips
// of rows without ocean.
//
// Input rows j-2..j+1 sit in a ring of RING shared-memory slots.  A slot
// holds a 36-column segment of the six state fields and of the static
// fields (rest depth, forcing; in the general variant also viscosity, drag
// and water flux), brought by two 3-D tiled TMA loads from field-blocked
// arrays (cp.async.bulk.tensor, each copy for one CTA), plus the row's T-mask bits
// (and, in the general variant, its metric coefficients) by 1-D bulk copies.
// One elected lane refills the slot of row j-2 with row j-2+RING once every
// lane is past it.  Every wait is bounded: on timeout the CTA sets a status bit,
// drains its own copies (bounded) and returns.
//
// Two variants: UNI for square uniform grids (every metric array equal to
// one spacing d; all metric factors fold into a few constants and only the
// Coriolis parameter varies by row) with spatially uniform viscosity, drag
// and water flux; GEN for metrics that vary along y and 2-D forcing fields.
#include "fused.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

namespace inmsom {
namespace fused {

namespace {

constexpr int NL = 32;            // lanes = threads per CTA = strip columns
constexpr int OUTW = NL - 2;      // written columns per strip
constexpr int SEG = NL + 4;       // ring segment: strip columns -2 .. 33
constexpr unsigned WAIT_LIMIT = 1u << 20;

struct alignas(64) Params {
    CUtensorMap tm_src;    // source state set {pitch, rows, 6 fields}, box {SEG, 1, 6}
    CUtensorMap tm_stat;   // static block, box {SEG, 1, Layout::NS}
    CUtensorMap tm_ssh;    // FP32-velocity kernel: the source set's SSH fields, box {SEG, 1, 2}
    CUtensorMap tm_rhs;    // FP32-velocity kernel: RHSx, RHSy in FP32, box {VSEG, 1, 2}
    double *dst[NSET];
    float *vdst[4];        // FP32-velocity kernel: u, up, v, vp of the destination
    double *acc[4];
    const uint32_t *bits;
    const RowCoef *rows;
    const double *cor;
    const int4 *items;     // work items {g0, first row, end row (exclusive), 0}
    long long pitch;
    int bm_words;
    int c_first, c_last;   // interior device columns
    double two_ti, gam, rhs_scale, mu0, rd0, wq0, inv_rho;
    // time means: a substep adds ca * (old level's term) + cb * (new level's)
    double ca, cb;
    double d, inv_d, d4, gd, d2, tt;   // UNI: d, 1/d, d/4, g*d, d*d, two_ti/d^2
    int vort_zero;
    unsigned *flags;
    // RHS scale from device memory (replayable launches): rs_dev[*rs_base + rs_k]
    const double *rs_dev;
    const int *rs_base;
    int rs_k;
    // polls of a bounded mbarrier wait before it gives up; and a test hook:
    // work item hold_item (-1: none) does not issue the copies of its
    // hold_row-th ring row (counted from its first, clamped to its last),
    // so that its wait for that row runs out
    unsigned wait_limit;
    int hold_item, hold_row;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
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

__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// non-blocking: has the phase with this parity completed?
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned limit)
{
    for (unsigned i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Ring slot layout.  FP64 state: [6 state fields][static fields][RowCoef]
// [mask bits].  FP32 velocities (uniform variant only): [u up v vp as FP32,
// VSEG columns from g0 rounded down to a multiple of 4, so that the TMA
// x-coordinate is 16-byte aligned for 4-byte elements][ssh sshp][H][RHSx
// RHSy as FP32, the same columns as the velocities][bits].
template <bool GEN, bool F32 = false>
struct Layout {
    static_assert(!(GEN && F32), "FP32 velocities exist in the uniform variant only");
    static constexpr int VSEG = F32 ? SEG + 4 : 0;                       // FP32 columns per velocity field
    static constexpr int SSH_OFF = F32 ? (4 * VSEG * 4 + 127) / 128 * 128 : 0;
    static constexpr int NS = F32 ? 1 : (GEN ? 6 : 3);                   // static fields in a slot
    static constexpr int STAT_OFF = F32 ? (SSH_OFF + 2 * SEG * 8 + 127) / 128 * 128 : 1792;
    static constexpr int COEF_OFF = STAT_OFF + NS * SEG * 8;             // general variant: RowCoef
    static constexpr int RHS_OFF = F32 ? (COEF_OFF + 127) / 128 * 128 : COEF_OFF;   // FP32 RHSx, RHSy
    static constexpr int BITS_OFF = F32 ? RHS_OFF + 2 * VSEG * 4 : COEF_OFF + (GEN ? (int)sizeof(RowCoef) : 0);
    static constexpr int SLOT_B = (BITS_OFF + 32 + 127) / 128 * 128;
    static constexpr uint32_t row_tx =
        (uint32_t)((F32 ? 4 * VSEG * 4 + 2 * SEG * 8 + 2 * VSEG * 4 : NSET * SEG * 8) + NS * SEG * 8 +
                   (GEN ? (int)sizeof(RowCoef) : 0) + 32);
};

// ring slots: rows j-2..j+1 in use plus one row in flight for the plain
// substep (16 CTAs per SM fit, 20 with FP32 velocities), two in flight where
// the registers hold the CTAs per SM to 12 (time-mean sums)
template <bool GEN, int MODE, bool F32 = false>
__host__ __device__ constexpr int ring_slots()
{
    return (MODE % 3 != 0) ? 6 : 5;
}
template <bool GEN, int MODE, bool F32 = false>
constexpr size_t ring_bytes()
{
    return (size_t)ring_slots<GEN, MODE, F32>() * (Layout<GEN, F32>::SLOT_B + sizeof(uint64_t));
}

// resident CTAs per SM the register budget is cut for: 16 one-warp CTAs
// (4 warps per SM sub-partition, 128 registers) for the plain substep, 20
// (5 warps per sub-partition, 96 registers) for its FP32-velocity form with
// FP32 momentum arithmetic, 12 where the time-mean sums need more registers,
// 11 for the general variant, and never more than the shared memory holds
// (228 KB per SM, 1 KB of it reserved per CTA): 16 for the FP64 uniform ring
// of 5 slots, 20 for the FP32 one, 11 for the general one.  (A 6-slot ring holds 13 uniform CTAs: 6 % slower on the
// 2048 x 1536 basin; 128 bytes of alignment slack per CTA leave room for 15:
// 2 % slower; reading the forcing from global memory instead of the ring
// exposes the load latency: 5 % slower.)
template <bool GEN, int MODE, bool F32 = false>
constexpr int min_ctas()
{
    constexpr int by_smem = (int)(233472 / (ring_bytes<GEN, MODE, F32>() + 1024));
    constexpr int want = GEN ? 11 : (MODE % 3 ? 12 : (F32 ? 20 : 16));
    return by_smem < want ? by_smem : want;
}
static_assert(NSET * SEG * 8 <= 1792, "state segment overlaps the static segment");
static_assert(Layout<false>::COEF_OFF % 16 == 0 && Layout<true>::BITS_OFF % 16 == 0, "bulk copy alignment");
static_assert(Layout<false, true>::RHS_OFF % 128 == 0 && Layout<false, true>::SSH_OFF % 128 == 0 &&
                  Layout<false, true>::STAT_OFF % 128 == 0,
              "TMA destinations of the FP32 slot");
static_assert(Layout<false, true>::BITS_OFF % 16 == 0 && (Layout<false, true>::VSEG * 4) % 16 == 0,
              "FP32 segment alignment");

// One lane elected by elect.sync announces the bytes of a row to the slot's
// mbarrier and starts its copies: the state and static segments (3-D tiled
// TMA, x = g0 even, so 16-byte aligned), the mask-bit window and, in the
// general variant, the row's coefficients (1-D bulk copies).  No branch.
template <bool GEN, bool F32 = false>
__device__ __forceinline__ void issue_row(unsigned char *slot, uint64_t *bar, const CUtensorMap *src,
                                          const CUtensorMap *stat, const CUtensorMap *ssh, const CUtensorMap *rhs,
                                          const void *coef, const void *bits, int x, int row)
{
    using L = Layout<GEN, F32>;
    const int z = 0;
    if constexpr (F32) {
        // velocities from x rounded down to a multiple of 4 (16 bytes of
        // FP32); SSH and SSHP are fields 4 and 5 of the FP64 set
        const int x4 = x & ~3, zs = S_SSH;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "elect.sync _|P, 0xffffffff;\n\t"
            "@P mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n\t"
            "@P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%2], [%3, {%4, %5, %6}], [%0];\n\t"
            "@P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%7], [%8, {%9, %5, %10}], [%0];\n\t"
            "@P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%11], [%12, {%9, %5, %6}], [%0];\n\t"
            "@P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%15], [%16, {%4, %5, %6}], [%0];\n\t"
            "@P cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%13], [%14], 32, [%0];\n\t"
            "}" ::"r"(smem_addr(bar)),
            "r"(L::row_tx), "r"(smem_addr(slot)), "l"(reinterpret_cast<uint64_t>(src)), "r"(x4), "r"(row), "r"(z),
            "r"(smem_addr(slot + L::SSH_OFF)), "l"(reinterpret_cast<uint64_t>(ssh)), "r"(x), "r"(zs),
            "r"(smem_addr(slot + L::STAT_OFF)), "l"(reinterpret_cast<uint64_t>(stat)),
            "r"(smem_addr(slot + L::BITS_OFF)), "l"(bits),
            "r"(smem_addr(slot + L::RHS_OFF)), "l"(reinterpret_cast<uint64_t>(rhs))
            : "memory");
    } else if constexpr (GEN) {
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "elect.sync _|P, 0xffffffff;\n\t"
            "@P mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n\t"
            "@P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%2], [%3, {%4, %5, %6}], [%0];\n\t"
            "@P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%7], [%8, {%4, %5, %6}], [%0];\n\t"
            "@P cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%9], [%10], %11, [%0];\n\t"
            "@P cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%12], [%13], 32, [%0];\n\t"
            "}" ::"r"(smem_addr(bar)),
            "r"(L::row_tx), "r"(smem_addr(slot)), "l"(reinterpret_cast<uint64_t>(src)), "r"(x), "r"(row), "r"(z),
            "r"(smem_addr(slot + L::STAT_OFF)), "l"(reinterpret_cast<uint64_t>(stat)),
            "r"(smem_addr(slot + L::COEF_OFF)), "l"(coef), "n"((int)sizeof(RowCoef)),
            "r"(smem_addr(slot + L::BITS_OFF)), "l"(bits)
            : "memory");
    } else {
        (void)coef;
        (void)ssh;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "elect.sync _|P, 0xffffffff;\n\t"
            "@P mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n\t"
            "@P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%2], [%3, {%4, %5, %6}], [%0];\n\t"
            "@P cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%7], [%8, {%4, %5, %6}], [%0];\n\t"
            "@P cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%9], [%10], 32, [%0];\n\t"
            "}" ::"r"(smem_addr(bar)),
            "r"(L::row_tx), "r"(smem_addr(slot)), "l"(reinterpret_cast<uint64_t>(src)), "r"(x), "r"(row), "r"(z),
            "r"(smem_addr(slot + L::STAT_OFF)), "l"(reinterpret_cast<uint64_t>(stat)),
            "r"(smem_addr(slot + L::BITS_OFF)), "l"(bits)
            : "memory");
    }
}

__device__ __forceinline__ double sel(int m, double x) { return m ? x : 0.0; }
__device__ __forceinline__ float sel(int m, float x) { return m ? x : 0.0f; }

// 1 / (number of ocean T points) for the mask-weighted depth averages
template <class R>
__device__ __forceinline__ R rcount(int n)
{
    return n == 4 ? R(0.25) : (n == 3 ? R(1.0 / 3.0) : (n == 2 ? R(0.5) : (n == 1 ? R(1.0) : R(0.0))));
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
// the FP32 reciprocal, rounded to nearest
__device__ __forceinline__ float rcp_nr(float x) { return __frcp_rn(x); }

// state field F of the slot at byte offset o, at the lane's column + dk:
// FP64, or FP32 velocities widened to FP64
template <bool GEN, bool F32, int F>
__device__ __forceinline__ double ld_state(const unsigned char *lane, const unsigned char *lane32, int o, int dk)
{
    using L = Layout<GEN, F32>;
    if constexpr (F32 && F < S_SSH)
        return (double)*reinterpret_cast<const float *>(lane32 + o + (F * L::VSEG + dk) * 4);
    else if constexpr (F32)
        return *reinterpret_cast<const double *>(lane + o + L::SSH_OFF + ((F - S_SSH) * SEG + dk) * 8);
    else
        return *reinterpret_cast<const double *>(lane + o + (F * SEG + dk) * 8);
}

// a velocity field (u, up, v, vp) in the arithmetic type of the variant:
// FP64, or the FP32 values as stored
template <bool GEN, bool F32, int F>
__device__ __forceinline__ std::conditional_t<F32, float, double> ld_vel(const unsigned char *lane,
                                                                       const unsigned char *lane32, int o, int dk)
{
    using L = Layout<GEN, F32>;
    static_assert(F < S_SSH, "velocity fields only");
    if constexpr (F32)
        return *reinterpret_cast<const float *>(lane32 + o + (F * L::VSEG + dk) * 4);
    else
        return *reinterpret_cast<const double *>(lane + o + (F * SEG + dk) * 8);
}

// a constant in the momentum arithmetic's type: the FP64 value, or its
// FP32 copy
template <bool F32>
__device__ __forceinline__ std::conditional_t<F32, float, double> pick_real(double pv, float fv)
{
    if constexpr (F32)
        return fv;
    else
        return pv;
}

// store a new state value; FP32 velocities are rounded to nearest
template <bool F32, int F, class T>
__device__ __forceinline__ void st_state(float *const *vdst, double *const *dst, long long idx, T v)
{
    if constexpr (F32 && F < S_SSH)
        vdst[F][idx] = (float)v;
    else
        dst[F][idx] = v;
}

#define SHFL_UP(x) __shfl_up_sync(0xffffffffu, (x), 1)
#define SHFL_DN(x) __shfl_down_sync(0xffffffffu, (x), 1)

// R: the arithmetic type of the momentum terms (FP64, or FP32 in the
// FP32-velocity variant); SSH levels and the continuity stay FP64
template <class R>
struct HQ {          // H + ssh of a row at columns k, k+1
    R a, b;
};
// values of row j from stage 1, carried to the next iteration
template <class R>
struct S1 {
    R U, Ul, V, Vr;          // U = u*hu at k, k-1; V = v*hv at k, k+1
    R Ru;                    // u equation of row j: forcing + pressure gradient - drag
    R Rv;                    // v equation of row j: forcing + pressure gradient - drag
    R cor;                   // uniform variant: Coriolis factor of row j
    R slx, sly;              // pressure-gradient terms (time means only)
    HQ<R> hq;                // H + ssh of row j+1
};
// values of row j-1 from stage 2 (and of stage 1 routed on), carried on
template <class R>
struct S2 {
    double sn;               // new SSH of the row
    R V, Uo;                 // V and U of the row
    R vs;                    // v(k) + v(k+1) of the row
    R Cu;                    // the row's part of the u equation of the row above
    R Pv;                    // the row's part of its own v equation, less the GX flux
    R sly;                   // pressure-gradient term of the row (time means only)
    HQ<R> hqm;               // H + ssh of row j
    double au0, au2;         // time-mean sums (u, pgrx) of row j, for the next iteration's stage 3u
    double av1, av3;         // time-mean sums (v, pgry) of row j-1, for its stage 3v
};

template <bool B>
using On = std::integral_constant<bool, B>;

// One substep of one work item (a chunk of rows of a strip), by one warp:
// reads the source set through *tm_src, writes dst[] (and the time-mean
// sums), RHS scaled by rs.  The ring and its mbarriers are this CTA's
// shared memory; they are initialised here and left invalidated (ready for
// the next call) when the item completes.  Returns false after a wait that
// gave up (FLAG_TIMEOUT is set).
// MODE = acc + 3*write: acc 0 none, 1 first substep (write), 2 accumulate;
// write 1 stores the new state
template <bool GEN, int MODE, bool F32 = false>
__device__ __forceinline__ bool substep_item(const Params &p, const CUtensorMap *tm_src, double *const *dst,
                                             const double rs, const int4 item, unsigned char *ring, uint64_t *mbar)
{
    using L = Layout<GEN, F32>;
    constexpr int ACC = MODE % 3;
    constexpr bool WRITE = MODE / 3 != 0;
    constexpr int RING = ring_slots<GEN, MODE, F32>();

    const int l = threadIdx.x;
    const int g0 = item.x;                     // device column of segment offset 0
    const int k = g0 + 2 + l;                  // this lane's column
    const int r0 = item.y, r1 = item.z;        // output rows [r0, r1), r1 > r0
    const int row_lo = r0 - 2, row_hi = r1 + 1;             // rows kept in the ring
    const int wbase = (g0 >> 7) << 2;                       // first mask word of the window
    const int bsh = k - wbase * 32;                         // bit of k in the window
    const unsigned char *lane = ring + (l + 2) * 8;         // this lane's column in a segment
    const unsigned char *lane32 = ring + (l + 2 + (g0 & 3)) * 4;   // ... in an FP32 segment (from g0 & ~3)

    // field f of the state / static segment of the slot at byte offset o
#define AS(o, f, dk) ld_state<GEN, F32, (f)>(lane, lane32, (o), (dk))
#define AV(o, f, dk) ld_vel<GEN, F32, (f)>(lane, lane32, (o), (dk))
#define AT(o, f, dk) (*reinterpret_cast<const double *>(lane + (o) + L::STAT_OFF + ((f) * SEG + (dk)) * 8))
#define CF(o, x) (reinterpret_cast<const RowCoef *>(ring + (o) + L::COEF_OFF)->x)

    auto issue = [&](int row, int slot) {
        if ((int)blockIdx.x == p.hold_item && row == min(row_lo + p.hold_row, row_hi)) return;   // test hook
        issue_row<GEN, F32>(ring + slot * L::SLOT_B, &mbar[slot], tm_src, &p.tm_stat, &p.tm_ssh, &p.tm_rhs, p.rows + row,
                       p.bits + (size_t)row * p.bm_words + wbase, g0, row);
    };
    auto mask2 = [&](int o) -> uint32_t {   // bits: lu(k), lu(k+1)
        const uint32_t *w = reinterpret_cast<const uint32_t *>(ring + o + L::BITS_OFF);
        return __funnelshift_r(w[bsh >> 5], w[(bsh >> 5) + 1], bsh & 31) & 3u;
    };

    if (l == 0) {
        for (int s = 0; s < RING; s++) mbar_init(&mbar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    int issued = row_lo - 1;
    for (int t = 0; t < RING && row_lo + t <= row_hi; t++) issue(row_lo + t, t), issued = row_lo + t;

    const bool out = l >= 1 && l <= NL - 2 && k >= p.c_first && k <= p.c_last;
    const double gam = p.gam, two_ti = p.two_ti;
    // the momentum arithmetic's type, and FP32 copies of the uniform
    // variant's constants for it (the FP64 kernel reads the parameters)
    using R = std::conditional_t<F32, float, double>;
    const float f_gam = (float)p.gam, f_rs = (float)rs, f_d4 = (float)p.d4, f_d = (float)p.d,
                f_inv_d = (float)p.inv_d, f_gd = (float)p.gd, f_tt = (float)p.tt, f_d2 = (float)p.d2,
                f_rd0 = (float)p.rd0, f_mu0 = (float)p.mu0;
#define RK(pv, fv) pick_real<F32>((pv), (fv))

    // slots of rows j-2, j-1, j, j+1 and the fill parity of row j+1
    int i_m2 = RING - 1, i_m1 = 0, i_0 = 1, i_p1 = 2;
    uint32_t ph = 0;
    // T-mask bits, 2 per row: row j+1 in bits 0-1, j in 2-3, j-1 in 4-5, j-2 in 6-7
    uint32_t mk = 0;
    int waited = row_lo - 1;
    bool ready = false;   // row j+1 found complete by a test in the previous iteration
    bool ok = mbar_wait(&mbar[0], 0, p.wait_limit);
    ok = __all_sync(0xffffffffu, ok && mbar_wait(&mbar[1], 0, p.wait_limit));
    if (ok) waited = row_lo + 1;

    S1<R> A{}, B{};
    S2<R> X{}, Y{};
    if (ok) {
        mk = (mask2(0) << 2) | mask2(L::SLOT_B);
        // H + ssh of row r0-1, the "current" row of the first iteration
        B.hq.a = (R)(AT(L::SLOT_B, T_H, 0) + AS(L::SLOT_B, S_SSH, 0));
        B.hq.b = (R)(AT(L::SLOT_B, T_H, 1) + AS(L::SLOT_B, S_SSH, 1));
    }
    long long gi = (long long)(r0 - 1) * p.pitch + k;   // element (row j, column k)

    // One iteration of the row loop; the flags say which stages are valid
    // for row j (the first three and the last iteration lack some).
    auto step = [&](const int j, auto on1, auto on2, auto on3u, auto on3v, S1<R> &n, const S1<R> &c, S2<R> &q,
                    const S2<R> &qc) {
        constexpr bool D1 = decltype(on1)::value, D2 = decltype(on2)::value;
        constexpr bool D3U = decltype(on3u)::value, D3V = decltype(on3v)::value;
        if (!ok) return;
        const int o_m2 = i_m2 * L::SLOT_B, o_m1 = i_m1 * L::SLOT_B, o_0 = i_0 * L::SLOT_B, o_p1 = i_p1 * L::SLOT_B;
        if constexpr (D1) {   // stage 1 reads row j+1
            if (!__all_sync(0xffffffffu, ready)) {
                ok = __all_sync(0xffffffffu, mbar_wait(&mbar[i_p1], ph, p.wait_limit));
                if (!ok) return;
            }
            waited = j + 1;
            mk = (mk << 2) | mask2(o_p1);
        } else {
            mk <<= 2;   // keep the row alignment of mk
        }
        if constexpr (ACC == 2 && D1) {
            // the sums the next iteration's stage 3 adds to, loaded one
            // iteration ahead; exactly where it will write them
            const uint32_t mj = (mk >> 2) & 3u, mj1 = (mk >> 4) & 3u;   // rows j, j-1
            if (out && j >= r0 && j < r1 && mj == 3u) {
                q.au0 = p.acc[0][gi];
                q.au2 = p.acc[2][gi];
            }
            if (out && j - 1 >= r0 && j - 1 < r1 && (mj & mj1 & 1u)) {
                q.av1 = p.acc[1][gi - p.pitch];
                q.av3 = p.acc[3][gi - p.pitch];
            }
        }

        // ---------------- stage 1: row j (independent of stage 2) -------
        if constexpr (D1) {
            const uint32_t mj = (mk >> 2) & 3u, mn = mk & 3u;
            n.hq.a = (R)(AT(o_p1, T_H, 0) + AS(o_p1, S_SSH, 0));
            n.hq.b = (R)(AT(o_p1, T_H, 1) + AS(o_p1, S_SSH, 1));
            const int a = mj & 1, b = (mj >> 1) & 1, cc = mn & 1;
            // Function/depth.f90:127-139 mask-weighted averages to u and v points
            R hu, hv;
            if constexpr (GEN) {
                hu = (sel(a, c.hq.a) + sel(b, c.hq.b)) * (a & b ? CF(o_0, ku2) : (a | b ? CF(o_0, ku) : 0.0));
                hv = (sel(a, c.hq.a * CF(o_0, wv0)) + sel(cc, n.hq.a * CF(o_0, wv1))) *
                     (a & cc ? 0.5 : (a | cc ? 1.0 : 0.0));
            } else {
                hu = (sel(a, c.hq.a) + sel(b, c.hq.b)) * (a & b ? R(0.5) : (a | b ? R(1.0) : R(0.0)));
                hv = (sel(a, c.hq.a) + sel(cc, n.hq.a)) * (a & cc ? R(0.5) : (a | cc ? R(1.0) : R(0.0)));
            }
            n.U = AV(o_0, S_U, 0) * hu;
            n.V = AV(o_0, S_V, 0) * hv;
            // vel_ssh.f90:536-545, :554-565: forcing, pressure gradient of
            // the current level and Rayleigh drag of the previous level
            const double e0 = AS(o_0, S_SSH, 0), e1 = AS(o_0, S_SSH, 1), e1v = AS(o_p1, S_SSH, 0);
            R slx, sly, rdu, rdv, au, av;
            if constexpr (GEN) {
                slx = -(e1 - e0) * CF(o_0, gdyh) * hu;
                sly = -(e1v - e0) * CF(o_0, gdxh) * hv;
                rdu = (AT(o_0, T_RD, 0) + AT(o_0, T_RD, 1)) * 0.5;
                rdv = (AT(o_0, T_RD, 0) + AT(o_p1, T_RD, 0)) * 0.5;
                au = CF(o_0, au);
                av = CF(o_0, av);
            } else {
                slx = -(R)(e1 - e0) * RK(p.gd, f_gd) * hu;
                sly = -(R)(e1v - e0) * RK(p.gd, f_gd) * hv;
                rdu = rdv = RK(p.rd0, f_rd0);
                au = av = RK(p.d2, f_d2);
                n.cor = (R)p.cor[j];
            }
            // RHS: from the ring (FP64 state) or from the FP32 copy
            const R rx = F32 ? (R)*reinterpret_cast<const float *>(lane32 + o_0 + L::RHS_OFF) : (R)AT(o_0, T_RX, 0);
            const R ry = F32 ? (R)*reinterpret_cast<const float *>(lane32 + o_0 + L::RHS_OFF + L::VSEG * 4)
                             : (R)AT(o_0, T_RY, 0);
            n.Ru = rx * RK(rs, f_rs) + slx - rdu * AV(o_0, S_UP, 0) * au * hu;
            n.Rv = ry * RK(rs, f_rs) + sly - rdv * AV(o_0, S_VP, 0) * av * hv;
            if (ACC) {
                n.slx = slx;
                n.sly = sly;
            }
        }

        // forcing of the rows that stage 3 updates, loaded early

        // ---------------- stage 2: row rho = j-1 -------------------------
        double sn;
        R FX, FY, GY, ST, SS, QU, QV, vs, u_r, up_r, v_m, vp_m;
        if constexpr (D2) {
            const uint32_t mr = (mk >> 4) & 3u, mu_ = (mk >> 2) & 3u;   // rows rho, rho+1
            const int lc = mr & 1, lr = (mr >> 1) & 1, lu = mu_ & 1, lur = (mu_ >> 1) & 1;
            const int luu = lc & lr & lu & lur;
            u_r = AV(o_m1, S_U, 0);
            up_r = AV(o_m1, S_UP, 0);
            v_m = AV(o_m2, S_V, 0);
            vp_m = AV(o_m2, S_VP, 0);
            const R u_l = AV(o_m1, S_U, -1), u_u = AV(o_0, S_U, 0);
            const R v_r = AV(o_m1, S_V, 0), v_rr = AV(o_m1, S_V, 1);
            const R up_l = AV(o_m1, S_UP, -1), up_u = AV(o_0, S_UP, 0);
            const R vp_r = AV(o_m1, S_VP, 0), vp_rr = AV(o_m1, S_VP, 1);
            R mu_t = RK(p.mu0, f_mu0), mu_h = RK(p.mu0, f_mu0);
            double wq = p.wq0;
            if constexpr (GEN) {
                mu_t = AT(o_m1, T_MU, 0);
                mu_h = (mu_t + AT(o_m1, T_MU, 1) + AT(o_0, T_MU, 0) + AT(o_0, T_MU, 1)) * 0.25;
                wq = AT(o_m1, T_WF, 0) * p.inv_rho;
            }
            // vel_ssh.f90:491-494 continuity over 2*tau_inner, in FP64 (the
            // FP32 transports widened: their differences are exact)
            const double div = GEN ? (c.U - c.Ul) * CF(o_m1, c_u) + c.V * CF(o_m1, c_v0) - qc.V * CF(o_m1, c_v1)
                                   : (((double)c.U - (double)c.Ul) + ((double)c.V - (double)qc.V)) * p.inv_d;
            sn = sel(lc, AS(o_m1, S_SSHP, 0) + two_ti * (wq - div));
            // vel_ssh.f90:63-73, :88-98 advective fluxes on T and h faces
            vs = v_r + v_rr;
            FX = (c.Ul + c.U) * (u_l + u_r) * (GEN ? (R)CF(o_m1, fx) : RK(p.d4, f_d4));
            FY = sel(luu, (c.V + c.Vr) * (u_r + u_u) * (GEN ? (R)CF(o_m1, fy) : RK(p.d4, f_d4)));
            GY = (GEN ? (R)(qc.V * CF(o_m1, gy0) + c.V * CF(o_m1, gy1)) : (qc.V + c.V) * RK(p.d4, f_d4)) * (v_m + v_r);
            // depth.f90:141-147 depth on the h point
            const R sa = sel(lc, qc.hqm.a) + sel(lr, qc.hqm.b);
            const R sb = sel(lu, c.hq.a) + sel(lur, c.hq.b);
            const R hh = (GEN ? (R)(sa * CF(o_m1, wh0) + sb * CF(o_m1, wh1)) : sa + sb) * rcount<R>(lc + lr + lu + lur);
            // vel_ssh.f90:35-37 metric vorticity (zero on uniform grids) + Coriolis
            R cor;
            if constexpr (GEN) {
                cor = CF(o_m1, cor);
                if (!p.vort_zero)
                    cor += sel(luu, (v_rr - v_r) * CF(o_m1, vt0) - u_u * CF(o_m1, vt1) + u_r * CF(o_m1, vt2));
            } else {
                cor = c.cor;
            }
            const R Wh = hh * cor;
            QU = Wh * vs;
            QV = Wh * (u_r + u_u);
            // mixing.f90:134-148 stresses from the previous level
            const R str_t = GEN ? (R)sel(lc, CF(o_m1, t1) * (up_r - up_l) - (CF(o_m1, t2) * vp_r - CF(o_m1, t3) * vp_m))
                                : sel(lc, ((up_r - up_l) - (vp_r - vp_m)) * RK(p.inv_d, f_inv_d));
            const R str_s = GEN ? (R)sel(luu, CF(o_m1, s1) * up_u - CF(o_m1, s2) * up_r + CF(o_m1, s3) * (vp_rr - vp_r))
                                : sel(luu, ((up_u - up_r) + (vp_rr - vp_r)) * RK(p.inv_d, f_inv_d));
            ST = mu_t * qc.hqm.a * str_t;
            SS = mu_h * hh * str_s;
        }
        R FXr, STr, QVl, SSl;
        double SNr;
        if constexpr (D2) {
            FXr = SHFL_DN(FX);
            STr = SHFL_DN(ST);
            SNr = SHFL_DN(sn);
            QVl = SHFL_UP(QV);
            SSl = SHFL_UP(SS);
        }
        if constexpr (D1) {
            n.Ul = SHFL_UP(n.U);
            n.Vr = SHFL_DN(n.V);
        }
        // test (without waiting) whether row j+2 has arrived, so that the
        // next iteration's branch on it does not wait for the test
        {
            const int ns = i_p1 == RING - 1 ? 0 : i_p1 + 1;
            ready = mbar_test(&mbar[ns], ph ^ (ns == 0 ? 1u : 0u));
        }

        // ---------------- stage 3u: row rho = j-1 (u and SSH) -----------
        if constexpr (D3U) {
            const uint32_t mr = (mk >> 4) & 3u;
            if (__any_sync(0xffffffffu, out && (mr & 1u))) {
                const int lc = mr & 1, lr = (mr >> 1) & 1;
                const bool wu = out && (lc & lr), wt = out && lc;
                const double e0 = AS(o_m1, S_SSH, 0);
                const double sp0 = AS(o_m1, S_SSHP, 0), sp1 = AS(o_m1, S_SSHP, 1);
                const double h0 = AT(o_m1, T_H, 0), h1 = AT(o_m1, T_H, 1);
                // vel_ssh.f90:536-551
                const R ku2 = GEN ? (R)CF(o_m1, ku2) : R(0.5);
                const R hup = (R)((h0 + sp0) + (h1 + sp1)) * ku2;
                const R hun = (R)((h0 + sn) + (h1 + SNr)) * ku2;
                const R difx = GEN ? (R)((STr - ST) * CF(o_m1, dux) + SS * CF(o_m1, dus0)) : ((STr - ST) + SS) * RK(p.d, f_d);
                const R grx = c.Ru + qc.Cu - ((FXr - FX) + FY) + difx + QU * R(0.25);
                const R un = (up_r * hup + grx * (GEN ? (R)(two_ti * CF(o_m1, rau)) : RK(p.tt, f_tt))) * rcp_nr(hun);
                const long long idx = gi - p.pitch;
                if (ACC && wu) {
                    const double slxn = -(SNr - sn) * (GEN ? CF(o_m1, gdyh) : p.gd) * hun;
                    double a = c.U * p.ca + un * hun * p.cb, b = c.slx * p.ca + slxn * p.cb;
                    if (ACC == 2) { a += qc.au0; b += qc.au2; }
                    p.acc[0][idx] = a;
                    p.acc[2][idx] = b;
                }
                if (WRITE && wu) {
                    st_state<F32, S_UP>(p.vdst, dst, idx, u_r + RK(gam, f_gam) * (un - R(2.0) * u_r + up_r));
                    st_state<F32, S_U>(p.vdst, dst, idx, un);
                }
                if (WRITE && wt) {   // vel_ssh.f90:593-596
                    dst[S_SSHP][idx] = e0 + gam * (sn - 2.0 * e0 + sp0);
                    dst[S_SSH][idx] = sn;
                }
            }
        }

        // ---------------- stage 3v: row R = j-2 (v) ----------------------
        if constexpr (D3V) {
            // vel_ssh.f90:88-98 the x flux of v on the h point of row R,
            // from the transports of rows R and R+1
            const R GX = (GEN ? (R)(qc.Uo * CF(o_m2, gx0) + c.U * CF(o_m2, gx1)) : (qc.Uo + c.U) * RK(p.d4, f_d4)) * qc.vs;
            const R GXl = SHFL_UP(GX);
            const uint32_t mR = (mk >> 6) & 3u, mU = (mk >> 4) & 3u;   // rows R, R+1
            if (__any_sync(0xffffffffu, out && (mR & mU & 1u))) {
                const bool wv = out && (mR & mU & 1u);
                const double sp0 = AS(o_m2, S_SSHP, 0), sp1 = AS(o_m1, S_SSHP, 0);
                const double h0 = AT(o_m2, T_H, 0), h1 = AT(o_m1, T_H, 0);
                const R v0 = v_m, vp0 = vp_m;
                const double sn0 = qc.sn, sn1 = sn;
                // vel_ssh.f90:554-569
                R hvp, hvn;
                if constexpr (GEN) {
                    hvp = ((h0 + sp0) * CF(o_m2, wv0) + (h1 + sp1) * CF(o_m2, wv1)) * 0.5;
                    hvn = ((h0 + sn0) * CF(o_m2, wv0) + (h1 + sn1) * CF(o_m2, wv1)) * 0.5;
                } else {
                    hvp = (R)((h0 + sp0) + (h1 + sp1)) * R(0.5);
                    hvn = (R)((h0 + sn0) + (h1 + sn1)) * R(0.5);
                }
                const R gry = qc.Pv - (GX - GXl) - GY - ST * (GEN ? (R)CF(o_m2, dvt1) : RK(p.d, f_d));
                const R vn = (vp0 * hvp + gry * (GEN ? (R)(two_ti * CF(o_m2, rav)) : RK(p.tt, f_tt))) * rcp_nr(hvn);
                const long long idx = gi - 2 * p.pitch;
                if (ACC && wv) {
                    const double slyn = -(sn1 - sn0) * (GEN ? CF(o_m2, gdxh) : p.gd) * hvn;
                    double a = qc.V * p.ca + vn * hvn * p.cb, b = qc.sly * p.ca + slyn * p.cb;
                    if (ACC == 2) { a += qc.av1; b += qc.av3; }
                    p.acc[1][idx] = a;
                    p.acc[3][idx] = b;
                }
                if (WRITE && wv) {
                    st_state<F32, S_VP>(p.vdst, dst, idx, v0 + RK(gam, f_gam) * (vn - R(2.0) * v0 + vp0));
                    st_state<F32, S_V>(p.vdst, dst, idx, vn);
                }
            }
        }

        // ---------------- carry row rho on ------------------------------
        if constexpr (D2) {
            // its part of the u equation of row rho+1 (vel_ssh.f90:539-541):
            // +FY(rho), -SS(rho)*dxb(rho)^2/dxt(rho+1), +QU(rho)/4
            q.Cu = FY + QU * R(0.25) - SS * (GEN ? (R)CF(o_0, dus1) : RK(p.d, f_d));
            // its part of its own v equation (vel_ssh.f90:557-560); the
            // next iteration adds -(GX - GX(k-1)), -GY(rho+1) and
            // -ST(rho+1)*dx(rho+1)^2/dxh(rho)
            const R dify = GEN ? (R)(ST * CF(o_m1, dvt0) + (SS - SSl) * CF(o_m1, dvs)) : (ST + (SS - SSl)) * RK(p.d, f_d);
            q.Pv = c.Rv + GY + dify - (QV + QVl) * R(0.25);
            q.sn = sn;
            q.vs = vs;
        }
        q.V = c.V;
        q.Uo = c.U;
        q.hqm = c.hq;
        if (ACC) q.sly = c.sly;

        // row j-2 was last read above: once every lane is past it, its slot
        // takes row j-2+RING
        __syncwarp();
        if (j - 2 >= row_lo && j - 2 + RING <= row_hi) {
            issue(j - 2 + RING, i_m2);
            issued = j - 2 + RING;
        }
        i_m2 = i_m1;
        i_m1 = i_0;
        i_0 = i_p1;
        i_p1 = i_p1 == RING - 1 ? 0 : i_p1 + 1;
        ph ^= i_p1 == 0 ? 1u : 0u;
        gi += p.pitch;
    };

    // two instances of each carried struct, renamed (not copied) by the
    // two-fold unrolled loop; iterations r0-1, r0, r0+1 and r1+1 lack stages
    const On<true> Y1;
    const On<false> N0;
    step(r0 - 1, Y1, N0, N0, N0, A, B, X, Y);
    step(r0, Y1, Y1, N0, N0, B, A, Y, X);
    step(r0 + 1, Y1, Y1, Y1, N0, A, B, X, Y);
    int j = r0 + 2;
    for (; j + 1 <= r1 && ok; j += 2) {
        step(j, Y1, Y1, Y1, Y1, B, A, Y, X);
        step(j + 1, Y1, Y1, Y1, Y1, A, B, X, Y);
    }
    if (j <= r1) {
        step(j, Y1, Y1, Y1, Y1, B, A, Y, X);
        step(j + 1, N0, Y1, N0, Y1, A, B, X, Y);
    } else {
        step(j, N0, Y1, N0, Y1, B, A, Y, X);
    }
    if (!ok) {
        if (l == 0) {
            atomicOr(p.flags, FLAG_TIMEOUT);
            // drain this CTA's copies still in flight (bounded) before exiting
            for (int row = waited + 1; row <= issued; row++)
                (void)mbar_wait(&mbar[(row - row_lo) % RING], (uint32_t)(((row - row_lo) / RING) & 1),
                                p.wait_limit);
        }
        return false;
    }
    // every copy issued was waited for: the barriers can be retired
    __syncwarp();
    if (l == 0)
        for (int t = 0; t < RING; t++) mbar_inval(&mbar[t]);
    __syncwarp();
    return true;
#undef AS
#undef AV
#undef RK
#undef AT
#undef CF
}

template <bool GEN, int MODE, bool F32 = false>
__global__ void __launch_bounds__(NL, min_ctas<GEN, MODE, F32>()) k_substep(const __grid_constant__ Params p)
{
    using L = Layout<GEN, F32>;
    constexpr int RING = ring_slots<GEN, MODE, F32>();
    // launched with programmatic stream serialisation: the CTAs may become
    // resident while the previous substep's last CTAs run; nothing global
    // is read or written before that grid has completed
    asm volatile("griddepcontrol.wait;" ::: "memory");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // the dynamic shared memory is the ring itself (no alignment slack, so
    // that 16 uniform CTAs fit per SM): its TMA slots need a 128-byte base
    unsigned char *ring = smem_raw;
    if (smem_addr(smem_raw) & 127u) {
        if (threadIdx.x == 0) atomicOr(p.flags, FLAG_SMEM);
        return;
    }
    uint64_t *mbar = reinterpret_cast<uint64_t *>(ring + RING * L::SLOT_B);
    const double rs = p.rs_dev ? p.rs_dev[*p.rs_base + p.rs_k] : p.rhs_scale;
    (void)substep_item<GEN, MODE, F32>(p, &p.tm_src, p.dst, rs, p.items[blockIdx.x], ring, mbar);
}

// ---------------------------------------------------------------------
// Persistent ensemble kernel: ONE cooperative launch advances every member
// of an ensemble by a group of plain substeps.  Its CTAs (one wave, all
// resident) claim work items from one counter in the order (substep, member,
// item) (a table of {member, item} per claim of a substep); an item of
// member m at substep s starts once member m's items of
// substep s - 1 are all done (a per-member, per-substep completion counter),
// so members never wait for each other and a member's substeps follow one
// another with no launch boundary.  Claims are monotonic and every claimed
// item's dependencies were claimed earlier by resident CTAs, so the waits
// always end; they are bounded all the same (a wait that gives up sets the
// member's timeout bit and the item runs anyway, its result then wrong).
// The items and their arithmetic are those of k_substep: the same values
// bit for bit.
struct EnsItem {
    Params q[2];          // parity 0: reads the state set, writes the first ping-pong set; 1: back
    const int4 *items;
    int nitems, gen;
};
static_assert(sizeof(EnsItem) % 64 == 0, "tensor maps of consecutive members stay 64-byte aligned");

__device__ __forceinline__ unsigned ld_acquire(const unsigned *a)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
    return v;
}

// resident CTAs per SM the kernel is cut for: the general variant's where
// some member takes it, else 12 (on 64 regional basins 16 CTAs, at 128
// registers with a few bytes spilled, ran 8 % slower, 11 CTAs 10 % slower,
// and 8, 10 and 12 alike)
template <bool ANYGEN>
constexpr int ens_ctas()
{
    return ANYGEN ? min_ctas<true, 3>() : 12;
}
constexpr unsigned ENS_WAIT_POLLS = 1u << 16;

template <bool ANYGEN>
__global__ void __launch_bounds__(NL, ens_ctas<ANYGEN>())
    k_ens_persistent(const EnsItem *__restrict__ mem, const int2 *__restrict__ order, int total, int group,
                     unsigned *ctr, unsigned *done)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *ring = smem_raw;
    const int l = threadIdx.x;
    if (smem_addr(smem_raw) & 127u) {
        if (l == 0) atomicOr(mem[0].q[0].flags, FLAG_SMEM);
        return;
    }
    const unsigned work = (unsigned)total * (unsigned)group;
    for (;;) {
        unsigned c = 0;
        if (l == 0) c = atomicAdd(ctr, 1u);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= work) break;
        const int st = (int)(c / (unsigned)total);
        const int2 mi = order[c % (unsigned)total];   // {member, item} of this claim within the substep
        const int m = mi.x;
        const EnsItem &em = mem[m];
        const Params &q = em.q[st & 1];
        if (st > 0) {
            if (l == 0) {
                // an item lasts well under a millisecond: 2^16 polls of at
                // least 128 ns each are ample
                unsigned polls = 0;
                while (ld_acquire(&done[m * group + st - 1]) < (unsigned)em.nitems) {
                    if (++polls > ENS_WAIT_POLLS) {
                        atomicOr(q.flags, FLAG_TIMEOUT);
                        break;
                    }
                    __nanosleep(128);
                }
            }
            __syncwarp();
            // the bulk copies below read what other CTAs stored
            asm volatile("fence.proxy.async;" ::: "memory");
        }
        const double rs = q.rs_dev[*q.rs_base + st];
        const int4 item = em.items[mi.y];
        if (ANYGEN && em.gen) {
            uint64_t *mbar = reinterpret_cast<uint64_t *>(ring + ring_slots<true, 3>() * Layout<true>::SLOT_B);
            (void)substep_item<true, 3>(q, &q.tm_src, q.dst, rs, item, ring, mbar);
        } else {
            uint64_t *mbar = reinterpret_cast<uint64_t *>(ring + ring_slots<false, 3>() * Layout<false>::SLOT_B);
            (void)substep_item<false, 3>(q, &q.tm_src, q.dst, rs, item, ring, mbar);
        }
        // this item's stores, visible to the bulk copies of later items, then counted
        asm volatile("fence.proxy.async;" ::: "memory");
        __threadfence();
        __syncwarp();
        if (l == 0) atomicAdd(&done[m * group + st], 1u);
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

// FP64 -> FP32 (round to nearest), n values
// FP64 -> FP32, rounded to nearest; four values per thread and iteration
// (two 16-byte loads, one 16-byte store) where the arrays allow it
__global__ void k_to_f32(const double *a, float *b, long long n)
{
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, st = (long long)gridDim.x * blockDim.x;
    const bool vec = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15u) == 0;
    const long long n4 = vec ? n / 4 : 0;
    for (long long i = t0; i < n4; i += st) {
        const double2 x = reinterpret_cast<const double2 *>(a)[2 * i], y = reinterpret_cast<const double2 *>(a)[2 * i + 1];
        reinterpret_cast<float4 *>(b)[i] = make_float4((float)x.x, (float)x.y, (float)y.x, (float)y.y);
    }
    for (long long i = 4 * n4 + t0; i < n; i += st) b[i] = (float)a[i];
}

// FP32 velocities back into an FP64 set at the points the FP32 kernel
// writes: u, up on lcu, v, vp on lcv (interior); every other point of the
// FP64 set keeps its value
// (one thread per column of a row: blockIdx.y strides the rows)
__global__ void k_vel_from_f32(const float *vs, double *set, const float *lu, long long pitch, long long fs, int r0,
                               int r1, int c0, int c1)
{
    const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c > c1) return;
    for (int row = r0 + blockIdx.y; row <= r1; row += gridDim.y) {
        const long long i = (long long)row * pitch + c;
        const bool o = lu[i] > 0.5f;
        if (o && lu[i + 1] > 0.5f) {
            set[S_U * fs + i] = (double)vs[0 * fs + i];
            set[S_UP * fs + i] = (double)vs[1 * fs + i];
        }
        if (o && lu[i + pitch] > 0.5f) {
            set[S_V * fs + i] = (double)vs[2 * fs + i];
            set[S_VP * fs + i] = (double)vs[3 * fs + i];
        }
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

// copy the forcing fields the variant reads into the static block
int stage_forcing(Plan &p, double *forc[6], int gen, cudaStream_t s)
{
    p.f32_rhs_key = 0;   // the FP32 copy of RHSx, RHSy is stale
    const size_t fb = (size_t)p.fstride * sizeof(double);
    const int src_of[NSTAT] = {-1, 0, 1, 3, 5, 2};   // T_* <- forc index (RHSx RHSy wflux mu mu4 rdis)
    for (int t = 1; t < NSTAT; t++)
        if ((gen || t <= T_RY) &&
            cudaMemcpyAsync(p.stat + t * p.fstride, forc[src_of[t]], fb, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return 1;
    return 0;
}

Params base_params(const Plan &p, const Dom &d, const Consts &c, const Forcing &f, int gen)
{
    Params q;
    std::memset(&q, 0, sizeof q);
    q.tm_stat = p.tm_stat[gen];
    q.bits = p.bits;
    q.rows = p.rows;
    q.cor = p.cor;
    q.pitch = d.pitch;
    q.bm_words = p.bm_words;
    q.c_first = d.nx_start - d.bnd_x1 + d.xoff;
    q.c_last = d.nx_end - d.bnd_x1 + d.xoff;
    q.mu0 = f.mu0;
    q.rd0 = f.rd0;
    q.wq0 = f.wq0;
    q.inv_rho = 1.0 / c.rho;   // wflux/RefDen as wflux*(1/RefDen): within rounding
    q.rhs_scale = 1.0;
    q.vort_zero = p.vort_zero ? 1 : 0;
    q.flags = p.d_flags;
    q.wait_limit = p.wait_limit ? p.wait_limit : WAIT_LIMIT;
    q.hold_item = p.hold_item;
    q.hold_row = p.hold_row;
    q.d = p.d;
    q.inv_d = p.d != 0.0 ? 1.0 / p.d : 0.0;
    q.d4 = p.d / 4.0;
    q.gd = c.g * p.d;
    q.d2 = p.d * p.d;
    q.items = p.items[gen];
    return q;
}

void set_times(Params &q, double two_ti, const Plan &p)
{
    q.two_ti = two_ti;
    q.tt = p.d != 0.0 ? two_ti * (1.0 / (p.d * p.d)) : 0.0;
}

// source and destination sets of one launch (state order)
int set_io(const Plan &p, Params &q, double *const src[NSET], double *const dst[NSET])
{
    int s = -1;
    for (int b = 0; b < 3; b++)
        if (p.set[b] == src[0]) s = b;
    if (s < 0) return 1;
    q.tm_src = p.tm_set[s];
    for (int k = 0; k < NSET; k++) q.dst[k] = dst[k];
    return 0;
}

// a substep launch that may start while the previous one drains (the
// kernel waits for it with griddepcontrol.wait before touching memory):
// 2 % on the time-mean substeps of a drop-in call, none under graph replay
template <bool GEN, int MODE, bool F32 = false>
void launch_substep(int grid, const Params &q, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(NL);
    cfg.dynamicSmemBytes = ring_bytes<GEN, MODE, F32>();
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    (void)cudaLaunchKernelEx(&cfg, k_substep<GEN, MODE, F32>, q);   // errors: cudaGetLastError
}

template <bool GEN, int MODE>
void launch_t(const Plan &p, const Params &q, cudaStream_t s)
{
    const int v = item_table(GEN, MODE);
    Params r = q;
    r.items = p.items[v];
    launch_substep<GEN, MODE>(p.nitems[v], r, s);
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

// returns nonzero (nothing launched) if the static map does not bring
// exactly the fields the ring layout holds
int launch(Plan &p, const Params &q, int gen, int mode, cudaStream_t s)
{
    if (p.stat_box[gen] != (gen ? Layout<true>::NS : Layout<false>::NS)) return 1;
    p.last_variant = gen;
    if (gen) launch_g<true>(p, q, mode, s);
    else launch_g<false>(p, q, mode, s);
    return 0;
}

int sync_buffers(Plan &p, double *state[6], cudaStream_t s)
{
    const size_t bytes = (size_t)NSET * p.fstride * sizeof(double);
    for (int b = 0; b < 2; b++)
        if (cudaMemcpyAsync(p.buf[b][0], state[0], bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return 1;
    p.buffers_synced = true;
    for (bool &f : p.f32_land) f = false;
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
                                (int)ring_bytes<GEN, MODE>()) != cudaSuccess;
}

int set_smem()
{
    return set_smem1<false, 2>() | set_smem1<false, 3>() | set_smem1<false, 4>() | set_smem1<false, 5>() |
           set_smem1<true, 2>() | set_smem1<true, 3>() | set_smem1<true, 4>() | set_smem1<true, 5>() |
           (cudaFuncSetAttribute(k_substep<false, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ring_bytes<false, 3, true>()) != cudaSuccess);
}

using EncodeTiled = decltype(&cuTensorMapEncodeTiled);

// {pitch, rows, nfields} doubles with field stride fstride; box {SEG, 1, box_fields}
int encode_fields(EncodeTiled enc, CUtensorMap *map, void *base, const Dom &d, long long fstride, int nfields,
                  int box_fields, bool f32 = false)
{
    const cuuint64_t esz = f32 ? sizeof(float) : sizeof(double);
    const cuuint64_t dims[3] = {(cuuint64_t)d.pitch, (cuuint64_t)d.nya(), (cuuint64_t)nfields};
    const cuuint64_t strides[2] = {(cuuint64_t)d.pitch * esz, (cuuint64_t)fstride * esz};
    const cuuint32_t box[3] = {(cuuint32_t)(f32 ? Layout<false, true>::VSEG : SEG), 1u, (cuuint32_t)box_fields};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    return enc(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides,
               box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS;
}

constexpr double LAND_COST = 0.7;

// Ocean flags of the written columns of every strip and device row
// (strip-major, nya rows per strip), from the host T mask.
std::vector<uint8_t> ocean_rows(const Plan &p, const Dom &d, const float *lu)
{
    const int nxa = d.nxa(), nya = d.nya();
    const int cf = d.nx_start - d.bnd_x1 + d.xoff, cl = d.nx_end - d.bnd_x1 + d.xoff;
    std::vector<uint8_t> oc((size_t)p.nstrips * nya, 0);
    for (int s = 0; s < p.nstrips; s++) {
        const int g0 = s * p.outw;
        const int c0 = std::max(g0 + 3, cf), c1 = std::min(g0 + 2 + p.outw, cl);   // written columns
        for (int r = 0; r < nya; r++) {
            bool ocean = false;
            for (int col = c0; col <= c1 && !ocean; col++) ocean = lu[(size_t)r * nxa + (col - d.xoff)] > 0.5f;
            oc[(size_t)s * nya + r] = ocean;
        }
    }
    return oc;
}

// Work items of one variant: each strip's rows rf..rl (device rows; the
// interior unless a row strip computes into its halo) cut into chunks of
// about equal cost.  rows_per_item = 0: as many items in all as one wave of
// resident CTAs holds (`slots`), so that the wave finishes together; else
// about that many rows per item (several waves).  A row whose written
// columns are all land skips the momentum stages and costs about LAND_COST
// of an ocean row; no chunk is shorter than p.min_rows rows (each pays
// three warm-up iterations: 4 rows for a basin alone, where the items of a
// small basin would otherwise fill few SMs; 16 for an ensemble member, whose
// neighbours fill the rest).
std::vector<int4> partition(const Plan &p, const Dom &d, int slots, int rows_per_item, int rf, int rl)
{
    const int ny = rl - rf + 1, nya = d.nya();
    std::vector<std::vector<double>> cost(p.nstrips, std::vector<double>(ny));
    std::vector<double> total(p.nstrips, 0.0);
    double all = 0.0;
    for (int s = 0; s < p.nstrips; s++) {
        for (int r = 0; r < ny; r++) {
            cost[s][r] = p.ocean[(size_t)s * nya + rf + r] ? 1.0 : LAND_COST;
            total[s] += cost[s][r];
        }
        all += total[s];
    }
    const int maxc = std::max(1, ny / std::max(1, p.min_rows));
    std::vector<int> n(p.nstrips);
    if (rows_per_item > 0) {
        for (int s = 0; s < p.nstrips; s++)
            n[s] = std::min(maxc, std::max(1, (ny + rows_per_item / 2) / rows_per_item));
    } else {
        // chunks per strip in proportion to its cost (largest remainder)
        const int want = std::min(std::max(slots, p.nstrips), p.nstrips * maxc);
        std::vector<std::pair<double, int>> frac;
        int used = 0;
        for (int s = 0; s < p.nstrips; s++) {
            const double exact = all > 0.0 ? want * total[s] / all : 1.0;
            n[s] = std::min(maxc, std::max(1, (int)exact));
            used += n[s];
            frac.push_back({exact - (int)exact, s});
        }
        std::sort(frac.begin(), frac.end(), [](const std::pair<double, int> &a, const std::pair<double, int> &b) {
            return a.first > b.first;
        });
        for (size_t t = 0; used < want && t < frac.size(); t++)
            if (n[frac[t].second] < maxc) n[frac[t].second]++, used++;
    }
    // cut each strip at equal shares of its cumulative cost
    std::vector<int4> items;
    for (int s = 0; s < p.nstrips; s++) {
        const double share = total[s] / n[s];
        double acc = 0.0;
        int start = rf, made = 0;
        for (int r = rf; r <= rl; r++) {
            acc += cost[s][r - rf];
            const bool last_row = r == rl;
            const bool cut = made < n[s] - 1 && acc >= share * (made + 1) && rl - r >= n[s] - 1 - made;
            if (cut || last_row) {
                items.push_back(make_int4(s * p.outw, start, r + 1, 0));
                start = r + 1;
                made++;
            }
        }
    }
    return items;
}

std::vector<int4> partition(const Plan &p, const Dom &d, int slots, int rows_per_item)
{
    return partition(p, d, slots, rows_per_item, d.ny_start - d.bnd_y1, d.ny_end - d.bnd_y1);
}

// waves of work items per table: one for the plain substep (measured on the
// 2048 x 1536 basin: 2 waves +5.6 %, 1.5 waves +15 %), two for the
// time-mean substeps (-1.9 % against one)
int item_waves(int table) { return table == 2 || table == 3 ? 2 : 1; }

// Replaces table v.  On failure the plan keeps its previous table (a
// launch never sees a count without its items).
int upload_items(Plan &p, int v, const std::vector<int4> &items, cudaStream_t s)
{
    int4 *t = nullptr;
    if (cudaMalloc(&t, items.size() * sizeof(int4)) != cudaSuccess) return 1;
    // the item table is a host vector: finish its copy before returning
    if (cudaMemcpyAsync(t, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaFree(t);
        return 1;
    }
    p.generation++;
    cudaFree(p.items[v]);
    p.items[v] = t;
    p.nitems[v] = (int)items.size();
    return 0;
}

void release(Plan &p)
{
    cudaFree(p.rows);
    cudaFree(p.cor);
    cudaFree(p.bits);
    // the plan owns the two sets that are not the caller's current state
    cudaFree(p.buf[0][0]);
    cudaFree(p.buf[1][0]);
    cudaFree(p.stat);
    cudaFree(p.d_uniform);
    cudaFree(p.d_flags);
    for (auto &it : p.items) {
        cudaFree(it);
        it = nullptr;
    }
    for (auto &t : p.ext) cudaFree(t.items);
    p.ext.clear();
    for (auto &v : p.vset) {
        cudaFree(v);
        v = nullptr;
    }
    cudaFree(p.stat32);
    p.stat32 = nullptr;
    p.rows = nullptr;
    p.cor = nullptr;
    p.bits = nullptr;
    for (auto &b : p.buf)
        for (auto &x : b) x = nullptr;
    p.stat = nullptr;
    p.d_uniform = nullptr;
    p.d_flags = nullptr;
}


EncodeTiled encoder()
{
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) != cudaSuccess ||
        qr != cudaDriverEntryPointSuccess)
        return nullptr;
    return reinterpret_cast<EncodeTiled>(fn);
}

// FP32 velocity sets (u up v vp per state set), FP32 forcing and their
// tensor maps, made on the first FP32-velocity run
int ensure_f32(Plan &p, const Dom &d, cudaStream_t s)
{
    if (p.vset[0]) return 0;
    for (bool &f : p.f32_land) f = false;
    p.f32_rhs_key = 0;
    EncodeTiled enc = encoder();
    if (!enc) return 1;
    const size_t fb = (size_t)p.fstride * sizeof(float);
    for (int b = 0; b < 3; b++) {
        if (cudaMalloc(&p.vset[b], 4 * fb) != cudaSuccess) return 1;
        if (cudaMemsetAsync(p.vset[b], 0, 4 * fb, s) != cudaSuccess) return 1;
        if (encode_fields(enc, &p.tm_vel[b], p.vset[b], d, p.fstride, 4, 4, true)) return 1;
        if (encode_fields(enc, &p.tm_ssh[b], p.set[b], d, p.fstride, NSET, 2)) return 1;
    }
    if (encode_fields(enc, &p.tm_stat_f32, p.stat, d, p.fstride, NSTAT, Layout<false, true>::NS)) return 1;
    p.stat_box_f32 = Layout<false, true>::NS;
    if (cudaMalloc(&p.stat32, 2 * fb) != cudaSuccess) return 1;
    if (cudaMemsetAsync(p.stat32, 0, 2 * fb, s) != cudaSuccess) return 1;
    // RHSx, RHSy in FP32: the box brings both fields, as the slot layout holds
    if (encode_fields(enc, &p.tm_rhs32, p.stat32, d, p.fstride, 2, 2, true)) return 1;
    return 0;
}

int set_index(const Plan &p, const double *base)
{
    for (int b = 0; b < 3; b++)
        if (p.set[b] == base) return b;
    return -1;
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
    // a row strip of a larger basin: the halo rows next to another strip
    // hold that strip's values (they may be ocean), and there the halo may
    // be wider than 2 rows (an even number: a strip that advances k
    // substeps per exchange computes 2(k-1) rows into it)
    const bool open_s = d.ny_start > d.nnn, open_n = d.ny_end < d.nn;
    const int hs = d.ny_start - d.bnd_y1, hn = d.bnd_y2 - d.ny_end;
    if (d.bnd_x1 != d.nx_start - 2 || d.bnd_x2 != d.nx_end + 2 || (open_s ? hs < 2 || hs % 2 : hs != 2) ||
        (open_n ? hn < 2 || hn % 2 : hn != 2))
        return "array bounds are not the interior plus a 2-point halo (an even wider one next to another strip)";
    if (d.px || d.py) return "periodic wrap";
    if (c.ffs != 1) return "full_free_surface != 1";
    if (d.xoff != XOFF) return "device layout without the fused column offset";
    const int nxa = d.nxa(), nya = d.nya();
    auto at = [&](const float *a, int m, int n) { return a[(size_t)(n - d.bnd_y1) * nxa + (m - d.bnd_x1)]; };
    if (d.nx_start != d.mmm || d.nx_end != d.mm) return "domain split along x (only row strips are supported)";
    const float *lu = masks[0];
    for (int n = d.bnd_y1; n <= d.bnd_y2; n++)
        for (int m = d.bnd_x1; m <= d.bnd_x2; m++) {
            float v = at(lu, m, n);
            if (v != 0.0f && v != 1.0f) return "lu is not 0/1";
            const bool row_ok = (n >= d.ny_start || open_s) && (n <= d.ny_end || open_n);
            bool interior = m >= d.nx_start && m <= d.nx_end && row_ok;
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
    // rows next to another strip carry that strip's masks: not compared
    for (int k = 0; k < 6; k++)
        for (int n = d.bnd_y1; n <= d.bnd_y2; n++) {
            if ((n < d.ny_start - 1 && open_s) || (n > d.ny_end && open_n)) continue;
            const size_t o = (size_t)(n - d.bnd_y1) * nxa;
            if (std::memcmp(ref[k].data() + o, masks[k + 1] + o, (size_t)nxa * sizeof(float)) != 0)
                return "derived masks differ from gridcon(lu)";
        }
    // metrics and Coriolis constant along rows over the points the step reads
    // (rows bnd_y1+1..bnd_y2-1: ny_start-1..ny_end+1 with a 2-row halo)
    for (int k = 0; k < 9; k++)
        for (int n = d.bnd_y1 + 1; n <= d.bnd_y2 - 1; n++) {
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
          const double *d_hrest, const float *d_lu, double *state[NSET], cudaStream_t s)
{
    release(p);
    p.prepared = false;
    p.staged_key = 0;
    const int nxa = d.nxa(), nya = d.nya();
    // metrics of the rows the step reads: bnd_y1+1..bnd_y2-1 (ny_start-1..
    // ny_end+1 with a 2-row halo); rows outside repeat the nearest
    auto row_of = [&](int k, int n) {
        n = std::min(std::max(n, d.bnd_y1 + 1), d.bnd_y2 - 1);
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
        if (n >= d.bnd_y1 + 1 && n <= d.bnd_y2 - 2 && (q.vt0 != 0.0 || q.vt1 != 0.0 || q.vt2 != 0.0)) vz = false;
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
        for (int n = d.bnd_y1 + 1; n <= d.bnd_y2 - 1 && p.uni; n++)
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
    // field-blocked sets: the caller's state block and two ping-pong sets
    p.fstride = d.pitch * nya;
    const size_t fb = (size_t)p.fstride * sizeof(double);
    for (int b = 0; b < 2; b++) {
        double *blk = nullptr;
        if (cudaMalloc(&blk, NSET * fb) != cudaSuccess) return 1;
        if (cudaMemsetAsync(blk, 0, NSET * fb, s) != cudaSuccess) return 1;
        for (int k = 0; k < NSET; k++) p.buf[b][k] = blk + k * p.fstride;
    }
    if (cudaMalloc(&p.stat, NSTAT * fb) != cudaSuccess) return 1;
    if (cudaMemsetAsync(p.stat, 0, NSTAT * fb, s) != cudaSuccess) return 1;
    if (cudaMemcpyAsync(p.stat + T_H * p.fstride, d_hrest, fb, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return 1;
    p.set[0] = state[0];
    p.set[1] = p.buf[0][0];
    p.set[2] = p.buf[1][0];
    EncodeTiled enc = encoder();
    if (!enc) return 1;
    for (int b = 0; b < 3; b++)
        if (encode_fields(enc, &p.tm_set[b], p.set[b], d, p.fstride, NSET, NSET)) return 1;
    if (encode_fields(enc, &p.tm_stat[0], p.stat, d, p.fstride, NSTAT, Layout<false>::NS)) return 1;
    if (encode_fields(enc, &p.tm_stat[1], p.stat, d, p.fstride, NSTAT, Layout<true>::NS)) return 1;
    p.stat_box[0] = Layout<false>::NS;
    p.stat_box[1] = Layout<true>::NS;

    if (cudaMalloc(&p.d_uniform, (size_t)MINMAX_BLOCKS * 6 * sizeof(double)) != cudaSuccess) return 1;
    if (cudaMalloc(&p.d_flags, sizeof(unsigned)) != cudaSuccess) return 1;
    if (cudaMemsetAsync(p.d_flags, 0, sizeof(unsigned), s) != cudaSuccess) return 1;
    p.lu = d_lu;
    p.buffers_synced = false;
    if (set_smem()) return 1;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    p.nsm = nsm;
    // one item table per variant for the plain substep and one for the
    // time-mean substeps, each one wave of the kernel's resident CTAs
    int occ[NTABLE] = {1, 1, 1, 1, 1};
    cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], k_substep<false, 3>, NL,
                                                                   ring_bytes<false, 3>());
    if (oe == cudaSuccess)
        oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], k_substep<true, 3>, NL, ring_bytes<true, 3>());
    if (oe == cudaSuccess)
        oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], k_substep<false, 5>, NL, ring_bytes<false, 5>());
    if (oe == cudaSuccess)
        oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[3], k_substep<true, 5>, NL, ring_bytes<true, 5>());
    if (oe == cudaSuccess)
        oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[4], k_substep<false, 3, true>, NL,
                                                           ring_bytes<false, 3, true>());
    if (oe != cudaSuccess) return 1;
    p.ocean = ocean_rows(p, d, masks[0]);
    for (int v = 0; v < NTABLE; v++) {
        p.occ[v] = occ[v] < 1 ? 1 : occ[v];
        if (upload_items(p, v, partition(p, d, item_waves(v) * nsm * p.occ[v], 0), s)) return 1;
    }
    p.rows_per_item[0] = p.rows_per_item[1] = 0;
    return 0;
}

int dynamics(Plan &p, const Dom &d, const Consts &c, double tau, int nstep, double *state[6], double *acc[4],
             double *forc[6], cudaStream_t s)
{
    Forcing f;
    p.staged_key = 0;
    if (forcing_mode(p, d, c, forc, s, f)) return 1;
    if (!p.buffers_synced && sync_buffers(p, state, s)) return 1;
    if (cudaMemsetAsync(p.d_flags, 0, sizeof(unsigned), s) != cudaSuccess) return 1;
    const size_t fb = (size_t)d.pitch * d.nya() * sizeof(double);
    for (int k = 0; k < 4; k++)
        if (cudaMemsetAsync(acc[k], 0, fb, s) != cudaSuccess) return 1;   // vel_ssh.f90:479-482
    const int gen = (p.uni && f.uniform) ? 0 : 1;
    if (stage_forcing(p, forc, gen, s)) return 1;
    Params q = base_params(p, d, c, f, gen);
    const double ti = tau / (double)nstep;
    set_times(q, 2.0 * ti, p);
    q.gam = c.ts / 2.0 / (double)nstep;
    for (int k = 0; k < 4; k++) q.acc[k] = acc[k];
    // The time means of vel_ssh.f90:549-550, :567-568 add (X(s-1) + X(s)) /
    // (4*nstep) in every substep s = 1..2*nstep, X being a transport or a
    // pressure-gradient term of a time level: that is X(0)/(4 nstep) +
    // sum_{s=1}^{2 nstep-1} X(s)/(2 nstep) + X(2 nstep)/(4 nstep).  The sums
    // are read and written in substep 1 (X(0)) and the even substeps
    // (X(s-1) + X(s), the last one's X(s) with half the weight) only; the
    // odd substeps after the first run the plain kernel.  Same sum, a
    // different rounding order, half the time-mean traffic.
    const double c2 = 1.0 / (double)(2 * nstep), c4 = 1.0 / (double)(4 * nstep);
    // (every odd substep writes the state: only the last, even one does not)
    auto mode_of = [&](int st, bool write) {
        if (st == 1) { q.ca = c4; q.cb = 0.0; return 4; }
        if (st & 1) return 3;
        q.ca = c2;
        q.cb = st == 2 * nstep ? c4 : c2;
        return write ? 5 : 2;
    };
    // substeps 1..nstep ping-pong between state[] and buf[0]; the state
    // after substep nstep (vel_ssh.f90:638-648) is then swapped into state[]
    for (int step = 1; step <= nstep; step++) {
        const bool odd = step & 1;
        if (set_io(p, q, odd ? state : p.buf[0], odd ? p.buf[0] : state)) return 1;
        if (launch(p, q, gen, mode_of(step, true), s) || cudaGetLastError() != cudaSuccess) return 1;
    }
    if (nstep & 1)
        for (int k = 0; k < 6; k++) std::swap(state[k], p.buf[0][k]);
    // substeps nstep+1..2*nstep feed only the time means: state[] -> buf[0],
    // then buf[0] <-> buf[1]; the last one writes no state
    for (int k2 = 1; k2 <= nstep; k2++) {
        double *const *src = k2 == 1 ? state : ((k2 & 1) ? p.buf[1] : p.buf[0]);
        double *const *dst = (k2 & 1) ? p.buf[0] : p.buf[1];
        if (set_io(p, q, src, dst)) return 1;
        if (launch(p, q, gen, mode_of(nstep + k2, k2 < nstep), s) || cudaGetLastError() != cudaSuccess) return 1;
    }
    unsigned flags = 0;
    if (read_flags(p, s, &flags)) return 1;
    p.last_flags = flags;
    return 0;
}

int run_substeps(Plan &p, const Dom &d, const Consts &c, int nsub, double dt, const double *rhs_scale,
                 double *state[6], double *forc[6], cudaStream_t s)
{
    if (p.f32) {
        // FP32 velocity storage: u, up, v, vp of the state and ping-pong
        // sets in FP32 for the run, SSH in the FP64 sets
        const int rc = prepare_steps_f32(p, d, c, state, forc, s);
        if (rc) return rc;
        if (launch_steps_f32(p, d, c, dt, nsub, nullptr, nullptr, rhs_scale, state, s)) return 1;
        return finish_steps_f32(p, d, state, s);
    }
    Forcing f;
    p.staged_key = 0;
    if (forcing_mode(p, d, c, forc, s, f)) return 1;
    if (!p.buffers_synced && sync_buffers(p, state, s)) return 1;
    if (cudaMemsetAsync(p.d_flags, 0, sizeof(unsigned), s) != cudaSuccess) return 1;
    const int gen = (p.uni && f.uniform) ? 0 : 1;
    if (stage_forcing(p, forc, gen, s)) return 1;
    Params q = base_params(p, d, c, f, gen);
    set_times(q, 2.0 * dt, p);
    q.gam = c.ts / 2.0;   // nstep = 1
    for (int k = 0; k < 4; k++) q.acc[k] = nullptr;
    for (int step = 0; step < nsub; step++) {
        if (set_io(p, q, (step & 1) ? p.buf[0] : state, (step & 1) ? state : p.buf[0])) return 1;
        q.rhs_scale = rhs_scale ? rhs_scale[step] : 1.0;
        if (launch(p, q, gen, 3, s) || cudaGetLastError() != cudaSuccess) return 1;
    }
    if (nsub & 1)
        for (int k = 0; k < 6; k++) std::swap(state[k], p.buf[0][k]);
    unsigned flags = 0;
    if (read_flags(p, s, &flags)) return 1;
    p.last_flags = flags;
    return 0;
}

int prepare_steps_f32(Plan &p, const Dom &d, const Consts &c, double *state[6], double *forc[6], cudaStream_t s,
                      unsigned key)
{
    if (prepare_steps(p, d, c, state, forc, s, key)) return 1;
    if (p.prep_gen) return 2;
    if (ensure_f32(p, d, s)) return 1;
    const int blocks = 4 * p.nsm;
    const int a = set_index(p, state[0]), b = set_index(p, p.buf[0][0]);
    if (a < 0 || b < 0) return 1;
    // the state's velocities every run (the FP64 state may have changed);
    // the partner set's only for the values at the points the kernel does
    // not write, once after they were synchronised; RHSx, RHSy once per
    // staging of the forcing
    k_to_f32<<<blocks, 256, 0, s>>>(p.set[a], p.vset[a], 4 * p.fstride);
    p.f32_land[a] = true;
    if (!p.f32_land[b]) {
        k_to_f32<<<blocks, 256, 0, s>>>(p.set[b], p.vset[b], 4 * p.fstride);
        p.f32_land[b] = true;
    }
    if (key == 0 || p.f32_rhs_key != key) {
        k_to_f32<<<blocks, 256, 0, s>>>(p.stat + T_RX * p.fstride, p.stat32, 2 * p.fstride);
        p.f32_rhs_key = key;
    }
    return cudaGetLastError() != cudaSuccess;
}

int launch_steps_f32(Plan &p, const Dom &d, const Consts &c, double dt, int nsteps, const double *rs_dev,
                     const int *rs_base, const double *rs_host, double *state[6], cudaStream_t s)
{
    if (!p.prepared || p.prep_gen) return 1;
    // the ring's static segment holds Layout<false, true>::NS fields: the
    // map must bring exactly that many
    if (p.stat_box_f32 != Layout<false, true>::NS) return 1;
    Forcing f{true, p.prep_mu0, p.prep_rd0, p.prep_wq0};
    Params q = base_params(p, d, c, f, 0);
    set_times(q, 2.0 * dt, p);
    q.gam = c.ts / 2.0;   // nstep = 1
    for (int k = 0; k < 4; k++) q.acc[k] = nullptr;
    q.tm_rhs = p.tm_rhs32;
    q.tm_stat = p.tm_stat_f32;
    q.items = p.items[TABLE_F32];
    q.rs_dev = rs_dev;
    q.rs_base = rs_base;
    const int a = set_index(p, state[0]), b = set_index(p, p.buf[0][0]);
    if (a < 0 || b < 0) return 1;
    for (int step = 0; step < nsteps; step++) {
        const int si = (step & 1) ? b : a, di = (step & 1) ? a : b;
        q.tm_src = p.tm_vel[si];
        q.tm_ssh = p.tm_ssh[si];
        for (int k = 0; k < NSET; k++) q.dst[k] = p.set[di] + k * p.fstride;
        for (int k = 0; k < 4; k++) q.vdst[k] = p.vset[di] + k * p.fstride;
        q.rhs_scale = rs_host ? rs_host[step] : 1.0;
        q.rs_k = step;
        p.last_variant = 2;
        launch_substep<false, 3, true>(p.nitems[TABLE_F32], q, s);
        if (cudaGetLastError() != cudaSuccess) return 1;
    }
    if (nsteps & 1)
        for (int k = 0; k < 6; k++) std::swap(state[k], p.buf[0][k]);
    return 0;
}

int finish_steps_f32(Plan &p, const Dom &d, double *state[6], cudaStream_t s)
{
    const int fi = set_index(p, state[0]);
    if (fi < 0) return 1;
    const int c0 = d.nx_start - d.bnd_x1 + d.xoff, c1 = d.nx_end - d.bnd_x1 + d.xoff;
    const int r0 = d.ny_start - d.bnd_y1, r1 = d.ny_end - d.bnd_y1;
    if (c1 >= c0 && r1 >= r0) {
        const dim3 grid((unsigned)((c1 - c0 + 1 + 127) / 128), (unsigned)std::min(r1 - r0 + 1, 65535));
        k_vel_from_f32<<<grid, 128, 0, s>>>(p.vset[fi], p.set[fi], p.lu, d.pitch, p.fstride, r0, r1, c0, c1);
        if (cudaGetLastError() != cudaSuccess) return 1;
    }
    return finish_steps(p, s);
}

int repartition(Plan &p, const Dom &d, int rows_per_item, cudaStream_t s)
{
    for (int v = 0; v < NTABLE; v++) {
        p.rows_per_item[v & 1] = rows_per_item;
        if (upload_items(p, v, partition(p, d, item_waves(v) * p.nsm * p.occ[v], rows_per_item), s)) return 1;
    }
    return 0;
}

int prepare_steps(Plan &p, const Dom &d, const Consts &c, double *state[6], double *forc[6], cudaStream_t s,
                  unsigned key)
{
    if (!p.buffers_synced && sync_buffers(p, state, s)) return 1;
    if (cudaMemsetAsync(p.d_flags, 0, sizeof(unsigned), s) != cudaSuccess) return 1;
    // the forcing fields are unchanged since the last preparation with
    // this key: their classification and the staged copies still hold
    if (key != 0 && key == p.staged_key && p.prepared) return 0;
    p.staged_key = 0;
    Forcing f;
    if (forcing_mode(p, d, c, forc, s, f)) return 1;
    const int gen = (p.uni && f.uniform) ? 0 : 1;
    if (stage_forcing(p, forc, gen, s)) return 1;
    p.prep_gen = gen;
    p.prep_mu0 = f.mu0;
    p.prep_rd0 = f.rd0;
    p.prep_wq0 = f.wq0;
    p.prepared = true;
    p.staged_key = key;
    return 0;
}

int launch_steps(Plan &p, const Dom &d, const Consts &c, double dt, int nsteps, const double *rs_dev,
                 const int *rs_base, double *state[6], cudaStream_t s, double rs_host)
{
    if (!p.prepared) return 1;
    Forcing f{true, p.prep_mu0, p.prep_rd0, p.prep_wq0};
    const int gen = p.prep_gen;
    Params q = base_params(p, d, c, f, gen);
    set_times(q, 2.0 * dt, p);
    q.gam = c.ts / 2.0;   // nstep = 1
    for (int k = 0; k < 4; k++) q.acc[k] = nullptr;
    q.rs_dev = rs_dev;
    q.rs_base = rs_base;
    q.rhs_scale = rs_host;
    for (int step = 0; step < nsteps; step++) {
        if (set_io(p, q, (step & 1) ? p.buf[0] : state, (step & 1) ? state : p.buf[0])) return 1;
        q.rs_k = step;
        if (launch(p, q, gen, 3, s) || cudaGetLastError() != cudaSuccess) return 1;
    }
    if (nsteps & 1)
        for (int k = 0; k < 6; k++) std::swap(state[k], p.buf[0][k]);
    return 0;
}

namespace {
// the plain-substep items over device rows extended es rows south and en
// rows north of the interior, built (and kept) on first use; nullptr if
// the halo is too narrow for them (the kernel reads two rows below and two
// above the rows it computes)
const Plan::ExtTable *ext_table(Plan &p, const Dom &d, int gen, int es, int en, cudaStream_t s)
{
    for (const auto &t : p.ext)
        if (t.gen == gen && t.s == es && t.n == en) return &t;
    const int rf = d.ny_start - d.bnd_y1 - es, rl = d.ny_end - d.bnd_y1 + en;
    if (es < 0 || en < 0 || rf < 2 || rl + 2 > d.nya() - 1) return nullptr;
    const std::vector<int4> items = partition(p, d, item_waves(gen) * p.nsm * p.occ[gen], 0, rf, rl);
    Plan::ExtTable t{gen, es, en, (int)items.size(), nullptr};
    if (cudaMalloc(&t.items, items.size() * sizeof(int4)) != cudaSuccess) return nullptr;
    p.ext.push_back(t);   // owned by the plan from here on (freed by release)
    if (cudaMemcpyAsync(t.items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return nullptr;
    return &p.ext.back();
}
}  // namespace

int launch_step_ext(Plan &p, const Dom &d, const Consts &c, double dt, int ext_s, int ext_n, double *state[6],
                    cudaStream_t s, double rs_host)
{
    if (!p.prepared) return 1;
    if (ext_s == 0 && ext_n == 0) return launch_steps(p, d, c, dt, 1, nullptr, nullptr, state, s, rs_host);
    const int gen = p.prep_gen;
    if (p.stat_box[gen] != (gen ? Layout<true>::NS : Layout<false>::NS)) return 1;
    const Plan::ExtTable *t = ext_table(p, d, gen, ext_s, ext_n, s);
    if (!t) return 1;
    Forcing f{true, p.prep_mu0, p.prep_rd0, p.prep_wq0};
    Params q = base_params(p, d, c, f, gen);
    set_times(q, 2.0 * dt, p);
    q.gam = c.ts / 2.0;   // nstep = 1
    for (int k = 0; k < 4; k++) q.acc[k] = nullptr;
    q.rhs_scale = rs_host;
    if (set_io(p, q, state, p.buf[0])) return 1;
    q.items = t->items;
    p.last_variant = gen;
    if (gen) launch_substep<true, 3>(t->nitems, q, s);
    else launch_substep<false, 3>(t->nitems, q, s);
    if (cudaGetLastError() != cudaSuccess) return 1;
    for (int k = 0; k < 6; k++) std::swap(state[k], p.buf[0][k]);
    return 0;
}

int ens_table(const std::vector<EnsMemberIn> &mem, int group, const double *rs_dev, const int *rs_base, EnsTable &t,
              cudaStream_t s)
{
    ens_free(t);
    if (mem.empty() || group < 2 || group % 2) return 1;
    std::vector<EnsItem> h(mem.size());
    int total = 0;
    for (size_t i = 0; i < mem.size(); i++) {
        Plan &p = *mem[i].p;
        if (!p.prepared) return 1;
        const int gen = p.prep_gen;
        if (p.stat_box[gen] != (gen ? Layout<true>::NS : Layout<false>::NS)) return 1;
        Forcing f{true, p.prep_mu0, p.prep_rd0, p.prep_wq0};
        for (int par = 0; par < 2; par++) {
            Params q = base_params(p, *mem[i].d, *mem[i].c, f, gen);
            set_times(q, 2.0 * mem[i].dt, p);
            q.gam = mem[i].c->ts / 2.0;   // nstep = 1
            for (int k = 0; k < 4; k++) q.acc[k] = nullptr;
            q.rs_dev = rs_dev;
            q.rs_base = rs_base;
            q.rhs_scale = 1.0;
            double *const *state = mem[i].state;
            if (set_io(p, q, par ? p.buf[0] : state, par ? state : p.buf[0])) return 1;
            q.items = p.items[gen];
            h[i].q[par] = q;
        }
        h[i].items = p.items[gen];
        h[i].nitems = p.nitems[gen];
        h[i].gen = gen;
        total += p.nitems[gen];
    }
    // claim order within a substep: member after member, each member's items
    // in table order (strip after strip).  Interleaving the members' items
    // (item k of member i at phase i / nmem + (k + 1/2) / n_i, modulo 1, so
    // that the items in flight spread over all members) ran 26 % slower on
    // 64 regional basins: neighbouring items of one member share rows in L2
    std::vector<int2> order;
    order.reserve((size_t)total);
    for (size_t i = 0; i < h.size(); i++)
        for (int k = 0; k < h[i].nitems; k++) order.push_back(make_int2((int)i, k));
    bool anygen = false;
    for (const EnsItem &e : h) anygen = anygen || e.gen;
    const size_t smem = anygen ? ring_bytes<true, 3>() : ring_bytes<false, 3>();
    const void *kern = anygen ? (const void *)k_ens_persistent<true> : (const void *)k_ens_persistent<false>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 1;
    int occ = 0, dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NL, smem) != cudaSuccess || occ < 1)
        return 1;
    EnsItem *dm = nullptr;
    if (cudaMalloc(&dm, h.size() * sizeof(EnsItem)) != cudaSuccess) return 1;
    t.d_mem = dm;
    if (cudaMalloc(&t.d_order, order.size() * sizeof(int2)) != cudaSuccess ||
        cudaMalloc(&t.d_ctr, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&t.d_done, mem.size() * (size_t)group * sizeof(unsigned)) != cudaSuccess)
        return 1;
    if (cudaMemcpyAsync(dm, h.data(), h.size() * sizeof(EnsItem), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(t.d_order, order.data(), order.size() * sizeof(int2), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)   // the host vectors go out of scope
        return 1;
    t.nmem = (int)mem.size();
    t.total = total;
    t.group = group;
    t.grid = occ * nsm;
    t.anygen = anygen;
    t.smem = smem;
    return 0;
}

int ens_launch(const EnsTable &t, cudaStream_t s)
{
    if (!t.d_mem) return 1;
    if (cudaMemsetAsync(t.d_ctr, 0, sizeof(unsigned), s) != cudaSuccess ||
        cudaMemsetAsync(t.d_done, 0, (size_t)t.nmem * t.group * sizeof(unsigned), s) != cudaSuccess)
        return 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(t.grid);
    cfg.blockDim = dim3(NL);
    cfg.dynamicSmemBytes = t.smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;   // every CTA resident: the completion waits end
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, t.anygen ? k_ens_persistent<true> : k_ens_persistent<false>,
                              (const EnsItem *)t.d_mem, (const int2 *)t.d_order, t.total, t.group, t.d_ctr,
                              t.d_done) != cudaSuccess;
}

void ens_free(EnsTable &t)
{
    cudaFree(t.d_mem);
    cudaFree(t.d_order);
    cudaFree(t.d_ctr);
    cudaFree(t.d_done);
    t = EnsTable{};
}

int finish_steps(Plan &p, cudaStream_t s)
{
    unsigned flags = 0;
    if (read_flags(p, s, &flags)) return 1;
    p.last_flags = flags;
    return 0;
}

void free_plan(Plan &p)
{
    release(p);
    p = Plan{};
}

}  // namespace fused
}  // namespace inmsom
