// Training gradient of the closure MLP (45 -> 64 -> 64 -> 2, GELU, mean
// squared error) on the fifth-generation tensor cores: tcgen05.mma with
// BF16 operands in shared memory and FP32 accumulators in tensor memory.
// No counterpart in the reference (the closure stands in for the Laplacian
// viscosity of uv_diff2, Function/vel_ssh.f90:117-184, on coarse grids).
//
// One CTA of sixteen warps per SM, persistent over tiles of 128 samples.
// Warp w reads tensor-memory lanes 32 (w % 4) .. +31 (the lane quarter it
// may access), so each thread owns one sample (its lane) and 16 of the 64
// columns of every layer's output (w / 4 picks which); the next tile's
// inputs are fetched while a tile computes.  One thread issues the MMAs.
// Per tile:
//   forward   Z1 = X W1, A1 = GELU(Z1 + b1); Z2 = A1 W2, A2 = GELU(Z2 + b2);
//             O = A2 W3 (+ b3)                        (M = 128 samples)
//   backward  D3 = 2 (O - T) / (batch * 2); DA2 = D3 W3^T;
//             DZ2 = DA2 * GELU'(Z2 + b2); DA1 = DZ2 W2^T;
//             DZ1 = DA1 * GELU'(Z1 + b1)               (M = 128 samples)
//   weights   dW3 += A2^T D3, dW2 += A1^T DZ2, dW1 += X^T DZ1
//             (M = the layer's inputs, K = the tile's samples), accumulated
//             in tensor memory over all tiles of the CTA.
// The bias gradients come out of the same weight-gradient products: X, A1
// and A2 carry a column of ones (X column 48, A1/A2 column 64), whose row
// of dW is the column sum of the layer's output gradient.
//
// Shared-memory operands use the no-swizzle canonical layout of the
// tensor-core descriptors: 8 x 16-byte core matrices, element (r, c) of an
// R x C tile at ((r / 8) * (C / 8) + c / 8) * 128 + (r % 8) * 16 +
// (c % 8) * 2 bytes.  Read with rows as M/N and columns as K (K-major) it
// is the forward operand; read with columns as M/N and rows as K (MN-major)
// the same bytes are its transpose, so no tile is ever transposed.
//
// Every mbarrier wait is bounded; a wait that gives up makes the CTA's
// partial sums NaN (the gradient and the loss come out NaN), and the CTA
// frees its tensor memory and returns.
#include "inmsom_gpu.h"
#include "closure.h"
#include "gelu.cuh"

#include <cuda_bf16.h>

#include <cstdint>

namespace {

using namespace inmsom::closure;

constexpr int KIN = 48, HID = 64, NOUT = 2, N3 = 8;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + KIN * HID, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
              OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID * N3, NPARAM = OFF_B3 + N3;
constexpr int BOFF_W1 = 0, BOFF_W2 = KIN * HID, BOFF_W3 = BOFF_W2 + HID * HID;
static_assert(NPARAM == INMSOM_MLP_NPARAM, "parameter block size");
constexpr int NPART = NPARAM + 1;
constexpr int TILE = 128, THREADS = 512;
constexpr int SLICE = 16;                 // columns of a 64-column block per thread (4 warps per lane quarter)
constexpr int NO = 16;                    // output columns of the MMAs (2 used)
constexpr int XC = 64, AC = 128;          // columns of the X and A1/A2 tiles (data, a ones column, zeros)
constexpr unsigned WAIT_POLLS = 1u << 24;

// tensor-memory columns (512 allocated: one CTA per SM)
constexpr uint32_t TM_COLS = 512;
constexpr uint32_t C_Z1 = 0, C_Z2 = 64, C_O = 128, C_DA2 = 144, C_DA1 = 208, C_DW1 = 272, C_DW2 = 336,
                   C_DW3 = 400;
static_assert(C_DW3 + NO <= TM_COLS, "tensor-memory columns");

struct __align__(128) Smem {
    __nv_bfloat16 w1t[HID * XC];     // W1^T: rows = 64 outputs, columns = 48 inputs (+16 unused)
    __nv_bfloat16 w2t[HID * HID];    // W2^T
    __nv_bfloat16 w3t[NO * HID];     // W3^T: rows = 16 outputs (2 used)
    __nv_bfloat16 x[TILE * XC];      // inputs, column 48 = 1
    __nv_bfloat16 a1[TILE * AC];     // GELU(Z1 + b1), column 64 = 1
    __nv_bfloat16 a2[TILE * AC];
    __nv_bfloat16 d3[TILE * NO];
    __nv_bfloat16 dz2[TILE * HID];
    __nv_bfloat16 dz1[TILE * HID];
    float b1[HID], b2[HID], b3[NO];
    float loss[4];
    uint64_t mbar;
    uint32_t tmem_base;
    int gave_up;
};

// element (r, c) of an R x C tile with C columns, in elements
__device__ __forceinline__ int blk(int r, int c, int C) { return ((r >> 3) * (C >> 3) + (c >> 3)) * 64 + (r & 7) * 8 + (c & 7); }

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle: lbo / sbo in bytes
__device__ __forceinline__ uint64_t sdesc(const void *p, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr(p) >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: BF16 A and B, FP32 D
__host__ __device__ constexpr uint32_t idesc(int M, int N, bool a_mn, bool b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(id), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ bool wait_bar(uint64_t *bar, uint32_t parity)
{
    for (unsigned i = 0; i < WAIT_POLLS; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(saddr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    wait_ld();
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// 2 x 16 consecutive FP32 columns of this thread's lane (two blocks of
// tensor memory), both loads in flight before one wait; the registers are
// operands of the wait, so nothing reads them before it
__device__ __forceinline__ void ld16x2(uint32_t ta, uint32_t tb, float (&a)[16], float (&b)[16])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(ta));
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(tb));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) {
        a[k] = __uint_as_float(r[k]);
        b[k] = __uint_as_float(r[16 + k]);
    }
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// 8 consecutive values as one 16-byte chunk of row r of a tile
__device__ __forceinline__ void st_chunk(__nv_bfloat16 *tile, int r, int c0, int C, const float *v)
{
    const uint4 q = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
    *reinterpret_cast<uint4 *>(tile + blk(r, c0, C)) = q;
}

// all threads: smem writes visible to the tensor cores, tensor-memory reads
// done, then one barrier
__device__ __forceinline__ void handoff()
{
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
}

__global__ void __launch_bounds__(THREADS, 1)
    k_mlp_grad_tc(const __nv_bfloat16 *__restrict__ x, const float *__restrict__ tgt, const int *__restrict__ idx,
                  int batch, const float *__restrict__ prm, const __nv_bfloat16 *__restrict__ wb,
                  float *__restrict__ partial)
{
    extern __shared__ __align__(1024) unsigned char raw[];
    Smem &s = *reinterpret_cast<Smem *>(raw);
    const int t = threadIdx.x, w = t >> 5, q = w & 3, cs = w >> 2;
    const int r = 32 * q + (t & 31);       // this thread's sample row and tensor-memory lane
    const int c0 = SLICE * cs;             // its columns of a 64-column block
    const bool issuer = t == 0;

    if (issuer) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&s.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s.gave_up = 0;
    }
    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&s.tmem_base)),
                     "r"(TM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // weights transposed into the K-major operands: 16-byte reads of 8
    // consecutive outputs of one input row of the [in][out] layout, all
    // issued before any is stored; biases, constant columns
    {
        constexpr int N1 = KIN * HID / 8, N2 = HID * HID / 8, NW3 = HID * N3 / 8;   // 16-byte pieces
        static_assert(N1 <= THREADS && N2 <= THREADS && NW3 <= THREADS, "one piece per thread");
        const uint4 *w16 = reinterpret_cast<const uint4 *>(wb);
        uint4 p1 = make_uint4(0u, 0u, 0u, 0u), p2 = p1, p3 = p1;
        if (t < N1) p1 = w16[(BOFF_W1 / 8) + t];
        if (t < N2) p2 = w16[(BOFF_W2 / 8) + t];
        if (t < NW3) p3 = w16[(BOFF_W3 / 8) + t];
        auto put = [&](__nv_bfloat16 *dst, int C, int k, int o0, const uint4 &v) {
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
            for (int j = 0; j < 8; j++) dst[blk(o0 + j, k, C)] = e[j];
        };
        if (t < N1) put(s.w1t, XC, t / (HID / 8), 8 * (t % (HID / 8)), p1);
        if (t < N2) put(s.w2t, HID, t / (HID / 8), 8 * (t % (HID / 8)), p2);
        if (t < NW3) put(s.w3t, HID, t, 0, p3);   // W3 row k = t: outputs 0..7
        // W1^T columns 48..63 and W3^T rows 8..15 are zero
        for (int i = t; i < HID * (XC - KIN); i += THREADS)
            s.w1t[blk(i / (XC - KIN), KIN + i % (XC - KIN), XC)] = __float2bfloat16(0.f);
        for (int i = t; i < (NO - N3) * HID; i += THREADS)
            s.w3t[blk(N3 + i / HID, i % HID, HID)] = __float2bfloat16(0.f);
    }
    if (t < HID) {
        s.b1[t] = prm[OFF_B1 + t];
        s.b2[t] = prm[OFF_B2 + t];
    }
    if (t < NO) s.b3[t] = t < N3 ? prm[OFF_B3 + t] : 0.f;
    if (cs == 0) {
        float one[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, zero[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        st_chunk(s.x, r, 48, XC, one);
        st_chunk(s.x, r, 56, XC, zero);
        for (int c = 64; c < AC; c += 8) {
            st_chunk(s.a1, r, c, AC, c == 64 ? one : zero);
            st_chunk(s.a2, r, c, AC, c == 64 ? one : zero);
        }
        st_chunk(s.d3, r, 8, NO, zero);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tb = s.tmem_base;
    const uint32_t lane = tb + ((uint32_t)(32 * q) << 16);   // this warp's lane quarter
    const float scale = 2.0f / ((float)batch * NOUT);
    const int ntiles = batch / TILE;
    uint32_t ph = 0;
    float lsum = 0.f;
    bool ok = true, first = true;

    // one commit of the issuer's MMAs, waited for by every thread
    auto sync_mma = [&]() -> bool {
        if (issuer) commit(&s.mbar);
        const bool got = wait_bar(&s.mbar, ph);
        ph ^= 1u;
        if (!got) s.gave_up = 1;
        __syncthreads();
        fence_after();
        return s.gave_up == 0;
    };
    // this thread's part of a sample: 16-byte chunks cs and cs + 4 (of 6),
    // and (slice 0) the two targets
    uint4 xa = make_uint4(0u, 0u, 0u, 0u), xb = xa;
    float t0 = 0.f, t1 = 0.f;
    auto fetch = [&](int tile) {
        if (tile >= ntiles) return;
        const long long row = idx ? (long long)idx[tile * TILE + r] : (long long)tile * TILE + r;
        const uint4 *src = reinterpret_cast<const uint4 *>(x + row * KIN);
        xa = src[cs];
        if (cs + 4 < 6) xb = src[cs + 4];
        if (cs == 0) {
            t0 = tgt[row * NOUT];
            t1 = tgt[row * NOUT + 1];
        }
    };
    fetch(blockIdx.x);

    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        // ---- this tile's samples into X; the next tile's are fetched while
        // this one computes
        *reinterpret_cast<uint4 *>(s.x + blk(r, 8 * cs, XC)) = xa;
        if (cs + 4 < 6) *reinterpret_cast<uint4 *>(s.x + blk(r, 8 * (cs + 4), XC)) = xb;
        const float tg0 = t0, tg1 = t1;
        handoff();
        fetch(tile + gridDim.x);
        // ---- Z1 = X W1 (K = 48)
        if (issuer)
            for (int ks = 0; ks < 3; ks++)
                mma(tb + C_Z1, sdesc(s.x + 128 * ks, 128, 1024), sdesc(s.w1t + 128 * ks, 128, 1024),
                    idesc(128, 64, false, false), ks > 0);
        if (!(ok = sync_mma())) break;
        {
            float z[16];
            ld16(lane + C_Z1 + c0, z);
#pragma unroll
            for (int k = 0; k < 16; k++) z[k] = gelu(z[k] + s.b1[c0 + k]);
            st_chunk(s.a1, r, c0, AC, z);
            st_chunk(s.a1, r, c0 + 8, AC, z + 8);
        }
        handoff();
        // ---- Z2 = A1 W2 (K = 64)
        if (issuer)
            for (int ks = 0; ks < 4; ks++)
                mma(tb + C_Z2, sdesc(s.a1 + 128 * ks, 128, 2048), sdesc(s.w2t + 128 * ks, 128, 1024),
                    idesc(128, 64, false, false), ks > 0);
        if (!(ok = sync_mma())) break;
        {
            float z[16];
            ld16(lane + C_Z2 + c0, z);
#pragma unroll
            for (int k = 0; k < 16; k++) z[k] = gelu(z[k] + s.b2[c0 + k]);
            st_chunk(s.a2, r, c0, AC, z);
            st_chunk(s.a2, r, c0 + 8, AC, z + 8);
        }
        handoff();
        // ---- O = A2 W3 (N = 16, 2 used)
        if (issuer)
            for (int ks = 0; ks < 4; ks++)
                mma(tb + C_O, sdesc(s.a2 + 128 * ks, 128, 2048), sdesc(s.w3t + 128 * ks, 128, 1024),
                    idesc(128, NO, false, false), ks > 0);
        if (!(ok = sync_mma())) break;
        if (cs == 0) {
            float o[16];
            ld16(lane + C_O, o);
            const float e0 = o[0] + s.b3[0] - tg0, e1 = o[1] + s.b3[1] - tg1;
            lsum += e0 * e0 + e1 * e1;
            float d[8] = {scale * e0, scale * e1, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            st_chunk(s.d3, r, 0, NO, d);
        }
        handoff();
        // ---- DA2 = D3 W3^T (K = 16); dW3 += A2^T D3 (M = 128 columns of A2, K = 128 samples)
        if (issuer) {
            mma(tb + C_DA2, sdesc(s.d3, 128, 256), sdesc(s.w3t, 1024, 128), idesc(128, 64, false, true), 0);
            for (int ks = 0; ks < 8; ks++)
                mma(tb + C_DW3, sdesc(s.a2 + ks * 16 * AC, 2048, 128), sdesc(s.d3 + ks * 16 * NO, 256, 128),
                    idesc(128, NO, true, true), !(first && ks == 0));
        }
        if (!(ok = sync_mma())) break;
        {
            float da[16], z[16];
            ld16x2(lane + C_DA2 + c0, lane + C_Z2 + c0, da, z);
#pragma unroll
            for (int k = 0; k < 16; k++)
                da[k] *= gelu_d(z[k] + s.b2[c0 + k]);
            st_chunk(s.dz2, r, c0, HID, da);
            st_chunk(s.dz2, r, c0 + 8, HID, da + 8);
        }
        handoff();
        // ---- DA1 = DZ2 W2^T (K = 64); dW2 += A1^T DZ2
        if (issuer) {
            for (int ks = 0; ks < 4; ks++)
                mma(tb + C_DA1, sdesc(s.dz2 + 128 * ks, 128, 1024), sdesc(s.w2t + ks * 16 * HID, 1024, 128),
                    idesc(128, 64, false, true), ks > 0);
            for (int ks = 0; ks < 8; ks++)
                mma(tb + C_DW2, sdesc(s.a1 + ks * 16 * AC, 2048, 128), sdesc(s.dz2 + ks * 16 * HID, 1024, 128),
                    idesc(128, 64, true, true), !(first && ks == 0));
        }
        if (!(ok = sync_mma())) break;
        {
            float da[16], z[16];
            ld16x2(lane + C_DA1 + c0, lane + C_Z1 + c0, da, z);
#pragma unroll
            for (int k = 0; k < 16; k++)
                da[k] *= gelu_d(z[k] + s.b1[c0 + k]);
            st_chunk(s.dz1, r, c0, HID, da);
            st_chunk(s.dz1, r, c0 + 8, HID, da + 8);
        }
        handoff();
        // ---- dW1 += X^T DZ1 (M = 64 columns of X)
        if (issuer)
            for (int ks = 0; ks < 8; ks++)
                mma(tb + C_DW1, sdesc(s.x + ks * 16 * XC, 1024, 128), sdesc(s.dz1 + ks * 16 * HID, 1024, 128),
                    idesc(64, 64, true, true), !(first && ks == 0));
        if (!(ok = sync_mma())) break;
        first = false;
    }

    if (ok && !first) {
        float *out = partial + (size_t)blockIdx.x * NPART;
        {
            // dW1: M = 64 rows in lanes 32 q + (0..15) of quarter q: row 16 q + lane
            const int lr = t & 31, m64 = 16 * q + lr;
            float v[16];
            ld16(lane + C_DW1 + c0, v);
            if (lr < 16) {
                if (m64 < KIN)
                    for (int k = 0; k < 16; k++) out[OFF_W1 + m64 * HID + c0 + k] = v[k];
                else if (m64 == KIN)
                    for (int k = 0; k < 16; k++) out[OFF_B1 + c0 + k] = v[k];
            }
        }
        {
            float v[16];
            ld16(lane + C_DW2 + c0, v);
            if (r < HID)
                for (int k = 0; k < 16; k++) out[OFF_W2 + r * HID + c0 + k] = v[k];
            else if (r == HID)
                for (int k = 0; k < 16; k++) out[OFF_B2 + c0 + k] = v[k];
        }
        if (cs == 0) {
            float v[16];
            ld16(lane + C_DW3, v);
            if (r < HID)
                for (int k = 0; k < N3; k++) out[OFF_W3 + r * N3 + k] = v[k];
            else if (r == HID)
                for (int k = 0; k < N3; k++) out[OFF_B3 + k] = v[k];
#pragma unroll
            for (int m = 16; m > 0; m >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, m);
            if ((t & 31) == 0) s.loss[q] = lsum;
        }
        __syncthreads();
        if (t == 0) out[NPARAM] = (s.loss[0] + s.loss[1]) + (s.loss[2] + s.loss[3]);
    }
    if (!ok) {
        // a wait gave up: the CTA's partial sums are NaN (so the gradient
        // and the loss are), and the MMAs of the step that timed out are
        // waited for (bounded) before the tensor memory is freed
        float *out = partial + (size_t)blockIdx.x * NPART;
        for (int i = t; i < NPART; i += THREADS) out[i] = __int_as_float(0x7fc00000);
        if (issuer) (void)wait_bar(&s.mbar, ph ^ 1u);
    }
    fence_before();
    __syncthreads();
    if (w == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tb), "r"(TM_COLS) : "memory");
    }
}

}  // namespace

namespace inmsom {
namespace closure {

// the operand tiles plus 24 KB of slack after them, so that no descriptor
// can reach past the CTA's shared memory
size_t grad_tc_smem() { return sizeof(Smem) + 24 * 1024; }

int grad_tc(const void *x, const float *targets, const int *idx, int batch, const float *params, const void *wbf16,
            float *partial, int grid, cudaStream_t s)
{
    k_mlp_grad_tc<<<grid, THREADS, grad_tc_smem(), s>>>((const __nv_bfloat16 *)x, targets, idx, batch, params,
                                                       (const __nv_bfloat16 *)wbf16, partial);
    return cudaGetLastError() != cudaSuccess;
}

int grad_tc_setup()
{
    return cudaFuncSetAttribute(k_mlp_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_tc_smem()) !=
           cudaSuccess;
}

}  // namespace closure
}  // namespace inmsom
