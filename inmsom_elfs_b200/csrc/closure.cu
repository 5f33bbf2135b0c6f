// Learned subgrid momentum closure: a 45 -> 64 -> 64 -> 2 MLP with GELU,
// BF16 weights and activations on the tensor cores (FP32 accumulate), FP32
// master weights and Adam.  Inference (fused into the step's forcing, and
// on feature rows) chains the layers through registers with mma.sync
// m16n8k16; the training gradient is closure_tc.cu's tcgen05 kernel.  No counterpart in the
// reference: it stands in for the Laplacian viscosity of uv_diff2
// (Function/vel_ssh.f90:117-184) on coarse grids.
//
// Parameter block (FP32, flat): W1[48][64] b1[64] W2[64][64] b2[64]
// W3[64][8] b3[8]; rows 45..47 of W1 (padded inputs) and columns 2..7 of
// W3 and b3 (padded outputs) stay zero.  The BF16 copy holds W1, W2, W3 in
// the same layout.  A sample is 48 BF16 features (45 used).
#include "inmsom_gpu.h"
#include "closure.h"
#include "gelu.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

namespace inmsom {
int record_error(int code, const char *msg);
}

namespace {

using namespace inmsom::closure;

constexpr int KIN = 48, HID = 64, NOUT = 2, N3 = 8;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + KIN * HID, OFF_W2 = OFF_B1 + HID, OFF_B2 = OFF_W2 + HID * HID,
              OFF_W3 = OFF_B2 + HID, OFF_B3 = OFF_W3 + HID * N3, NPARAM = OFF_B3 + N3;
constexpr int BOFF_W1 = 0, BOFF_W2 = KIN * HID, BOFF_W3 = BOFF_W2 + HID * HID, NBF = BOFF_W3 + HID * N3;
static_assert(NPARAM == INMSOM_MLP_NPARAM, "parameter block size");
constexpr int TILE = 128;     // batch unit of inmsom_mlp_grad (one partial sum set per TILE samples)
constexpr int WARPS = 8;      // warps per CTA of the inference kernels (one per tile row)
constexpr int NPART = NPARAM + 1;   // per-CTA partial gradient + loss

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ uint32_t pack_raw(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    const uint32_t a = *reinterpret_cast<const uint16_t *>(&lo), b = *reinterpret_cast<const uint16_t *>(&hi);
    return a | (b << 16);
}

// C[16x8] += A[16x16] * B[16x8], BF16 inputs, FP32 accumulate
__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// grad[p] = sum over CTAs of partial[c][p] in CTA order (deterministic);
// grad[NPARAM] = mean squared error
// 32 parameters per block of 8 warps: warp w sums CTAs w, w+8, ... (each a
// coalesced 128-byte row piece), then warp 0 adds the 8 sums in order
__global__ void __launch_bounds__(256) k_mlp_reduce(const float *partial, int ntiles, int batch, float *grad)
{
    __shared__ float part[8][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, p = 32 * blockIdx.x + l;
    float a = 0.f;
    if (p <= NPARAM)
        for (int t = w; t < ntiles; t += 8) a += partial[(size_t)t * NPART + p];
    part[w][l] = a;
    __syncthreads();
    if (w == 0 && p <= NPARAM) {
        float v = 0.f;
        for (int k = 0; k < 8; k++) v += part[k][l];
        grad[p] = p == NPARAM ? v / ((float)batch * NOUT) : v;
    }
}

// Adam (Kingma & Ba), bias-corrected, then the BF16 weight copy
__global__ void k_mlp_adam(float *prm, __nv_bfloat16 *wb, float *m, float *v, const float *grad, int step,
                           float lr, float b1, float b2, float eps)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    const bool pad = (p >= OFF_W1 + 45 * HID && p < OFF_B1) || (p >= OFF_W3 && p < OFF_B3 && (p - OFF_W3) % N3 >= NOUT) ||
                     (p >= OFF_B3 + NOUT);
    float w = prm[p];
    if (!pad) {
        const float g = grad[p];
        const float mm = b1 * m[p] + (1.f - b1) * g, vv = b2 * v[p] + (1.f - b2) * g * g;
        m[p] = mm;
        v[p] = vv;
        const float mh = mm / (1.f - powf(b1, (float)step)), vh = vv / (1.f - powf(b2, (float)step));
        w -= lr * mh / (sqrtf(vh) + eps);
        prm[p] = w;
    }
    int bi = -1;
    if (p < OFF_B1) bi = BOFF_W1 + p;
    else if (p >= OFF_W2 && p < OFF_B2) bi = BOFF_W2 + (p - OFF_W2);
    else if (p >= OFF_W3 && p < OFF_B3) bi = BOFF_W3 + (p - OFF_W3);
    if (bi >= 0) wb[bi] = __float2bfloat16(w);
}

__global__ void k_mlp_pack(const float *prm, __nv_bfloat16 *wb)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < KIN * HID) wb[BOFF_W1 + p] = __float2bfloat16(prm[OFF_W1 + p]);
    else if (p < KIN * HID + HID * HID) wb[BOFF_W2 + p - KIN * HID] = __float2bfloat16(prm[OFF_W2 + p - KIN * HID]);
    else if (p < NBF) wb[BOFF_W3 + p - KIN * HID - HID * HID] = __float2bfloat16(prm[OFF_W3 + p - KIN * HID - HID * HID]);
}

// splitmix64 of (seed, step, i): uniform sample indices in [0, n)
__global__ void k_batch_indices(int *idx, int batch, long long n, unsigned long long seed, int step)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * ((unsigned long long)step * 0x100000001ull + i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    idx[i] = (int)(z % (unsigned long long)n);
}


// ============================================================ inference
// Features of cell (m, n): 5 fields x the 3 x 3 stencil around it, feature
// k = 9 f + 3 (dy + 1) + (dx + 1) for field f (u, v, ssh, H, rlh_s) at
// (m + dx, n + dy), normalised (x - mean_f) * inv_std_f and rounded to BF16;
// features 45..47 are zero.  A CTA stages a tile of TCOLS x TROWS cells plus
// a one-cell ring of the five fields in shared memory; each warp then runs
// the network on 16-cell row segments, the activations of one layer going
// to the next as MMA fragments in registers.
constexpr int TCOLS = 64, TROWS = 8, FW = TCOLS + 2, FH = TROWS + 2, NFLD = 5, NTILE = NFLD * FH * FW;
constexpr int W1S = KIN + 8, W2S = HID + 8;   // padded rows: conflict-free B fragment loads
static_assert(TROWS == WARPS, "one tile row per warp");

struct ClSmem {
    __nv_bfloat16 w1t[HID][W1S];   // W1 transposed, [n][k]
    __nv_bfloat16 w2t[HID][W2S];
    __nv_bfloat16 w3t[N3][W2S];
    float b1[HID], b2[HID], b3[N3];
    __nv_bfloat16 tile[NTILE];
    float y[WARPS][16][2];
};

__device__ __forceinline__ int feat_off(int k)   // tile offset of feature k, cell at ring (0, 0)
{
    const int f = k / 9, q = k % 9;
    return f * FH * FW + (q / 3) * FW + (q % 3);
}

__device__ void stage_tile(__nv_bfloat16 *tile, const inmsom::closure::Args &a, int m0, int n0)
{
    for (int i = threadIdx.x; i < NTILE; i += blockDim.x) {
        const int f = i / (FH * FW), rem = i - f * (FH * FW), r = rem / FW, cidx = rem - r * FW;
        const int m = m0 - 1 + cidx, n = n0 - 1 + r;
        float v = 0.f;
        if (m >= a.x1 && m <= a.x2 && n >= a.y1 && n <= a.y2)
            v = (float)a.fld[f][(long long)(n - a.y1) * a.pitch + (m - a.x1 + a.xoff)];
        tile[i] = __float2bfloat16((v - a.mean[f]) * a.inv_std[f]);
    }
}

__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }
__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// y (outputs 0, 1 of cells g and g+8 in o[0..3] of lanes t == 0) of the
// 16 cells whose layer-1 A fragments are a1.  The hidden activations are
// kept as 2 GELU (gelu2) and s.w2t, s.w3t hold the halved weights: the same
// products, one multiplication fewer per activation.
template <class S>
__device__ __forceinline__ void mlp16(const S &s, const uint32_t a1[3][4], float o[4])
{
    const int l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        acc[nt][0] = acc[nt][2] = s.b1[8 * nt + 2 * t];
        acc[nt][1] = acc[nt][3] = s.b1[8 * nt + 2 * t + 1];
    }
#pragma unroll
    for (int kb = 0; kb < 3; kb++)
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const uint32_t b[2] = {lds32(&s.w1t[8 * nt + g][16 * kb + 2 * t]), lds32(&s.w1t[8 * nt + g][16 * kb + 2 * t + 8])};
            mma16816(acc[nt], a1[kb], b);
        }
    uint32_t a2[4][4];
#pragma unroll
    for (int kb = 0; kb < 4; kb++) {
        a2[kb][0] = pack2(gelu2(acc[2 * kb][0]), gelu2(acc[2 * kb][1]));
        a2[kb][1] = pack2(gelu2(acc[2 * kb][2]), gelu2(acc[2 * kb][3]));
        a2[kb][2] = pack2(gelu2(acc[2 * kb + 1][0]), gelu2(acc[2 * kb + 1][1]));
        a2[kb][3] = pack2(gelu2(acc[2 * kb + 1][2]), gelu2(acc[2 * kb + 1][3]));
    }
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        acc[nt][0] = acc[nt][2] = s.b2[8 * nt + 2 * t];
        acc[nt][1] = acc[nt][3] = s.b2[8 * nt + 2 * t + 1];
    }
#pragma unroll
    for (int kb = 0; kb < 4; kb++)
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const uint32_t b[2] = {lds32(&s.w2t[8 * nt + g][16 * kb + 2 * t]), lds32(&s.w2t[8 * nt + g][16 * kb + 2 * t + 8])};
            mma16816(acc[nt], a2[kb], b);
        }
#pragma unroll
    for (int kb = 0; kb < 4; kb++) {
        a2[kb][0] = pack2(gelu2(acc[2 * kb][0]), gelu2(acc[2 * kb][1]));
        a2[kb][1] = pack2(gelu2(acc[2 * kb][2]), gelu2(acc[2 * kb][3]));
        a2[kb][2] = pack2(gelu2(acc[2 * kb + 1][0]), gelu2(acc[2 * kb + 1][1]));
        a2[kb][3] = pack2(gelu2(acc[2 * kb + 1][2]), gelu2(acc[2 * kb + 1][3]));
    }
    o[0] = o[2] = s.b3[2 * t];
    o[1] = o[3] = s.b3[2 * t + 1];
#pragma unroll
    for (int kb = 0; kb < 4; kb++) {
        const uint32_t b[2] = {lds32(&s.w3t[g][16 * kb + 2 * t]), lds32(&s.w3t[g][16 * kb + 2 * t + 8])};
        mma16816(o, a2[kb], b);
    }
}

// Persistent over tiles: out[c] = base[c] + MLP(features)_c * out_scale[c] * fac[c]
__global__ void __launch_bounds__(WARPS * 32, 2) k_closure_apply(const __grid_constant__ inmsom::closure::Args a)
{
    __shared__ __align__(16) ClSmem s;
    const __nv_bfloat16 *wb = (const __nv_bfloat16 *)a.wb;
    for (int i = threadIdx.x; i < KIN * HID; i += blockDim.x) s.w1t[i % HID][i / HID] = wb[BOFF_W1 + i];
    // layers 2 and 3 take 2 GELU (gelu2) as their input: their weights are
    // halved here (exact in BF16), so that every product is the network's
    for (int i = threadIdx.x; i < HID * HID; i += blockDim.x)
        s.w2t[i % HID][i / HID] = __float2bfloat16(0.5f * __bfloat162float(wb[BOFF_W2 + i]));
    for (int i = threadIdx.x; i < HID * N3; i += blockDim.x)
        s.w3t[i % N3][i / N3] = __float2bfloat16(0.5f * __bfloat162float(wb[BOFF_W3 + i]));
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
        s.b1[i] = a.prm[OFF_B1 + i];
        s.b2[i] = a.prm[OFF_B2 + i];
    }
    if (threadIdx.x < N3) s.b3[threadIdx.x] = a.prm[OFF_B3 + threadIdx.x];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    // this lane's 12 feature offsets of the layer-1 A fragments (k >= 45: zero)
    int koff[3][4];
#pragma unroll
    for (int kb = 0; kb < 3; kb++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int k = 16 * kb + 2 * t + (q & 1) + 8 * (q >> 1);
            koff[kb][q] = k < 45 ? feat_off(k) : -1;
        }
    const int nx = a.mx1 - a.mx0 + 1, ny = a.ny1 - a.ny0 + 1;
    const int ntx = (nx + TCOLS - 1) / TCOLS, nty = (ny + TROWS - 1) / TROWS;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int tix = blockIdx.x; tix < ntx * nty; tix += gridDim.x) {
        const int m0 = a.mx0 + (tix % ntx) * TCOLS, n0 = a.ny0 + (tix / ntx) * TROWS;
        __syncthreads();   // the previous tile's reads are done (and the weights are in)
        stage_tile(s.tile, a, m0, n0);
        __syncthreads();
        const int n = n0 + w;
        if (n > a.ny1) continue;
        for (int c0 = 0; c0 < TCOLS && m0 + c0 <= a.mx1; c0 += 16) {
            uint32_t a1[3][4];
            const int base_g = w * FW + c0 + g, base_h = base_g + 8;   // cells g, g+8 at ring offset
#pragma unroll
            for (int kb = 0; kb < 3; kb++)
#pragma unroll
                for (int h = 0; h < 2; h++) {   // h: features 2t.. (h = 0) or 2t+8.. (h = 1)
                    const int ka = koff[kb][2 * h], kc = koff[kb][2 * h + 1];
                    const __nv_bfloat16 xg0 = ka >= 0 ? s.tile[ka + base_g] : zero, xg1 = kc >= 0 ? s.tile[kc + base_g] : zero;
                    const __nv_bfloat16 xh0 = ka >= 0 ? s.tile[ka + base_h] : zero, xh1 = kc >= 0 ? s.tile[kc + base_h] : zero;
                    a1[kb][2 * h] = pack_raw(xg0, xg1);
                    a1[kb][2 * h + 1] = pack_raw(xh0, xh1);
                }
            float o[4];
            mlp16(s, a1, o);
            if (t == 0) {
                s.y[w][g][0] = o[0];
                s.y[w][g][1] = o[1];
                s.y[w][g + 8][0] = o[2];
                s.y[w][g + 8][1] = o[3];
            }
            __syncwarp();
            const int cell = l >> 1, comp = l & 1, m = m0 + c0 + cell;
            if (m <= a.mx1) {
                const long long idx = (long long)(n - a.y1) * a.pitch + (m - a.x1 + a.xoff);
                const double f = a.fac[comp][idx];
                if (f != 0.0) a.out[comp][idx] = a.base[comp][idx] + (double)(s.y[w][cell][comp] * a.out_scale[comp]) * f;
            }
            __syncwarp();
        }
    }
}

// the 48 BF16 features of every interior cell, row-major over (n, m)
__global__ void __launch_bounds__(WARPS * 32) k_closure_features(const __grid_constant__ inmsom::closure::Args a)
{
    __shared__ __align__(16) __nv_bfloat16 tile[NTILE];
    __shared__ int koff[KIN];
    if (threadIdx.x < KIN) koff[threadIdx.x] = threadIdx.x < 45 ? feat_off(threadIdx.x) : -1;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int nx = a.mx1 - a.mx0 + 1, ny = a.ny1 - a.ny0 + 1;
    const int ntx = (nx + TCOLS - 1) / TCOLS, nty = (ny + TROWS - 1) / TROWS;
    uint32_t *feat = (uint32_t *)a.feat;
    for (int tix = blockIdx.x; tix < ntx * nty; tix += gridDim.x) {
        const int m0 = a.mx0 + (tix % ntx) * TCOLS, n0 = a.ny0 + (tix / ntx) * TROWS;
        __syncthreads();
        stage_tile(tile, a, m0, n0);
        __syncthreads();
        const int n = n0 + w;
        if (n > a.ny1) continue;
        for (int j = l; j < TCOLS * (KIN / 2); j += 32) {
            const int cell = j / (KIN / 2), p = j - cell * (KIN / 2), m = m0 + cell;
            if (m > a.mx1) continue;
            const int b = w * FW + cell, k0 = koff[2 * p], k1 = koff[2 * p + 1];
            const __nv_bfloat16 z = __float2bfloat16(0.f);
            const uint32_t v = pack_raw(k0 >= 0 ? tile[k0 + b] : z, k1 >= 0 ? tile[k1 + b] : z);
            feat[((long long)(n - a.ny0) * nx + (m - a.mx0)) * (KIN / 2) + p] = v;
        }
    }
}

__global__ void k_closure_factors(inmsom::closure::Args a, const float *lcu, const float *lcv, const double *dxt,
                                  const double *dyh, const double *dyt, const double *dxh, double *fu, double *fv)
{
    const int nx = a.mx1 - a.mx0 + 1, ny = a.ny1 - a.ny0 + 1;
    const double *H = a.fld[3];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < (long long)nx * ny;
         k += (long long)gridDim.x * blockDim.x) {
        const int m = a.mx0 + (int)(k % nx), n = a.ny0 + (int)(k / nx);
        const long long i = (long long)(n - a.y1) * a.pitch + (m - a.x1 + a.xoff);
        fu[i] = lcu[i] > 0.5f ? 0.5 * (H[i] + H[i + 1]) * dxt[i] * dyh[i] : 0.0;
        fv[i] = lcv[i] > 0.5f ? 0.5 * (H[i] + H[i + a.pitch]) * dyt[i] * dxh[i] : 0.0;
    }
}

// ======================================================= feature rows
// The training gradient runs on the tcgen05 tensor cores (closure_tc.cu).
// Here: the network of k_closure_apply on rows of features, 64 samples per
// tile, one warp per 16.
constexpr int GT = 64, GW = 4;            // samples per tile, warps per CTA
constexpr int XS = KIN + 8, HS = HID + 8;  // padded row strides (16-byte rows, conflict-free)

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void ldsm4(uint32_t r[4], const void *p)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(p)));
}

// y[n][0..1] = MLP(x[n]) for n < count: the network of k_closure_apply
// (mlp16) on feature rows, 64 per tile, one warp per 16
struct FSmem {
    alignas(16) __nv_bfloat16 w1t[HID][XS];
    alignas(16) __nv_bfloat16 w2t[HID][HS];
    alignas(16) __nv_bfloat16 w3t[16][HS];
    float b1[HID], b2[HID], b3[N3];
    alignas(16) __nv_bfloat16 x[GT][XS];
};

__global__ void __launch_bounds__(GW * 32) k_mlp_forward(const __nv_bfloat16 *x, long long count, const float *prm,
                                                        const __nv_bfloat16 *wb, float *y)
{
    __shared__ FSmem s;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    for (int i = threadIdx.x; i < KIN * HID; i += blockDim.x) s.w1t[i % HID][i / HID] = wb[BOFF_W1 + i];
    // layers 2 and 3 take 2 GELU (mlp16's gelu2): their weights halved (exact)
    for (int i = threadIdx.x; i < HID * HID; i += blockDim.x)
        s.w2t[i % HID][i / HID] = __float2bfloat16(0.5f * __bfloat162float(wb[BOFF_W2 + i]));
    for (int i = threadIdx.x; i < 16 * HS; i += blockDim.x) {
        const int o = i / HS, c = i % HS;
        s.w3t[o][c] = o < N3 && c < HID ? __float2bfloat16(0.5f * __bfloat162float(wb[BOFF_W3 + c * N3 + o]))
                                        : __float2bfloat16(0.f);
    }
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
        s.b1[i] = prm[OFF_B1 + i];
        s.b2[i] = prm[OFF_B2 + i];
    }
    if (threadIdx.x < N3) s.b3[threadIdx.x] = prm[OFF_B3 + threadIdx.x];
    const int m0 = 16 * w;
    const long long ntiles = (count + GT - 1) / GT;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();
        for (int i = threadIdx.x; i < GT * 6; i += blockDim.x) {
            const int r = i / 6, q = i % 6;
            const long long row = tile * GT + r;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (row < count) v = reinterpret_cast<const uint4 *>(x + row * KIN)[q];
            *reinterpret_cast<uint4 *>(&s.x[r][8 * q]) = v;
        }
        __syncthreads();
        uint32_t a1[3][4];
#pragma unroll
        for (int kb = 0; kb < 3; kb++) ldsm4(a1[kb], &s.x[m0 + (l & 7) + 8 * ((l >> 3) & 1)][16 * kb + 8 * (l >> 4)]);
        float o[4];
        mlp16(s, a1, o);
        if (t == 0) {
            const long long r0 = tile * GT + m0 + g, r1 = r0 + 8;
            if (r0 < count) {
                y[r0 * NOUT] = o[0];
                y[r0 * NOUT + 1] = o[1];
            }
            if (r1 < count) {
                y[r1 * NOUT] = o[2];
                y[r1 * NOUT + 1] = o[3];
            }
        }
    }
}

int fail(int code, const char *msg) { return inmsom::record_error(code, msg); }

int check_launch(const char *what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char buf[256];
        snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
        return fail(INMSOM_ECUDA, buf);
    }
    return INMSOM_OK;
}

bool smem_ready = false;

int ensure_smem()
{
    if (smem_ready) return INMSOM_OK;
    if (inmsom::closure::grad_tc_setup()) return fail(INMSOM_ECUDA, "MLP kernels: shared memory attribute");
    smem_ready = true;
    return INMSOM_OK;
}

}  // namespace

namespace inmsom {
namespace closure {

int apply(const Args &a, int nsm, cudaStream_t s)
{
    const int nx = a.mx1 - a.mx0 + 1, ny = a.ny1 - a.ny0 + 1;
    const int tiles = ((nx + TCOLS - 1) / TCOLS) * ((ny + TROWS - 1) / TROWS);
    const int grid = tiles < 2 * nsm ? tiles : 2 * nsm;
    k_closure_apply<<<grid, WARPS * 32, 0, s>>>(a);
    return check_launch("closure apply");
}

int features(const Args &a, int nsm, cudaStream_t s)
{
    const int nx = a.mx1 - a.mx0 + 1, ny = a.ny1 - a.ny0 + 1;
    const int tiles = ((nx + TCOLS - 1) / TCOLS) * ((ny + TROWS - 1) / TROWS);
    const int grid = tiles < 4 * nsm ? tiles : 4 * nsm;
    k_closure_features<<<grid, WARPS * 32, 0, s>>>(a);
    return check_launch("closure features");
}

int factors(const Args &a, const float *lcu, const float *lcv, const double *dxt, const double *dyh,
            const double *dyt, const double *dxh, double *fac_u, double *fac_v, cudaStream_t s)
{
    k_closure_factors<<<592, 256, 0, s>>>(a, lcu, lcv, dxt, dyh, dyt, dxh, fac_u, fac_v);
    return check_launch("closure factors");
}

}  // namespace closure
}  // namespace inmsom

extern "C" {

int inmsom_mlp_pack(const float *params, void *wbf16, void *stream)
{
    if (!params || !wbf16) return fail(INMSOM_EARG, "inmsom_mlp_pack: NULL argument");
    k_mlp_pack<<<(NBF + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, (__nv_bfloat16 *)wbf16);
    return check_launch("inmsom_mlp_pack");
}

int inmsom_mlp_forward(const void *x, long long count, const float *params, const void *wbf16, float *y,
                       void *stream)
{
    if (!x || !params || !wbf16 || !y || count < 0) return fail(INMSOM_EARG, "inmsom_mlp_forward: bad argument");
    if (count == 0) return INMSOM_OK;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (count + GT - 1) / GT;
    const int grid = (int)std::min<long long>(tiles, 8LL * nsm);
    k_mlp_forward<<<grid, GW * 32, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)x, count, params,
                                                              (const __nv_bfloat16 *)wbf16, y);
    return check_launch("inmsom_mlp_forward");
}

int inmsom_mlp_grad(const void *x, const float *targets, const int *idx, int batch, const float *params,
                    const void *wbf16, float *partial, float *grad, void *stream)
{
    if (!x || !targets || !params || !wbf16 || !partial || !grad)
        return fail(INMSOM_EARG, "inmsom_mlp_grad: NULL argument");
    if (batch <= 0 || batch % TILE) return fail(INMSOM_EARG, "inmsom_mlp_grad: batch must be a positive multiple of 128");
    if (ensure_smem()) return INMSOM_ECUDA;
    // persistent CTAs on the tcgen05 tensor cores, one per SM at most and
    // at most one per 128 samples (the partial buffer's size)
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(batch / TILE, nsm);
    if (inmsom::closure::grad_tc(x, targets, idx, batch, params, wbf16, partial, grid, (cudaStream_t)stream))
        return check_launch("inmsom_mlp_grad");
    k_mlp_reduce<<<(NPARAM + 1 + 31) / 32, 256, 0, (cudaStream_t)stream>>>(partial, grid, batch, grad);
    return check_launch("inmsom_mlp_grad reduce");
}

int inmsom_mlp_adam(float *params, void *wbf16, float *m, float *v, const float *grad, int step, float lr,
                    float beta1, float beta2, float eps, void *stream)
{
    if (!params || !wbf16 || !m || !v || !grad || step < 1) return fail(INMSOM_EARG, "inmsom_mlp_adam: bad argument");
    k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, (__nv_bfloat16 *)wbf16, m, v, grad,
                                                                       step, lr, beta1, beta2, eps);
    return check_launch("inmsom_mlp_adam");
}

int inmsom_mlp_batch_indices(int *idx, int batch, long long n, unsigned long long seed, int step, void *stream)
{
    if (!idx || batch <= 0 || n <= 0) return fail(INMSOM_EARG, "inmsom_mlp_batch_indices: bad argument");
    k_batch_indices<<<(batch + 255) / 256, 256, 0, (cudaStream_t)stream>>>(idx, batch, n, seed, step);
    return check_launch("inmsom_mlp_batch_indices");
}

}  // extern "C"
