// Learned closure on the resident state of a context: the feature stencil,
// the fused inference + forcing update, and the per-point factors that turn
// a velocity tendency into the step's RHS units.
#pragma once

#include <cuda_runtime.h>

namespace inmsom {
namespace closure {

// Device fields are pitched like the state: element (m, n) at
// (n - y1) * pitch + (m - x1 + xoff).
struct Args {
    const double *fld[5];          // u, v, ssh (current level), rest depth H, Coriolis rlh_s
    const double *fac[2];          // hu * dxt * dyh at ocean u points, hv * dyt * dxh at ocean v points, else 0
    const double *base[2];         // RHSx, RHSy without the closure
    double *out[2];                // RHSx, RHSy the substeps read
    void *feat;                    // features: BF16 [ny][nx][48], row n-ny0, column m-mx0
    const float *prm;              // FP32 parameter block (biases)
    const void *wb;                // BF16 weights
    long long pitch;
    int x1, x2, y1, y2, xoff;      // array bounds (bnd_*) and padding columns
    int mx0, mx1, ny0, ny1;        // interior
    float mean[5], inv_std[5];     // feature normalisation per field
    float out_scale[2];            // tendency (m/s^2) per unit network output
};

// out[c] = base[c] + y_c * out_scale[c] * fac[c] at the points where fac != 0
int apply(const Args &a, int nsm, cudaStream_t s);
// feat = the 48 features of every interior cell
int features(const Args &a, int nsm, cudaStream_t s);
// fac[0], fac[1] from the rest depth, the u/v masks and the metrics
int factors(const Args &a, const float *lcu, const float *lcv, const double *dxt, const double *dyh,
            const double *dyt, const double *dxh, double *fac_u, double *fac_v, cudaStream_t s);

// The training gradient on the tcgen05 tensor cores (closure_tc.cu):
// per-CTA partial sums (INMSOM_MLP_PARTIAL floats each) of grid persistent
// CTAs, one per SM at most, over the batch's tiles of 128 samples;
// grad_tc_setup sets the kernel's shared-memory size once.
size_t grad_tc_smem();
int grad_tc_setup();
int grad_tc(const void *x, const float *targets, const int *idx, int batch, const float *params, const void *wbf16,
            float *partial, int grid, cudaStream_t s);

}  // namespace closure
}  // namespace inmsom
