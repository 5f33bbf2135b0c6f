// GELU of the closure network in the tanh form of Hendrycks & Gimpel
// (2016), x * g(x) with the gate g(x) = 0.5 (1 + tanh(sqrt(2/pi)(x +
// 0.044715 x^3))), evaluated two ways that the network uses side by side:
//   * gelu_t: the gate through the hardware tanh (tanh.approx.f32, relative
//     error about 2^-11) on the special-function unit;
//   * gelu_p: the gate as an odd polynomial of degree 15, 0.5 + x P(x^2),
//     fitted by least squares at 4000 Chebyshev nodes of [-4, 4] to the
//     exact gate and clamped to [0, 1] (|x| > 4 gives 0 or 1, the exact
//     gate being within 2e-5 of them there); FP32 Horner on the FMA pipe,
//     largest error of the gate 4e-5.
// Both are far inside the BF16 rounding (2^-9) of the activations.  Of the
// 64 outputs of a layer, those in the even 8-column blocks use gelu_t and
// those in the odd ones gelu_p -- in training and inference alike -- so
// that the activations load the special-function unit and the FMA pipe in
// about equal parts.  gelu_dt / gelu_dp are the matching derivatives,
// g + x g' with g' = 0.5 (1 - t^2) (sqrt(2/pi) + 3 * 0.044715 sqrt(2/pi) x^2)
// = 2 g (1 - g) (...), t the tanh.
#pragma once

namespace inmsom {
namespace closure {

constexpr float GELU_C0 = 0.7978845608028654f, GELU_C1 = 0.7978845608028654f * 0.044715f;

__device__ __forceinline__ float tanh_hw(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float gate_t(float x) { return fmaf(0.5f, tanh_hw(x * fmaf(GELU_C1, x * x, GELU_C0)), 0.5f); }

__device__ __forceinline__ float gate_p(float x)
{
    // P(x^2), Horner from the highest power
    const float xc = fminf(fmaxf(x, -4.0f), 4.0f), x2 = xc * xc;
    float p = fmaf(-1.722785e-09f, x2, 1.3184966e-07f);
    p = fmaf(p, x2, -4.3967939e-06f);
    p = fmaf(p, x2, 8.5165426e-05f);
    p = fmaf(p, x2, -0.0010853761f);
    p = fmaf(p, x2, 0.0098192329f);
    p = fmaf(p, x2, -0.066405386f);
    p = fmaf(p, x2, 0.39881077f);
    return fminf(fmaxf(fmaf(xc, p, 0.5f), 0.0f), 1.0f);
}

__device__ __forceinline__ float gelu_t(float x) { return x * gate_t(x); }
__device__ __forceinline__ float gelu_p(float x) { return x * gate_p(x); }

__device__ __forceinline__ float gelu_dt(float x)
{
    const float x2 = x * x, t = tanh_hw(x * fmaf(GELU_C1, x2, GELU_C0));
    return fmaf(0.5f, 1.0f + t, 0.5f * x * (1.0f - t * t) * fmaf(3.0f * GELU_C1, x2, GELU_C0));
}
// beyond |x| = 4 the clamped gate is constant: its derivative term is taken
// at the clamp (largest error of the derivative 8e-4)
__device__ __forceinline__ float gelu_dp(float x)
{
    const float g = gate_p(x), xc = fminf(fmaxf(x, -4.0f), 4.0f);
    return fmaf(xc * (2.0f * g * (1.0f - g)), fmaf(3.0f * GELU_C1, xc * xc, GELU_C0), g);
}

}  // namespace closure
}  // namespace inmsom
