// GELU of the closure network in the tanh form of Hendrycks & Gimpel
// (2016), x * g(x) with the gate g(x) = 0.5 (1 + tanh(sqrt(2/pi)(x +
// 0.044715 x^3))), the gate through the hardware tanh (tanh.approx.f32,
// relative error about 2^-11: below the BF16 rounding, 2^-9, of the
// activations).  Training (closure_tc.cu) and inference (closure.cu) use
// this one definition, so the network the kernels train is the one they
// run.  gelu_d is its derivative, g + x g' with
// g' = 0.5 (1 - t^2) (sqrt(2/pi) + 3 * 0.044715 sqrt(2/pi) x^2), t the tanh.
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

__device__ __forceinline__ float gelu(float x)
{
    const float h = 0.5f * x;
    return fmaf(h, tanh_hw(x * fmaf(GELU_C1, x * x, GELU_C0)), h);
}

// 2 GELU(x) = x (1 + t), one multiplication fewer than GELU itself and
// bit for bit twice its value (a power-of-two scale commutes with the
// rounding): the inference kernel feeds it to the next layer with that
// layer's weights halved, which leaves every product a * w unchanged
__device__ __forceinline__ float gelu2(float x)
{
    return fmaf(x, tanh_hw(x * fmaf(GELU_C1, x * x, GELU_C0)), x);
}

__device__ __forceinline__ float gelu_d(float x)
{
    const float x2 = x * x, t = tanh_hw(x * fmaf(GELU_C1, x2, GELU_C0));
    return fmaf(0.5f, 1.0f + t, 0.5f * x * (1.0f - t * t) * fmaf(3.0f * GELU_C1, x2, GELU_C0));
}

}  // namespace closure
}  // namespace inmsom
