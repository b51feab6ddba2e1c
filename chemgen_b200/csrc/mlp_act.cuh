// The surrogate network's activation: GELU in tanh form,
// 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), with tanh from the
// hardware approximation (tanh.approx.f32, relative error about 2^-11).  The
// same function is evaluated in every training kernel and in the fused
// inference kernel, so the trained weights are exact for it.
#pragma once

namespace {

__device__ __forceinline__ float tanh_hw(float u) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return t;
}

// GELU(z); with dgelu != nullptr also its derivative.
__device__ __forceinline__ float gelu(float z, float* dgelu) {
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    const float u = k0 * fmaf(k1 * z * z, z, z);
    const float t = tanh_hw(u);
    if (dgelu) *dgelu = 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * k0 * fmaf(3.0f * k1, z * z, 1.0f);
    const float hz = 0.5f * z;
    return fmaf(hz, t, hz);
}

}  // namespace
