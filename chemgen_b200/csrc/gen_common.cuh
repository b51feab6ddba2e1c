// Helpers shared by the mechanism-specialised kernels that
// chemgen_b200/emit_cuda.py writes (generate_chemistry.py --language cuda).
//
// A generated kernel handles one grid point per thread.  Species indices,
// stoichiometry and coefficients are compile-time constants; the wdot
// accumulators are registers; C and EGp = exp(smh) * Patm/(R0 T) (FP64) or the
// log2 Gibbs terms (mixed) live in shared memory as [species][thread].
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/chemgen_b200.h"
#include "cg_math.cuh"

namespace cgg {

constexpr double kR0 = 8.314510e+07;
constexpr double kPatm = 1013250.0;
constexpr double kLog2e = 1.4426950408889634074;
constexpr double kLn10 = 2.302585092994045684;

// Newton-refined reciprocal (two iterations from the hardware estimate).
__device__ __forceinline__ double rcp(double x) { return cgm::cg_rcp(x); }

// ---------------------------------------------------------------- mixed
// 2^a for an FP64 exponent a, returned as FP64 with about 2^-22 relative
// error: a = n + f with n = nearest integer (round-to-nearest by adding
// 1.5*2^52), 2^f from the SFU's ex2 on FP32, and 2^n folded into the FP64
// exponent field with integer arithmetic.  `scale` multiplies 2^f (an FP32
// product, e.g. of concentrations) and `eoff` is an extra integer exponent.
// Results below 2^-1022 flush to zero; above 2^1023 they become +inf.
__device__ __forceinline__ float ex2f(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2f(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Split a (|a| < 2^30) into integer n and fraction f in [-0.5, 0.5].
__device__ __forceinline__ void split2(double a, int& n, float& f) {
    const double magic = 6755399441055744.0;   // 1.5 * 2^52
    const double t = a + magic;
    n = __double2loint(t);
    f = (float)(a - (t - magic));
}

// 2^k as FP64 for an integer k, built in the exponent field; k is clamped
// to [-1023, 1023] (2^-1023 encodes as +0).
__device__ __forceinline__ double exp2i(int k) {
    const int e = max(0, min(k + 1023, 2046));
    return __hiloint2double(e << 20, 0);
}

// 2^k as FP32 for -126 <= k <= 127, built in the exponent field (unsigned
// shift: no signed-overflow arithmetic for any k).
__device__ __forceinline__ float exp2f_int(int k) { return __uint_as_float((unsigned int)(k + 127) << 23); }

// lg2 of Pr/(1+Pr) for Pr = mpr 2^npr (mpr in [0.5, 1), l2m = lg2 mpr):
// Pr < 1: npr + l2m - lg2(1 + Pr), reported as l2r = l2m - lg2(1 + Pr) with
// nfix = npr; Pr >= 1: l2r = -lg2(1 + 1/Pr), nfix = 0.  Terms below 2^-126
// are dropped.  (A branch-free select of the two forms gave wrong results
// inside the large generated kernels although it matched this form in a
// stand-alone test; the branch is kept.)
__device__ __forceinline__ void falloff_blend(float mpr, int npr, float l2m, float& l2r, int& nfix) {
    if (npr < 0) {
        const float pr = npr > -126 ? mpr * exp2f_int(npr) : 0.0f;
        l2r = l2m - lg2f(1.0f + pr);
        nfix = npr;
    } else {
        const float ipr = npr < 126 ? __fdividef(1.0f, mpr) * exp2f_int(-npr) : 0.0f;
        l2r = -lg2f(1.0f + ipr);
        nfix = 0;
    }
}

// q = 2^a * prod  (prod an FP32 product of scaled concentrations, eoff the
// integer exponent that undoes their scaling): the FP32 value 2^f * prod,
// converted exactly to FP64, times 2^(n + eoff) -- exact for results in the
// FP64 normal range.
__device__ __forceinline__ double rate2(double a, float prod, int eoff) {
    int n;
    float f;
    split2(a, n, f);
    return (double)(ex2f(f) * prod) * exp2i(n + eoff);
}

}  // namespace cgg

