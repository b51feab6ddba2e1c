// Helpers shared by the mechanism-specialised kernels that
// chemgen_b200/emit_cuda.py writes (generate_chemistry.py --language cuda).
//
// A generated kernel handles one grid point per thread.  Species indices,
// stoichiometry and coefficients are compile-time constants; the wdot
// accumulators are registers; C lives in shared memory as [species][thread],
// and EGp = exp(smh) * Patm/(R0 T) (FP64) or the log2 Gibbs terms (mixed)
// either beside it or, when that lets the block grow, in tensor memory.
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

// ------------------------------------------------------- tensor memory
// When shared memory cannot hold both per-point arrays for the block size
// the kernel wants, the FP64 kernel keeps EGp in tensor memory instead (the
// mixed kernel can do the same with its log2 Gibbs terms): each thread owns
// one lane (warp w reaches lanes 32 (w % 4) .. 32 (w % 4) + 31)
// and, for warp slot w / 4, 2 ns consecutive 32-bit columns, species k at
// columns 2k, 2k+1 (low, high word).  The tcgen05 ld/st are warp-collective;
// the generated kernels call them from straight-line code that every thread
// of the warp executes, and each helper first reconverges the warp
// (__syncwarp) in case a rare special-argument path of cg_log diverged it.

// Allocates `ncols` columns for the block (warp 0), publishes the base
// through shared memory and orders it for all threads.
__device__ __forceinline__ uint32_t tm_alloc(uint32_t* slot, uint32_t ncols) {
    if ((threadIdx.x >> 5) == 0) {
        const uint32_t s = (uint32_t)__cvta_generic_to_shared(slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s), "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return *slot;
}

__device__ __forceinline__ void tm_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
    }
}

// This thread's first column: lane quadrant of the warp, column slot w / 4.
__device__ __forceinline__ uint32_t tm_thread_base(uint32_t base, int cols_per_slot) {
    const int w = threadIdx.x >> 5;
    return base + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)((w >> 2) * cols_per_slot);
}

__device__ __forceinline__ void tm_st(uint32_t a, double v) {
    __syncwarp();
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(a), "r"(__double2loint(v)),
                 "r"(__double2hiint(v)));
}

__device__ __forceinline__ void tm_wait_st() {
    __syncwarp();
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// Loads of 1..4 doubles, each batch completed by one wait inside the same
// asm so that no register is read before its load has landed.
__device__ __forceinline__ void tm_ld(uint32_t a0, double& v0) {
    uint32_t l0, h0;
    __syncwarp();
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n\t"
                 "tcgen05.wait::ld.sync.aligned;"
                 : "=r"(l0), "=r"(h0) : "r"(a0));
    v0 = __hiloint2double((int)h0, (int)l0);
}
__device__ __forceinline__ void tm_ld(uint32_t a0, uint32_t a1, double& v0, double& v1) {
    uint32_t l0, h0, l1, h1;
    __syncwarp();
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%4];\n\t"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%2, %3}, [%5];\n\t"
                 "tcgen05.wait::ld.sync.aligned;"
                 : "=r"(l0), "=r"(h0), "=r"(l1), "=r"(h1) : "r"(a0), "r"(a1));
    v0 = __hiloint2double((int)h0, (int)l0);
    v1 = __hiloint2double((int)h1, (int)l1);
}
__device__ __forceinline__ void tm_ld(uint32_t a0, uint32_t a1, uint32_t a2, double& v0, double& v1, double& v2) {
    uint32_t l0, h0, l1, h1, l2, h2;
    __syncwarp();
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%6];\n\t"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%2, %3}, [%7];\n\t"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%4, %5}, [%8];\n\t"
                 "tcgen05.wait::ld.sync.aligned;"
                 : "=r"(l0), "=r"(h0), "=r"(l1), "=r"(h1), "=r"(l2), "=r"(h2) : "r"(a0), "r"(a1), "r"(a2));
    v0 = __hiloint2double((int)h0, (int)l0);
    v1 = __hiloint2double((int)h1, (int)l1);
    v2 = __hiloint2double((int)h2, (int)l2);
}
__device__ __forceinline__ void tm_ld(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, double& v0, double& v1,
                                      double& v2, double& v3) {
    uint32_t l0, h0, l1, h1, l2, h2, l3, h3;
    __syncwarp();
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%8];\n\t"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%2, %3}, [%9];\n\t"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%4, %5}, [%10];\n\t"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%6, %7}, [%11];\n\t"
                 "tcgen05.wait::ld.sync.aligned;"
                 : "=r"(l0), "=r"(h0), "=r"(l1), "=r"(h1), "=r"(l2), "=r"(h2), "=r"(l3), "=r"(h3)
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3));
    v0 = __hiloint2double((int)h0, (int)l0);
    v1 = __hiloint2double((int)h1, (int)l1);
    v2 = __hiloint2double((int)h2, (int)l2);
    v3 = __hiloint2double((int)h3, (int)l3);
}

// Split form, so that the loads of the next reaction's values fly while this
// reaction computes: tm_issue starts the load of one double into two 32-bit
// registers without waiting; tm_wait_k completes every load issued so far
// and takes the k pending pairs as in/out operands, so that no use of them
// can be scheduled above it.
__device__ __forceinline__ void tm_issue(uint32_t a, uint32_t& lo, uint32_t& hi) {
    __syncwarp();
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(lo), "=r"(hi) : "r"(a));
}
__device__ __forceinline__ void tm_wait_1(uint32_t* r) {
    __syncwarp();
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1])::"memory");
}
__device__ __forceinline__ void tm_wait_2(uint32_t* r) {
    __syncwarp();
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])::"memory");
}
__device__ __forceinline__ void tm_wait_3(uint32_t* r) {
    __syncwarp();
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5])::"memory");
}
__device__ __forceinline__ void tm_wait_4(uint32_t* r) {
    __syncwarp();
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                   "+r"(r[7])::"memory");
}
__device__ __forceinline__ void tm_wait_5(uint32_t* r) {
    __syncwarp();
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                   "+r"(r[7]), "+r"(r[8]), "+r"(r[9])::"memory");
}
__device__ __forceinline__ void tm_wait_6(uint32_t* r) {
    __syncwarp();
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                   "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11])::"memory");
}

}  // namespace cgg

