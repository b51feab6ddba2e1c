// Device-side error gate of the surrogate: which points go to the exact
// kernel, their states gathered into a compact batch, and the exact results
// scattered back, with no host round trip between the surrogate's kernel and
// the exact one.
//
// * gate_select: a point falls back when its error estimate is not <= thr
//   (a NaN estimate falls back too).  Warp-aggregated atomics append the
//   point's index to idx[0, cap); *count receives the number of points that
//   fell back, which may exceed cap (the caller then treats the rest).
//   Slots are filled in no fixed order; every point's exact result depends
//   only on its own state, so the outcome does not depend on the order.
// * gate_gather: slot j < min(*count, cap) receives point idx[j]'s P, T and
//   Y (species-major with stride cap); slots past the count keep what they
//   held, which the caller keeps a valid state.
// * gate_scatter: W[k*ng + idx[j]] = Wc[k*cap + j] for j < min(*count, cap).
// All three are grid-stride loops over a device-side count, so a launch has
// the same shape whatever the count is; gather and scatter give each thread
// one (species, slot) pair, so a few thousand points still spread over
// hundreds of thousands of independent loads.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/chemgen_b200.h"

namespace {

__global__ void gate_select_kernel(const float* __restrict__ est, float thr, int64_t ng, int64_t* __restrict__ idx,
                                   int64_t cap, unsigned long long* __restrict__ count) {
    const int lane = threadIdx.x & 31;
    const int64_t step = (int64_t)blockDim.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * 4;
    // four estimates per thread in flight at once; the trip count is the
    // same for every lane of a warp (blockDim is a multiple of 32), so the
    // ballots below always have the full warp
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x * 4; base < ng; base += stride) {
        float e[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = base + u * step + threadIdx.x;
            e[u] = i < ng ? __ldcs(est + i) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = base + u * step + threadIdx.x;
            const bool bad = i < ng && !(e[u] <= thr);
            const unsigned m = __ballot_sync(0xffffffffu, bad);
            if (m == 0u) continue;
            const int leader = __ffs(m) - 1;
            unsigned long long b0 = 0;
            if (lane == leader) b0 = atomicAdd(count, (unsigned long long)__popc(m));
            b0 = __shfl_sync(0xffffffffu, b0, leader);
            if (bad) {
                const int64_t slot = (int64_t)b0 + __popc(m & ((1u << lane) - 1u));
                if (slot < cap) idx[slot] = i;
            }
        }
    }
}

__device__ __forceinline__ int64_t active_slots(const unsigned long long* count, int64_t cap) {
    const int64_t n = (int64_t)*count;
    return n < cap ? n : cap;
}

// One thread per (row, slot) pair, slots fastest: rows 0..ns-1 are the
// species, row ns is P and row ns+1 is T; the batch side is coalesced.
__global__ void gate_gather_kernel(const double* __restrict__ P, const double* __restrict__ T,
                                   const double* __restrict__ Y, int ns, int64_t ng, const int64_t* __restrict__ idx,
                                   const unsigned long long* __restrict__ count, int64_t cap, double* __restrict__ Pc,
                                   double* __restrict__ Tc, double* __restrict__ Yc) {
    const int64_t n = active_slots(count, cap);
    const int64_t total = n * (ns + 2);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const int k = (int)(t / n);
        const int64_t j = t - (int64_t)k * n;
        const int64_t i = idx[j];
        if (k < ns) Yc[(int64_t)k * cap + j] = Y[(int64_t)k * ng + i];
        else if (k == ns) Pc[j] = P[i];
        else Tc[j] = T[i];
    }
}

// One thread per (species, slot) pair, slots fastest.
__global__ void gate_scatter_kernel(const double* __restrict__ Wc, int ns, int64_t cap,
                                    const int64_t* __restrict__ idx, const unsigned long long* __restrict__ count,
                                    double* __restrict__ W, int64_t ng) {
    const int64_t n = active_slots(count, cap);
    const int64_t total = n * ns;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const int k = (int)(t / n);
        const int64_t j = t - (int64_t)k * n;
        W[(int64_t)k * ng + idx[j]] = Wc[(int64_t)k * cap + j];
    }
}

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return n;
}

// enough blocks to cover `work` threads' worth of slots, at most a few per SM
unsigned grid_for(int64_t work, int per_sm) {
    const int sms = sm_count();
    const int64_t want = (work + 255) / 256;
    const int64_t most = (int64_t)(sms > 0 ? sms : 1) * per_sm;
    return (unsigned)(want < 1 ? 1 : want < most ? want : most);
}

bool aligned8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7) == 0; }

}  // namespace

extern "C" {

int chemgen_gate_select(const float* est, float thr, int64_t ng, int64_t* idx, int64_t cap, uint64_t* count,
                        void* stream) {
    if (!est || !idx || !count || ng < 0 || cap < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (!aligned8(idx) || !aligned8(count)) return CHEMGEN_ERR_MISALIGNED;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(count, 0, sizeof(uint64_t), s) != cudaSuccess) return CHEMGEN_ERR_CUDA;
    if (ng == 0) return CHEMGEN_OK;
    gate_select_kernel<<<grid_for((ng + 3) / 4, 8), 256, 0, s>>>(est, thr, ng, idx, cap,
                                                        reinterpret_cast<unsigned long long*>(count));
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

int chemgen_gate_gather(const double* P, const double* T, const double* Y, int ns, int64_t ng, const int64_t* idx,
                        const uint64_t* count, int64_t cap, double* Pc, double* Tc, double* Yc, void* stream) {
    if (!P || !T || !Y || !idx || !count || !Pc || !Tc || !Yc || ns < 1 || ng < 0 || cap < 0)
        return CHEMGEN_ERR_INVALID_ARGUMENT;
    for (const void* p : {(const void*)P, (const void*)T, (const void*)Y, (const void*)idx, (const void*)count,
                          (const void*)Pc, (const void*)Tc, (const void*)Yc})
        if (!aligned8(p)) return CHEMGEN_ERR_MISALIGNED;
    if (ng == 0 || cap == 0) return CHEMGEN_OK;
    gate_gather_kernel<<<grid_for(cap * (ns + 2), 4), 256, 0, (cudaStream_t)stream>>>(
        P, T, Y, ns, ng, idx, reinterpret_cast<const unsigned long long*>(count), cap, Pc, Tc, Yc);
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

int chemgen_gate_scatter(const double* Wc, int ns, int64_t cap, const int64_t* idx, const uint64_t* count,
                         double* W, int64_t ng, void* stream) {
    if (!Wc || !idx || !count || !W || ns < 1 || ng < 0 || cap < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    for (const void* p : {(const void*)Wc, (const void*)idx, (const void*)count, (const void*)W})
        if (!aligned8(p)) return CHEMGEN_ERR_MISALIGNED;
    if (ng == 0 || cap == 0) return CHEMGEN_OK;
    gate_scatter_kernel<<<grid_for(cap * ns, 4), 256, 0, (cudaStream_t)stream>>>(
        Wc, ns, cap, idx, reinterpret_cast<const unsigned long long*>(count), W, ng);
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

}  // extern "C"
