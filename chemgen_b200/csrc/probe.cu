// Measurement helpers for the roofline denominators (include/chemgen_b200_probe.h):
// the FP64 FMA rate of this GPU and the cost, in FP64 FMA issue slots, of
// the exp / log / reciprocal the kernels use (cg_math.cuh).  Each kernel runs 8
// independent dependency chains per thread on a grid of many warps, so the
// timing is throughput-bound.
#include <cuda_runtime.h>

#include "../../include/chemgen_b200_probe.h"
#include "cg_math.cuh"

namespace {

constexpr int kChains = 8;

template <int OP>
__global__ void __launch_bounds__(256) probe_kernel(double* out, int iters, double seed) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = seed + 1e-3 * (threadIdx.x + c);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            if (OP == 0) x[c] = fma(x[c], 0.999999, 1e-7);
            if (OP == 1) x[c] = cgm::cg_exp(-x[c]);
            if (OP == 2) x[c] = cgm::cg_log(x[c] + 2.0);
            if (OP == 3) x[c] = cgm::cg_rcp(x[c] + 1.0);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 12345.678) out[0] = s;    // keeps the chains live
}

template <int OP>
float time_op(int blocks, int iters, double* out) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    probe_kernel<OP><<<blocks, 256>>>(out, iters / 8, 0.5);   // warm-up
    cudaEventRecord(a);
    probe_kernel<OP><<<blocks, 256>>>(out, iters, 0.5);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

}  // namespace

extern "C" int chemgen_probe_fp64(int device, double* fma_tflops, double* exp_fma, double* log_fma,
                                  double* rcp_fma) {
    if (cudaSetDevice(device) != cudaSuccess) return 3;
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return 3;
    double* out = nullptr;
    if (cudaMalloc(&out, 64) != cudaSuccess) return 4;
    const int blocks = p.multiProcessorCount * 8;
    const int it_fma = 8192, it_tr = 512;
    const float t_fma = time_op<0>(blocks, it_fma, out);
    const float t_exp = time_op<1>(blocks, it_tr, out);
    const float t_log = time_op<2>(blocks, it_tr, out);
    const float t_rcp = time_op<3>(blocks, it_tr, out);
    const double n_thr = (double)blocks * 256 * kChains;
    const double per_fma = t_fma / (n_thr * it_fma);
    if (fma_tflops) *fma_tflops = 2.0 * n_thr * it_fma / (t_fma * 1e-3) / 1e12;
    if (exp_fma) *exp_fma = (t_exp / (n_thr * it_tr)) / per_fma;
    if (log_fma) *log_fma = (t_log / (n_thr * it_tr)) / per_fma;
    if (rcp_fma) *rcp_fma = (t_rcp / (n_thr * it_tr)) / per_fma;
    cudaError_t e = cudaGetLastError();
    cudaFree(out);
    return e == cudaSuccess ? 0 : 3;
}

namespace {
__global__ void math_check_kernel(const double* x, int n, double* e, double* l, double* er, double* lr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    e[i] = cgm::cg_exp_clamped(x[i]);
    er[i] = exp(x[i]);
    const double y = fabs(x[i]) + 1e-300;
    l[i] = cgm::cg_log(y);
    lr[i] = log(y);
}
}  // namespace

// Evaluates the kernels' exp/log and CUDA's exp/log on n device values.
extern "C" int chemgen_probe_math(const double* x, int n, double* exp_out, double* log_out, double* exp_ref,
                                  double* log_ref) {
    if (n <= 0) return 0;
    math_check_kernel<<<(n + 255) / 256, 256>>>(x, n, exp_out, log_out, exp_ref, log_ref);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 3;
}

// ---------------------------------------------------------------------------
// Self-check of the tcgen05 building blocks (umma.cuh): one CTA computes
// D[128 x N] = A[128 x K] * B[N x K]^T, BF16 in, FP32 out.
#include "umma.cuh"

namespace {
__global__ void __launch_bounds__(128) umma_probe_kernel(const __nv_bfloat16* A, const __nv_bfloat16* B, float* D,
                                                         int N, int K, uint32_t ncols, int* err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* sA = sm;
    unsigned char* sB = sm + 128 * K * 2;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + N * K * 2);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int idx = tid; idx < 128 * K; idx += 128)
        *reinterpret_cast<__nv_bfloat16*>(sA + um::kmajor_offset(idx / K, idx % K, K)) = A[idx];
    for (int idx = tid; idx < N * K; idx += 128)
        *reinterpret_cast<__nv_bfloat16*>(sB + um::kmajor_offset(idx / K, idx % K, K)) = B[idx];
    if (tid == 0) {
        um::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) um::tmem_alloc(tslot, ncols);
    um::fence_proxy_async();
    um::fence_before_sync();
    __syncthreads();
    um::fence_after_sync();
    const uint32_t taddr = *tslot;
    if (tid == 0) {
        const uint32_t idesc = um::idesc_bf16(128, N);
        const uint32_t a0 = um::smem_addr(sA), b0 = um::smem_addr(sB);
        for (int s = 0; s < K / 16; ++s)
            um::mma_bf16(taddr, um::desc_kmajor(a0, K, s), um::desc_kmajor(b0, K, s), idesc, s > 0 ? 1u : 0u);
        um::commit(mbar);
    }
    const bool ok = um::mbar_wait(mbar, 0);
    if (!ok && lane == 0) atomicExch(err, 1);
    um::fence_after_sync();
    if (ok) {
        for (int c = 0; c < N; c += 16) {
            float v[16];
            um::tmem_ld16(um::tmem_lane_addr(taddr, warp, c), v);
            for (int j = 0; j < 16; ++j) D[(32 * warp + lane) * N + c + j] = v[j];
        }
    }
    um::fence_before_sync();
    __syncthreads();
    if (warp == 0) um::tmem_dealloc(taddr, ncols);
}
}  // namespace

extern "C" int chemgen_probe_umma(const void* A, const void* B, float* D, int N, int K, int* err) {
    if (N < 16 || N > 256 || N % 16 || K < 16 || K > 256 || K % 16 || !A || !B || !D || !err) return 1;
    uint32_t ncols = 32;
    while ((int)ncols < N) ncols <<= 1;
    const size_t smem = (size_t)(128 + N) * K * 2 + 16;
    if (cudaFuncSetAttribute(umma_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 3;
    umma_probe_kernel<<<1, 128, smem>>>((const __nv_bfloat16*)A, (const __nv_bfloat16*)B, D, N, K, ncols, err);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 3;
}
