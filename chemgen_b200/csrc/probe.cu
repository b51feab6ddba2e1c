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
