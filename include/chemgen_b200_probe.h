/*
 * Measurement helpers of libchemgen_b200.so (no counterpart in the
 * reference, whose timing is a Fortran cpu_time around one call,
 * chemgen/templates/chemistry_mini_app.j2:73-99).
 *
 * chemgen_probe_fp64: FP64 FMA throughput of `device` (TFLOP/s, 2 flops per
 * FMA) and the throughput cost of one exp, log and Newton-refined reciprocal
 * as used by the kernels, in FP64-FMA equivalents.  Returns 0 on success.
 */
#ifndef CHEMGEN_B200_PROBE_H
#define CHEMGEN_B200_PROBE_H
#ifdef __cplusplus
extern "C" {
#endif
int chemgen_probe_fp64(int device, double* fma_tflops, double* exp_fma, double* log_fma, double* rcp_fma);
/* The kernels' exp (clamped) and log next to CUDA's exp and log(|x|+1e-300)
 * on n device values; synchronous. */
int chemgen_probe_math(const double* x, int n, double* exp_out, double* log_out, double* exp_ref, double* log_ref);
/* Self-check of the library's tensor-core building blocks: one CTA computes
 * D[128 x N] = A[128 x K] B[N x K]^T (BF16 row-major inputs on the device,
 * FP32 output), N and K multiples of 16 up to 256; *err is set to 1 if the
 * completion wait timed out.  Synchronous. */
int chemgen_probe_umma(const void* A, const void* B, float* D, int N, int K, int* err);
#ifdef __cplusplus
}
#endif
#endif
