// Kernels of the learned wdot surrogate: a 4-layer MLP (inputs 1/T, ln T,
// ln P and the ns ln X_k -> 3 x 256 GELU -> the direction and log length of
// the wdot vector plus one error-estimate output), BF16 weights with FP32
// accumulation.
//
// The reference has no surrogate (its chemistry_nn.py:15-85 prototype never
// ran).  Everything here is this package's own:
// * mlp_gemm: C[i][j] (+)= sum_r A(i,r) B(j,r) on the tensor cores
//   (mma.sync m16n8k16, BF16 in, FP32 accumulate) with arbitrary element
//   strides, so one kernel serves the forward product (X W^T), the input
//   gradient (dZ W) and the weight gradient (dZ^T H); long reductions over
//   few output tiles (weight gradients) are split over r;
// * elementwise kernels: bias + GELU (tanh form, hardware tanh) forward, GELU backward, loss
//   gradient, column sums for bias gradients, Adam with FP32 master weights;
// * the feature / target transforms between (P, T, Y, wdot) and network
//   space, and the decode of predictions back to wdot.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/chemgen_b200.h"
#include "mlp_act.cuh"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kBM = 64, kBN = 64, kBR = 32, kPad = 8;

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// Stage rows [x0, x0 + 64) x columns [r0, r0 + kBR) of the operand
// X(x, r) = X[x * sx + r * sr] into S (zero outside [0, nx) x [0, R)).  The
// thread-to-element order follows whichever stride is 1 so that a warp's
// loads are contiguous, with 16-byte vectors when the r direction is
// contiguous and aligned.
__device__ __forceinline__ void load_tile(const bf16* __restrict__ X, int64_t sx, int64_t sr, int x0, int r0, int nx,
                                          int R, bf16 (*S)[kBR + kPad], int tid) {
    const bf16 zero = __float2bfloat16(0.0f);
    if (sr == 1 && (sx & 7) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0) {
        for (int e = tid; e < kBM * (kBR / 8); e += 128) {
            const int xx = e / (kBR / 8), rr = (e % (kBR / 8)) * 8;
            const int gx = x0 + xx, gr = r0 + rr;
            if (gx < nx && gr + 8 <= R) {
                *reinterpret_cast<uint4*>(&S[xx][rr]) = *reinterpret_cast<const uint4*>(X + gx * sx + gr);
            } else {
#pragma unroll
                for (int u = 0; u < 8; ++u) S[xx][rr + u] = (gx < nx && gr + u < R) ? X[gx * sx + gr + u] : zero;
            }
        }
    } else if (sr == 1) {
        for (int e = tid; e < kBM * kBR; e += 128) {
            const int xx = e / kBR, rr = e % kBR;
            const int gx = x0 + xx, gr = r0 + rr;
            S[xx][rr] = (gx < nx && gr < R) ? X[gx * sx + gr] : zero;
        }
    } else {
        for (int e = tid; e < kBM * kBR; e += 128) {
            const int xx = e % kBM, rr = e / kBM;
            const int gx = x0 + xx, gr = r0 + rr;
            S[xx][rr] = (gx < nx && gr < R) ? X[gx * sx + gr * sr] : zero;
        }
    }
}

// C = A B^T over r in [blockIdx.z * rchunk, (blockIdx.z + 1) * rchunk); with
// more than one r slice (gridDim.z > 1) the slices add into C atomically.
__global__ void __launch_bounds__(128) mlp_gemm_kernel(const bf16* __restrict__ A, int64_t sai, int64_t sar,
                                                       const bf16* __restrict__ B, int64_t sbj, int64_t sbr,
                                                       float* __restrict__ C, int64_t ldc, int M, int N, int R,
                                                       int rchunk, int accumulate) {
    __shared__ __align__(16) bf16 As[kBM][kBR + kPad];
    __shared__ __align__(16) bf16 Bs[kBN][kBR + kPad];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int i0 = blockIdx.y * kBM, j0 = blockIdx.x * kBN;
    const int wi = (warp >> 1) * 32, wj = (warp & 1) * 32;
    const int rbeg = blockIdx.z * rchunk, rend = min(R, rbeg + rchunk);
    float acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
    const int q = lane >> 2, c2 = (lane & 3) * 2;
    for (int r0 = rbeg; r0 < rend; r0 += kBR) {
        load_tile(A, sai, sar, i0, r0, M, rend, As, tid);
        load_tile(B, sbj, sbr, j0, r0, N, rend, Bs, tid);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kBR; k += 16) {
            uint32_t af[2][4], bfr[4][2];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const int row = wi + a * 16 + q;
                af[a][0] = pack2(As[row][k + c2], As[row][k + c2 + 1]);
                af[a][1] = pack2(As[row + 8][k + c2], As[row + 8][k + c2 + 1]);
                af[a][2] = pack2(As[row][k + c2 + 8], As[row][k + c2 + 9]);
                af[a][3] = pack2(As[row + 8][k + c2 + 8], As[row + 8][k + c2 + 9]);
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int col = wj + b * 8 + q;
                bfr[b][0] = pack2(Bs[col][k + c2], Bs[col][k + c2 + 1]);
                bfr[b][1] = pack2(Bs[col][k + c2 + 8], Bs[col][k + c2 + 9]);
            }
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
                        : "+f"(acc[a][b][0]), "+f"(acc[a][b][1]), "+f"(acc[a][b][2]), "+f"(acc[a][b][3])
                        : "r"(af[a][0]), "r"(af[a][1]), "r"(af[a][2]), "r"(af[a][3]), "r"(bfr[b][0]),
                          "r"(bfr[b][1]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int gi = i0 + wi + a * 16 + q + h * 8, gj = j0 + wj + b * 8 + c2 + e;
                    if (gi < M && gj < N) {
                        float* c = C + gi * ldc + gj;
                        if (gridDim.z > 1) atomicAdd(c, acc[a][b][h * 2 + e]);
                        else *c = accumulate ? *c + acc[a][b][h * 2 + e] : acc[a][b][h * 2 + e];
                    }
                }
}

// Z[m][n] += bias[n]; H = GELU(Z) as BF16 (and FP32 Z kept for the backward)
__global__ void bias_gelu_kernel(float* Z, const float* bias, bf16* H, int64_t M, int N, int apply_gelu) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= M * N) return;
    const float z = Z[idx] + bias[idx % N];
    Z[idx] = z;
    if (H) H[idx] = __float2bfloat16(apply_gelu ? gelu(z, nullptr) : z);
}

// dZ = dH * GELU'(Z), as BF16 for the next products
__global__ void gelu_backward_kernel(const float* dH, const float* Z, bf16* dZ, float* dZf, int64_t n) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    float d;
    gelu(Z[idx], &d);
    const float g = dH[idx] * d;
    dZ[idx] = __float2bfloat16(g);
    if (dZf) dZf[idx] = g;
}

// Loss L = mean over rows of sum_j w_j (out_j - target_j)^2; dOut = dL/dout (BF16 and FP32)
__global__ void mse_grad_kernel(const float* out, const float* target, const float* colw, bf16* dout, float* doutf,
                                float* loss, int64_t M, int N) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (idx < M * N) {
        const int j = (int)(idx % N);
        const float d = out[idx] - target[idx];
        const float g = 2.0f * colw[j] * d / (float)M;
        dout[idx] = __float2bfloat16(g);
        if (doutf) doutf[idx] = g;
        l = colw[j] * d * d / (float)M;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

// db[n] = sum_m dZ[m][n]
__global__ void colsum_kernel(const float* dZ, float* db, int64_t M, int N) {
    const int n = blockIdx.x;
    float s = 0.0f;
    for (int64_t m = threadIdx.x; m < M; m += blockDim.x) s += dZ[m * N + n];
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[n] = red[0];
}

// Adam on FP32 master weights; writes the BF16 copy the products use.  The
// step's learning rate and bias corrections come from device memory
// (hyper = {lr, 1/(1-b1^t), 1/(1-b2^t)}) so that a captured training step
// can be replayed along a schedule.
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, bf16* wb, int64_t n, const float* hyper,
                            float b1, float b2, float eps, float wd) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float lr = hyper[0], c1 = hyper[1], c2 = hyper[2];
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
}

// Network inputs per point: 1000/T, ln T, ln(P / 1 atm) and, for the ns
// species, ln X_k (mole fraction, from Y and the inverse molecular weights
// inv_mw; ln Y_k when inv_mw is null), each as (v - c) * s with the
// centring/scaling pairs in norm[0..7], the species ones clipped to [-6, 6];
// then zeros up to din.  In these variables the logarithm of a rate constant
// is linear (Arrhenius) and that of a concentration product is a sum.
//
// Each value f is stored as two BF16 numbers, hi = bf16(f) in X[i][0..din)
// and lo = bf16(f - hi) in X[i][din..2 din), so that the first layer, which
// multiplies both halves by the same weights, sees the input to ~16 bits
// (one BF16 alone would perturb 1000/T by up to 2^-9 relative, which moves
// a rate constant with E/R = 25000 K by ~10%).  Xf (optional) gets f in FP32.
__device__ __forceinline__ float feature_value(const double* P, const double* T, const double* Y, int64_t ng, int ns,
                                               const float* norm, const double* inv_mw, double lmix, int64_t i,
                                               int j) {
    if (j == 0) return (float)((1000.0 / T[i] - (double)norm[0]) * (double)norm[1]);
    if (j == 1) return (float)((log(T[i]) - (double)norm[2]) * (double)norm[3]);
    if (j == 2) return (float)((log(P[i] / 1013250.0) - (double)norm[4]) * (double)norm[5]);
    const int k = j - 3;
    if (k >= ns) return 0.0f;
    const double y = fmax(Y[(int64_t)k * ng + i], 1e-30);
    const double lx = inv_mw ? log(y * inv_mw[k]) - lmix : log(y);
    return (float)fmin(fmax((lx - (double)norm[6]) * (double)norm[7], -6.0), 6.0);
}

__device__ __forceinline__ double mixture_log(const double* Y, int64_t ng, int ns, const double* inv_mw, int64_t i) {
    if (!inv_mw) return 0.0;
    double s = 0.0;
    for (int k = 0; k < ns; ++k) s += fmax(Y[(int64_t)k * ng + i], 0.0) * inv_mw[k];
    return log(fmax(s, 1e-300));
}

__global__ void features_kernel(const double* P, const double* T, const double* Y, int64_t ng, int ns, int din,
                                const float* norm, const double* inv_mw, bf16* X, float* Xf) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ng) return;
    const double lmix = mixture_log(Y, ng, ns, inv_mw, i);
    bf16* x = X + i * (2 * (int64_t)din);
    for (int j = 0; j < din; ++j) {
        const float f = feature_value(P, T, Y, ng, ns, norm, inv_mw, lmix, i, j);
        const bf16 hi = __float2bfloat16(f);
        x[j] = hi;
        x[din + j] = __float2bfloat16(f - __bfloat162float(hi));
        if (Xf) Xf[i * din + j] = f;
    }
}

// Targets per point, width dout: the direction u_k = w_k / |w|_2 of the rate
// vector (columns 0..ns-1) and its log length (ln |w|_2 - c) / s in column
// ns, with (c, s) = lnorm[0..1]; other columns 0.  The normwise error of a
// decoded prediction is then max_k |du_k| / max_k |u_k| + |d ln |w|_2| to
// first order, so the regression loss measures what the error gate tests.
__global__ void targets_kernel(const double* W, int64_t ng, int ns, int dout, const float* lnorm, float* Tg) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ng) return;
    double n2 = 0.0;
    for (int k = 0; k < ns; ++k) {
        const double w = W[(int64_t)k * ng + i];
        n2 += w * w;
    }
    const double n = fmax(sqrt(n2), 1e-300);
    for (int k = 0; k < dout; ++k) {
        float y = 0.0f;
        if (k < ns) y = (float)(W[(int64_t)k * ng + i] / n);
        else if (k == ns) y = (float)((log(n) - (double)lnorm[0]) / (double)lnorm[1]);
        Tg[i * dout + k] = y;
    }
}

// Predictions -> wdot (species-major, FP64): w_k = u_k exp(c + s L); column
// ns + 1 is the network's estimate of log10 of its own normwise error.
__global__ void decode_kernel(const float* out, int64_t ng, int ns, int dout, const float* lnorm, double* W,
                              float* err_est) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ng) return;
    const double n = exp((double)lnorm[0] + (double)lnorm[1] * (double)out[i * dout + ns]);
    for (int k = 0; k < ns; ++k) W[(int64_t)k * ng + i] = (double)out[i * dout + k] * n;
    if (err_est) err_est[i] = out[i * dout + ns + 1];
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

inline int launch_status() { return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA; }

}  // namespace

extern "C" {

int chemgen_mlp_gemm(const void* A, int64_t sai, int64_t sar, const void* B, int64_t sbj, int64_t sbr, float* C,
                     int64_t ldc, int M, int N, int R, int accumulate, void* stream) {
    if (!A || !B || !C || M < 0 || N < 0 || R < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (M == 0 || N == 0) return CHEMGEN_OK;
    if (ldc < N) return CHEMGEN_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    // split r when the output tiles alone do not fill the GPU (weight
    // gradients: 256 x 256 outputs over a long batch)
    const int tiles = ((N + kBN - 1) / kBN) * ((M + kBM - 1) / kBM);
    int splits = 1;
    if (tiles < 148 && R >= 8 * kBR) splits = std::min((296 + tiles - 1) / tiles, R / (4 * kBR));
    const int rchunk = std::max(kBR, ((R + splits - 1) / splits + kBR - 1) / kBR * kBR);
    splits = std::max(1, (R + rchunk - 1) / rchunk);
    if (splits > 1 && !accumulate) {
        if (cudaMemset2DAsync(C, (size_t)ldc * sizeof(float), 0, (size_t)N * sizeof(float), (size_t)M, st) !=
            cudaSuccess)
            return CHEMGEN_ERR_CUDA;
    }
    dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM, splits);
    mlp_gemm_kernel<<<grid, 128, 0, st>>>((const bf16*)A, sai, sar, (const bf16*)B, sbj, sbr, C, ldc, M, N, R,
                                          rchunk, accumulate);
    return launch_status();
}

int chemgen_mlp_bias_gelu(float* Z, const float* bias, void* H, int64_t M, int N, int apply_gelu, void* stream) {
    if (!Z || !bias || M < 0 || N <= 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (M == 0) return CHEMGEN_OK;
    bias_gelu_kernel<<<blocks_for(M * N, 256), 256, 0, (cudaStream_t)stream>>>(Z, bias, (bf16*)H, M, N, apply_gelu);
    return launch_status();
}

int chemgen_mlp_gelu_backward(const float* dH, const float* Z, void* dZ, float* dZf, int64_t n, void* stream) {
    if (!dH || !Z || !dZ || n < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (n == 0) return CHEMGEN_OK;
    gelu_backward_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(dH, Z, (bf16*)dZ, dZf, n);
    return launch_status();
}

int chemgen_mlp_mse_grad(const float* out, const float* target, const float* colw, void* dout, float* doutf,
                         float* loss, int64_t M, int N, void* stream) {
    if (!out || !target || !colw || !dout || !loss || M < 0 || N <= 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (M == 0) return CHEMGEN_OK;
    mse_grad_kernel<<<blocks_for(M * N, 256), 256, 0, (cudaStream_t)stream>>>(out, target, colw, (bf16*)dout, doutf,
                                                                              loss, M, N);
    return launch_status();
}

int chemgen_mlp_colsum(const float* dZ, float* db, int64_t M, int N, void* stream) {
    if (!dZ || !db || M < 0 || N <= 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    colsum_kernel<<<N, 256, 0, (cudaStream_t)stream>>>(dZ, db, M, N);
    return launch_status();
}

int chemgen_mlp_adam(float* w, const float* g, float* m, float* v, void* wb, int64_t n, const float* hyper, float b1,
                     float b2, float eps, float wd, void* stream) {
    if (!w || !g || !m || !v || !hyper || n < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (n == 0) return CHEMGEN_OK;
    adam_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (bf16*)wb, n, hyper, b1, b2, eps,
                                                                      wd);
    return launch_status();
}

int chemgen_surrogate_features(const double* P, const double* T, const double* Y, int64_t ng, int ns, int din,
                               const float* norm, const double* inv_mw, void* X, float* Xf, void* stream) {
    if (!P || !T || !Y || !norm || !X || ng < 0 || ns < 1 || din < ns + 3) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (ng == 0) return CHEMGEN_OK;
    features_kernel<<<blocks_for(ng, 128), 128, 0, (cudaStream_t)stream>>>(P, T, Y, ng, ns, din, norm, inv_mw,
                                                                         (bf16*)X, Xf);
    return launch_status();
}

int chemgen_surrogate_targets(const double* W, int64_t ng, int ns, int dout, const float* lnorm, float* Tg,
                              void* stream) {
    if (!W || !lnorm || !Tg || ng < 0 || ns < 1 || dout < ns + 1) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (ng == 0) return CHEMGEN_OK;
    targets_kernel<<<blocks_for(ng, 128), 128, 0, (cudaStream_t)stream>>>(W, ng, ns, dout, lnorm, Tg);
    return launch_status();
}

int chemgen_surrogate_decode(const float* out, int64_t ng, int ns, int dout, const float* lnorm, double* W,
                             float* err_est, void* stream) {
    if (!out || !lnorm || !W || ng < 0 || ns < 1 || dout < ns + 2) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (ng == 0) return CHEMGEN_OK;
    decode_kernel<<<blocks_for(ng, 128), 128, 0, (cudaStream_t)stream>>>(out, ng, ns, dout, lnorm, W, err_est);
    return launch_status();
}

}  // extern "C"
