// Training products of the wdot surrogate on the 5th-generation tensor cores
// (tcgen05), each fused with the elementwise work that follows it.
//
// One kernel computes acc[m][n] = sum_k A[m][k] B[n][k] for a 128-row tile of
// A and a 32/64/128-column tile of B, both BF16 and K-major in global memory
// (rows of lda / ldb elements), with FP32 accumulation in tensor memory:
// * K runs in chunks of 64; all 128 threads copy a chunk of A and of B into
//   shared memory in the canonical no-swizzle K-major layout (16-byte
//   cp.async copies, one per core-matrix row), two stages deep, while the
//   tensor core works on the previous chunk; one thread issues the four
//   M = 128, N = tile, K = 16 MMAs of a chunk and commits them to the stage's
//   mbarrier.
// * The epilogue reads the accumulator from tensor memory (warp w owns rows
//   32 w .. 32 w + 31, one row per thread) and applies one of
//     STORE          C[m][n] (+)= acc                   (weight gradients)
//     STORE_T        C[n][m] (+)= acc                   (weight gradients, transposed)
//     BIAS_GELU      z = acc + b[n]; C = z; H = GELU(z) (hidden layers, forward)
//     BIAS           C = acc + b[n]                     (output layer)
//     GELU_BACKWARD  d = acc * GELU'(Zprev[m][n]); C = d (input gradient of
//                    the layer below, through its activation)
//   where H (BF16, row-major) and HT (BF16, transposed: HT[n][m]) are the
//   next products' operands.  The batch is the reduction dimension of the
//   weight gradients dW = dZ^T H, so those take the transposed copies as
//   their K-major operands; the forward and input-gradient products read the
//   row-major ones.
//
// Every mbarrier wait is bounded; a time-out sets an error word that
// chemgen_mlp_tc_error reports, and the kernel still frees its tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/chemgen_b200.h"
#include "mlp_act.cuh"
#include "umma.cuh"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kTM = 128;    // rows per tile (MMA M, tensor-memory lanes)
constexpr int kKC = 64;     // K per pipeline stage
constexpr int kStages = 3;  // shared-memory stages (two chunks in flight beside the one computed)
enum { kStore = 0, kStoreT = 1, kBiasGelu = 2, kBias = 3, kGeluBack = 4 };

__device__ int g_mlp_tc_err = 0;

struct TcArgs {
    const bf16* A;
    int64_t lda;
    const bf16* B;
    int64_t ldb;
    int M, N, K;
    int epi;
    const float* bias;
    const float* zprev;
    int64_t ldz;
    float* C;
    int64_t ldc;
    bf16* H;
    int64_t ldh;
    bf16* HT;
    int64_t ldt;
    int accumulate;
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(um::smem_addr(dst)),
                 "l"((uint64_t)__cvta_generic_to_global(src))
                 : "memory");
}


template <int NT>
__global__ void __launch_bounds__(128) mlp_gemm_tc_kernel(TcArgs g) {
    extern __shared__ __align__(1024) unsigned char sm[];
    constexpr int kABytes = kTM * kKC * 2;
    constexpr int kBBytes = NT * kKC * 2;
    constexpr int kStage = kABytes + kBBytes;
    constexpr uint32_t kCols = NT < 32 ? 32u : (uint32_t)NT;
    constexpr int kPipe = kStages * kStage, kEpi = 4 * 32 * ((NT + 4) * 4 + (NT + 8) * 2);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + (kPipe > kEpi ? kPipe : kEpi));
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + kStages);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * NT;
    const int kc0 = 0, kc1 = g.K / kKC;
    if (tid == 0) {
        for (int i = 0; i < kStages; ++i) um::mbar_init(&mbar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) um::tmem_alloc(tslot, kCols);
    um::fence_before_sync();
    __syncthreads();
    um::fence_after_sync();
    const uint32_t tbase = *tslot;
    const uint32_t idesc = um::idesc_bf16(kTM, NT);
    uint32_t parity[kStages] = {};
    bool ok = true;
    auto load = [&](int kc, int st) {
        const int k0 = kc * kKC;
        unsigned char* sA = sm + st * kStage;
        unsigned char* sB = sA + kABytes;
        for (int c = tid; c < kTM * 8; c += 128) {
            const int r = c >> 3, kk = (c & 7) * 8;
            cp_async16(sA + um::kmajor_offset(r, kk, kKC), g.A + (int64_t)(m0 + r) * g.lda + k0 + kk);
        }
        for (int c = tid; c < NT * 8; c += 128) {
            const int r = c >> 3, kk = (c & 7) * 8;
            cp_async16(sB + um::kmajor_offset(r, kk, kKC), g.B + (int64_t)(n0 + r) * g.ldb + k0 + kk);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // the copies of the next chunk fly while the tensor core works on this one
    if (kc0 < kc1) load(kc0, 0);
    for (int kc = kc0; kc < kc1; ++kc) {
        const int it = kc - kc0, st = it % kStages;
        if (kc + 1 < kc1) {
            const int st1 = (it + 1) % kStages;
            if (it + 1 >= kStages) {
                // the MMAs that read stage st1 (chunk it + 1 - kStages) have finished
                ok = um::mbar_wait(&mbar[st1], parity[st1]) && ok;
                parity[st1] ^= 1u;
            }
            load(kc + 1, st1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        um::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            um::fence_after_sync();
            const uint32_t a = um::smem_addr(sm + st * kStage), b = um::smem_addr(sm + st * kStage + kABytes);
#pragma unroll
            for (int ks = 0; ks < kKC / 16; ++ks)
                um::mma_bf16(tbase, um::desc_kmajor(a, kKC, ks), um::desc_kmajor(b, kKC, ks), idesc,
                             (it > 0 || ks > 0) ? 1u : 0u);
            um::commit(&mbar[st]);
        }
    }
    // the commits not yet waited for (the last min(kStages, chunks) ones)
    const int nit = kc1 - kc0;
    for (int j = nit > kStages ? nit - kStages : 0; j < nit; ++j) {
        const int st = j % kStages;
        ok = um::mbar_wait(&mbar[st], parity[st]) && ok;
        parity[st] ^= 1u;
    }
    um::fence_after_sync();
    const int m = m0 + 32 * warp + lane;
    if (ok && nit > 0) {
        // Epilogue.  Thread `lane` of warp w holds accumulator row m0 + 32 w +
        // lane; the row-major outputs (C, H) and the zprev input go through a
        // per-warp shared-memory stage ([32][NT + 4] FP32 and [32][NT + 8]
        // BF16, in the pipeline's buffers, now idle), so that global memory
        // sees whole rows; the transposed outputs (C for STORE_T, HT) are
        // stored straight from the thread, where lanes already run along m.
        constexpr int kLd = NT + 4, kLh = NT + 8;
        float* stg = reinterpret_cast<float*>(sm) + warp * 32 * kLd;
        bf16* hst = reinterpret_cast<bf16*>(reinterpret_cast<float*>(sm) + 4 * 32 * kLd) + warp * 32 * kLh;
        const int64_t mrow0 = m0 + 32 * warp;
        const bool rowC = g.C && g.epi != kStoreT;
        const bool rowH = g.H != nullptr;
        if (g.epi == kGeluBack) {
            for (int r = 0; r < 32; ++r)
                for (int c = 4 * lane; c < NT; c += 128)
                    *reinterpret_cast<float4*>(stg + r * kLd + c) =
                        __ldg(reinterpret_cast<const float4*>(g.zprev + (mrow0 + r) * g.ldz + n0 + c));
            __syncwarp();
        }
#pragma unroll 1
        for (int c0 = 0; c0 < NT; c0 += 16) {
            float v[16];
            um::tmem_ld16(um::tmem_lane_addr(tbase, warp, c0), v);
            const int nb = n0 + c0;
            float* srow = stg + lane * kLd + c0;
            if (g.epi == kStoreT) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    float* c = g.C + (int64_t)(nb + j) * g.ldc + m;
                    *c = g.accumulate ? *c + v[j] : v[j];
                }
                continue;
            }
            if (g.epi == kGeluBack) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 z = *reinterpret_cast<const float4*>(srow + 4 * q);
                    float d;
                    gelu(z.x, &d); v[4 * q] *= d;
                    gelu(z.y, &d); v[4 * q + 1] *= d;
                    gelu(z.z, &d); v[4 * q + 2] *= d;
                    gelu(z.w, &d); v[4 * q + 3] *= d;
                }
            } else if (g.epi == kBias || g.epi == kBiasGelu) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] += __ldg(g.bias + nb + j);
            }
            if (rowC)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    *reinterpret_cast<float4*>(srow + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            if (g.epi == kStore) continue;
            uint32_t hb[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float h0 = v[2 * j], h1 = v[2 * j + 1];
                if (g.epi == kBiasGelu) {
                    h0 = gelu(h0, nullptr);
                    h1 = gelu(h1, nullptr);
                }
                const __nv_bfloat162 pr = __floats2bfloat162_rn(h0, h1);
                hb[j] = *reinterpret_cast<const uint32_t*>(&pr);
            }
            if (rowH) {
                uint4* hrow = reinterpret_cast<uint4*>(hst + lane * kLh + c0);
                hrow[0] = make_uint4(hb[0], hb[1], hb[2], hb[3]);
                hrow[1] = make_uint4(hb[4], hb[5], hb[6], hb[7]);
            }
            if (g.HT)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    g.HT[(int64_t)(nb + 2 * j) * g.ldt + m] = __ushort_as_bfloat16((unsigned short)(hb[j] & 0xffffu));
                    g.HT[(int64_t)(nb + 2 * j + 1) * g.ldt + m] = __ushort_as_bfloat16((unsigned short)(hb[j] >> 16));
                }
        }
        __syncwarp();
        // whole rows out: FP32 C (4 floats a lane), BF16 H (8 a lane)
        if (rowC)
            for (int r = 0; r < 32; ++r)
                for (int c = 4 * lane; c < NT; c += 128) {
                    const float4 x = *reinterpret_cast<const float4*>(stg + r * kLd + c);
                    float* dst = g.C + (mrow0 + r) * g.ldc + n0 + c;
                    if (g.accumulate) {
                        float4 y = *reinterpret_cast<const float4*>(dst);
                        y.x += x.x; y.y += x.y; y.z += x.z; y.w += x.w;
                        *reinterpret_cast<float4*>(dst) = y;
                    } else {
                        *reinterpret_cast<float4*>(dst) = x;
                    }
                }
        if (rowH)
            for (int r = 0; r < 32; ++r)
                for (int c = 8 * lane; c < NT; c += 256)
                    *reinterpret_cast<uint4*>(g.H + (mrow0 + r) * g.ldh + n0 + c) =
                        *reinterpret_cast<const uint4*>(hst + r * kLh + c);
    }
    if (!ok && lane == 0) atomicExch(&g_mlp_tc_err, 1);
    um::fence_before_sync();
    __syncthreads();
    if (warp == 0) um::tmem_dealloc(tbase, kCols);
}

template <int NT>
cudaError_t launch_tc(const TcArgs& a, cudaStream_t s) {
    // the pipeline's stages, or the epilogue's per-warp stages if larger
    const size_t pipe = kStages * (size_t)(kTM * kKC * 2 + NT * kKC * 2);
    const size_t epi = 4 * 32 * ((size_t)(NT + 4) * 4 + (size_t)(NT + 8) * 2);
    const size_t smem = std::max(pipe, epi) + 64;
    cudaError_t e = cudaFuncSetAttribute(mlp_gemm_tc_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    // one CTA per output tile over the whole of K: every sum is formed in one
    // order, so that training is reproducible run to run (a split of K with
    // atomic adds was ~20 % faster on the weight gradients and was not)
    dim3 grid((unsigned)(a.M / kTM), (unsigned)(a.N / NT), 1u);
    mlp_gemm_tc_kernel<NT><<<grid, 128, smem, s>>>(a);
    return cudaGetLastError();
}

bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

extern "C" int chemgen_mlp_gemm_tc(const void* A, int64_t lda, const void* B, int64_t ldb, int M, int N, int K,
                                   int epilogue, const float* bias, const float* zprev, int64_t ldz, float* C,
                                   int64_t ldc, void* H, int64_t ldh, void* HT, int64_t ldt, int accumulate,
                                   void* stream) {
    if (!A || !B || M < 0 || N < 0 || K < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (M == 0 || N == 0) return CHEMGEN_OK;
    if (M % kTM || K == 0 || K % kKC || !(N == 32 || N == 64 || N % 128 == 0)) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (epilogue < kStore || epilogue > kGeluBack) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if ((epilogue == kStore || epilogue == kStoreT || epilogue == kBias) && !C) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if ((epilogue == kBiasGelu || epilogue == kBias) && !bias) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (epilogue == kGeluBack && (!zprev || ldz < N)) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (lda < K || ldb < K || (C && ldc < (epilogue == kStoreT ? M : N)) || (H && ldh < N) || (HT && ldt < M))
        return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (!al16(A) || !al16(B) || (lda & 7) || (ldb & 7)) return CHEMGEN_ERR_MISALIGNED;
    // the epilogue moves whole rows of C / zprev (4 floats) and H (8 BF16) at a time
    if (C && epilogue != kStoreT && (!al16(C) || (ldc & 3))) return CHEMGEN_ERR_MISALIGNED;
    if (epilogue == kGeluBack && (!al16(zprev) || (ldz & 3))) return CHEMGEN_ERR_MISALIGNED;
    if (H && (!al16(H) || (ldh & 7))) return CHEMGEN_ERR_MISALIGNED;
    TcArgs a{(const bf16*)A, lda, (const bf16*)B, ldb, M, N, K, epilogue, bias, zprev, ldz,
             C, ldc, (bf16*)H, ldh, (bf16*)HT, ldt, accumulate};
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (N <= 32) e = launch_tc<32>(a, s);
    else if (N <= 64) e = launch_tc<64>(a, s);
    else e = launch_tc<128>(a, s);
    return e == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

extern "C" int chemgen_mlp_tc_error(int reset) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_mlp_tc_err, sizeof(int)) != cudaSuccess) return -1;
    if (reset) {
        const int z = 0;
        if (cudaMemcpyToSymbol(g_mlp_tc_err, &z, sizeof(int)) != cudaSuccess) return -1;
    }
    return v;
}

namespace {
// dst[c * ldd + r] = src[r * lds + c] for r < rows, c < cols (BF16), through a
// 32 x 32 shared-memory tile so that both sides are coalesced.
__global__ void transpose_bf16_kernel(const bf16* __restrict__ src, int64_t lds, bf16* __restrict__ dst, int64_t ldd,
                                      int rows, int cols) {
    __shared__ bf16 t[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        if (r < rows && c < cols) t[y][threadIdx.x] = src[(int64_t)r * lds + c];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[(int64_t)c * ldd + r] = t[threadIdx.x][y];
    }
}
}  // namespace

extern "C" int chemgen_mlp_transpose_bf16(const void* src, int64_t lds, int rows, int cols, void* dst, int64_t ldd,
                                          void* stream) {
    if (!src || !dst || rows < 0 || cols < 0 || lds < cols || ldd < rows) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (rows == 0 || cols == 0) return CHEMGEN_OK;
    dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
    transpose_bf16_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const bf16*)src, lds, (bf16*)dst, ldd, rows,
                                                                        cols);
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

namespace {
// One Adam step over all of the network's tensors in one launch, which also
// writes the operands the tensor-core products read: the BF16 copy of a
// weight matrix [rows x cols] (wb), its transpose [cols x rows] (wt) and the
// first layer's doubled copy [rows x 2 cols] for its hi + lo inputs (wd).
constexpr int kAdamMax = 8;
struct AdamTensor {
    float* w;
    const float* g;
    float* m;
    float* v;
    bf16* wb;
    bf16* wt;
    bf16* wd;
    int rows, cols;
    float decay;
};
struct AdamArgs {
    AdamTensor t[kAdamMax];
    int64_t off[kAdamMax + 1];
    int count;
    const float* hyper;
    float b1, b2, eps;
};

__global__ void adam_multi_kernel(AdamArgs a) {
    const float lr = a.hyper[0], c1 = a.hyper[1], c2 = a.hyper[2];
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.off[a.count];
         e += (int64_t)gridDim.x * blockDim.x) {
        int k = 0;
        while (k + 1 < a.count && e >= a.off[k + 1]) ++k;
        const AdamTensor& t = a.t[k];
        const int64_t i = e - a.off[k];
        const float gi = t.g[i] + t.decay * t.w[i];
        const float mi = a.b1 * t.m[i] + (1.0f - a.b1) * gi;
        const float vi = a.b2 * t.v[i] + (1.0f - a.b2) * gi * gi;
        t.m[i] = mi;
        t.v[i] = vi;
        const float wi = t.w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + a.eps);
        t.w[i] = wi;
        const bf16 h = __float2bfloat16(wi);
        if (t.wb) t.wb[i] = h;
        const int r = (int)(i / t.cols), c = (int)(i % t.cols);
        if (t.wt) t.wt[(int64_t)c * t.rows + r] = h;
        if (t.wd) {
            t.wd[(int64_t)r * 2 * t.cols + c] = h;
            t.wd[(int64_t)r * 2 * t.cols + t.cols + c] = h;
        }
    }
}
}  // namespace

extern "C" int chemgen_mlp_adam_multi(int count, float* const* w, const float* const* g, float* const* m,
                                      float* const* v, void* const* wb, void* const* wt, void* const* wd,
                                      const int* rows, const int* cols, const float* decay, const float* hyper,
                                      float b1, float b2, float eps, void* stream) {
    if (count < 1 || count > kAdamMax || !w || !g || !m || !v || !rows || !cols || !hyper)
        return CHEMGEN_ERR_INVALID_ARGUMENT;
    AdamArgs a{};
    a.count = count;
    a.hyper = hyper;
    a.b1 = b1;
    a.b2 = b2;
    a.eps = eps;
    a.off[0] = 0;
    for (int k = 0; k < count; ++k) {
        if (!w[k] || !g[k] || !m[k] || !v[k] || rows[k] < 1 || cols[k] < 1) return CHEMGEN_ERR_INVALID_ARGUMENT;
        a.t[k] = AdamTensor{w[k], g[k], m[k], v[k], wb ? (bf16*)wb[k] : nullptr, wt ? (bf16*)wt[k] : nullptr,
                            wd ? (bf16*)wd[k] : nullptr, rows[k], cols[k], decay ? decay[k] : 0.0f};
        a.off[k + 1] = a.off[k] + (int64_t)rows[k] * cols[k];
    }
    const int64_t n = a.off[count];
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 4096);
    adam_multi_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Fused training passes.  One CTA of 256 threads owns a tile of 128 batch
// rows (tensor-memory lanes) and runs a whole chain of products on it, the
// activations staying in shared memory between layers:
//   forward : Z_l = H_{l-1} W_l^T + b_l, H_l = GELU(Z_l) for the three hidden
//             layers (H_{-1} = the input), out = H_2 W_3^T + b_3;
//   backward: dZ_2 = (dout W_3) * GELU'(Z_2), dZ_1 = (dZ_2 W_2) * GELU'(Z_1),
//             dZ_0 = (dZ_1 W_1) * GELU'(Z_0), and the bias gradients
//             (column sums of dZ_l over the batch).
// Per layer one thread issues the K/16 MMAs (M = 128, N = 256 or 64, BF16,
// FP32 accumulation in 256 tensor-memory columns) against the layer's B
// operand, which all threads copy into shared memory (16-byte cp.async into
// the canonical K-major layout) while the previous epilogue runs.  Warp w
// reads lane quadrant w % 4 and column quarter w / 4 of the accumulator.  What
// the weight-gradient products need leaves transposed, [feature][row], where
// a warp's lanes write consecutive addresses: Z_l (FP32), H_l and dZ_l (BF16),
// dout.  Shared memory: 64 KB activations, 32 KB input, 128 KB weights.
namespace {
constexpr int kFR = 128, kFT = 512, kFHid = 256, kFOut = 64;   // 16 warps: 4 per lane quadrant
constexpr uint32_t kFAOff = 0, kFXOff = kFR * kFHid * 2, kFWOff = kFXOff + kFR * 128 * 2,
                   kFTail = kFWOff + kFHid * kFHid * 2;
constexpr size_t kFSmem = (size_t)kFTail + 64;

// rows x K BF16 (row stride ld elements, K-major) -> canonical K-major tile
__device__ __forceinline__ void fused_load(unsigned char* dst, const bf16* src, int64_t ld, int rows, int K) {
    const int per = K / 8;
    for (int c = threadIdx.x; c < rows * per; c += kFT) {
        const int r = c / per, kk = (c - r * per) * 8;
        cp_async16(dst + um::kmajor_offset(r, kk, K), src + (int64_t)r * ld + kk);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void fused_mma(uint32_t tbase, const unsigned char* a, const unsigned char* b, int K,
                                          int N, uint64_t* bar) {
    um::fence_after_sync();
    const uint32_t idesc = um::idesc_bf16(kFR, N), sa = um::smem_addr(a), sb = um::smem_addr(b);
    for (int ks = 0; ks < K / 16; ++ks)
        um::mma_bf16(tbase, um::desc_kmajor(sa, K, ks), um::desc_kmajor(sb, K, ks), idesc, ks > 0 ? 1u : 0u);
    um::commit(bar);
}

// copies landed and shared-memory writes visible to the tensor core; tensor
// memory reads ordered before the next MMA
__device__ __forceinline__ void fused_step_end() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    um::fence_proxy_async();
    um::fence_before_sync();
    __syncthreads();
}

struct FwdArgs {
    const bf16* X;
    int64_t ldx;
    int K0;
    const bf16* W[4];
    const float* b[4];
    int B;
    float* ZT[3];
    bf16* HT[3];
    float* out;
};

__global__ void __launch_bounds__(kFT, 1) mlp_forward_fused_kernel(FwdArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* sA = sm + kFAOff;
    unsigned char* sX = sm + kFXOff;
    unsigned char* sW = sm + kFWOff;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kFTail);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g4 = warp & 3, qtr = warp >> 2, row = 32 * g4 + lane;
    const int64_t m0 = (int64_t)blockIdx.x * kFR, m = m0 + row;
    if (tid == 0) {
        um::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) um::tmem_alloc(tslot, 256);
    fused_load(sX, a.X + m0 * a.ldx, a.ldx, kFR, a.K0);
    fused_load(sW, a.W[0], a.K0, kFHid, a.K0);
    fused_step_end();
    um::fence_after_sync();
    const uint32_t tbase = *tslot;
    uint32_t parity = 0;
    bool ok = true;
    for (int l = 0; l < 4 && ok; ++l) {
        const int K = l == 0 ? a.K0 : kFHid, N = l == 3 ? kFOut : kFHid;
        if (tid == 0) fused_mma(tbase, l == 0 ? sX : sA, sW, K, N, bar);
        ok = um::mbar_wait(bar, parity);
        parity ^= 1u;
        um::fence_after_sync();
        if (!ok) break;
        // the next layer's weights stream in while this epilogue runs
        if (l < 3) fused_load(sW, a.W[l + 1], kFHid, l == 2 ? kFOut : kFHid, kFHid);
        if (l < 3) {
            const float* __restrict__ bl = a.b[l];
            float* __restrict__ zt = a.ZT[l];
            bf16* __restrict__ ht = a.HT[l];
#pragma unroll 1
            for (int c = 64 * qtr; c < 64 * qtr + 64; c += 16) {
                float bb[16], v[16];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 t = __ldg(reinterpret_cast<const float4*>(bl + c) + q);
                    bb[4 * q] = t.x;
                    bb[4 * q + 1] = t.y;
                    bb[4 * q + 2] = t.z;
                    bb[4 * q + 3] = t.w;
                }
                um::tmem_ld16(um::tmem_lane_addr(tbase, g4, c), v);
                uint32_t pk[8];
#pragma unroll
                for (int j = 0; j < 16; j += 2) {
                    const float z0 = v[j] + bb[j], z1 = v[j + 1] + bb[j + 1];
                    zt[(int64_t)(c + j) * a.B + m] = z0;
                    zt[(int64_t)(c + j + 1) * a.B + m] = z1;
                    const __nv_bfloat162 h = __floats2bfloat162_rn(gelu(z0, nullptr), gelu(z1, nullptr));
                    ht[(int64_t)(c + j) * a.B + m] = h.x;
                    ht[(int64_t)(c + j + 1) * a.B + m] = h.y;
                    pk[j / 2] = *reinterpret_cast<const uint32_t*>(&h);
                }
                *reinterpret_cast<uint4*>(sA + um::kmajor_offset(row, c, kFHid)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                *reinterpret_cast<uint4*>(sA + um::kmajor_offset(row, c + 8, kFHid)) =
                    make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
        } else {
            {
                const int c = 16 * qtr;
                float v[16];
                um::tmem_ld16(um::tmem_lane_addr(tbase, g4, c), v);
                float4* o = reinterpret_cast<float4*>(a.out + m * kFOut + c);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    o[q] = make_float4(v[4 * q] + __ldg(a.b[3] + c + 4 * q), v[4 * q + 1] + __ldg(a.b[3] + c + 4 * q + 1),
                                       v[4 * q + 2] + __ldg(a.b[3] + c + 4 * q + 2),
                                       v[4 * q + 3] + __ldg(a.b[3] + c + 4 * q + 3));
            }
        }
        fused_step_end();
    }
    if (!ok && lane == 0) atomicExch(&g_mlp_tc_err, 1);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    um::fence_before_sync();
    __syncthreads();
    if (warp == 0) um::tmem_dealloc(tbase, 256);
}

struct BwdArgs {
    const bf16* dout;      // [B x 64]
    const bf16* WT[4];     // W_l^T [in x out]; 1..3 used
    const float* ZT[3];
    int B;
    bf16* dZT[3];
    float* gb[3];          // column sums of dZ_l
    bf16* doutT;           // [64 x B]
    float* part;           // [3][B / 128][256] per-tile column sums
    unsigned* count;       // tiles done (the last one forms gb and resets it)
};

__global__ void __launch_bounds__(kFT, 1) mlp_backward_fused_kernel(BwdArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* sA = sm + kFAOff;
    unsigned char* sX = sm + kFXOff;
    unsigned char* sW = sm + kFWOff;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kFTail);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g4 = warp & 3, qtr = warp >> 2, row = 32 * g4 + lane;
    const int64_t m0 = (int64_t)blockIdx.x * kFR, m = m0 + row;
    if (tid == 0) {
        um::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) um::tmem_alloc(tslot, 256);
    fused_load(sX, a.dout + m0 * kFOut, kFOut, kFR, kFOut);
    fused_load(sW, a.WT[3], kFOut, kFHid, kFOut);
    fused_step_end();
    um::fence_after_sync();
    const uint32_t tbase = *tslot;
    // dout transposed for the last layer's weight gradient, from the tile copy
    for (int n = 16 * qtr; n < 16 * qtr + 16; ++n)
        a.doutT[(int64_t)n * a.B + m] = *reinterpret_cast<const bf16*>(sX + um::kmajor_offset(row, n, kFOut));
    __syncthreads();   // the epilogues reuse sX for the column sums
    float* red = reinterpret_cast<float*>(sX);   // [3 layers][4 lane quadrants][256], used from step 0's epilogue
    uint32_t parity = 0;
    bool ok = true;
    for (int s = 0; s < 3 && ok; ++s) {
        const int L = 3 - s, K = s == 0 ? kFOut : kFHid;     // weight layer, its output width
        if (tid == 0) fused_mma(tbase, s == 0 ? sX : sA, sW, K, kFHid, bar);
        ok = um::mbar_wait(bar, parity);
        parity ^= 1u;
        um::fence_after_sync();
        if (!ok) break;
        if (s < 2) fused_load(sW, a.WT[L - 1], kFHid, kFHid, kFHid);
        const float* __restrict__ z = a.ZT[L - 1];
        bf16* __restrict__ dzt = a.dZT[L - 1];
#pragma unroll 1
        for (int c = 64 * qtr; c < 64 * qtr + 64; c += 16) {
            // the 16 pre-activations first (one L2 round trip for all), then the accumulator
            float zv[16], v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) zv[j] = __ldcg(z + (int64_t)(c + j) * a.B + m);
            um::tmem_ld16(um::tmem_lane_addr(tbase, g4, c), v);
            uint32_t pk[8];
#pragma unroll
            for (int j = 0; j < 16; j += 2) {
                float d0, d1;
                gelu(zv[j], &d0);
                gelu(zv[j + 1], &d1);
                v[j] *= d0;
                v[j + 1] *= d1;
                const __nv_bfloat162 h = __floats2bfloat162_rn(v[j], v[j + 1]);
                dzt[(int64_t)(c + j) * a.B + m] = h.x;
                dzt[(int64_t)(c + j + 1) * a.B + m] = h.y;
                pk[j / 2] = *reinterpret_cast<const uint32_t*>(&h);
            }
            if (s < 2) {
                *reinterpret_cast<uint4*>(sA + um::kmajor_offset(row, c, kFHid)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                *reinterpret_cast<uint4*>(sA + um::kmajor_offset(row, c + 8, kFHid)) =
                    make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
            // bias gradient: the column sums of this warp's 32 rows (FP32),
            // kept per lane quadrant in the input buffer, idle after step 0
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                float t = v[j];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                if (lane == 0) red[((L - 1) * 4 + g4) * kFHid + c + j] = t;
            }
        }
        fused_step_end();
    }
    if (!ok && lane == 0) atomicExch(&g_mlp_tc_err, 1);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    um::fence_before_sync();
    __syncthreads();
    if (warp == 0) um::tmem_dealloc(tbase, 256);
    // bias gradients in a fixed order: this tile's column sums (quadrants in
    // order), then the last tile to finish adds the tiles' sums in order
    __shared__ unsigned last;
    const int nt = gridDim.x, col = tid;
    if (ok && col < kFHid)
        for (int l = 0; l < 3; ++l) {
            const float* q = red + l * 4 * kFHid + col;
            a.part[((int64_t)l * nt + blockIdx.x) * kFHid + col] = ((q[0] + q[kFHid]) + q[2 * kFHid]) + q[3 * kFHid];
        }
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(a.count, 1u) == (unsigned)(nt - 1);
    __syncthreads();
    if (last && col < kFHid) {
        __threadfence();
        for (int l = 0; l < 3; ++l) {
            float acc = 0.0f;
            for (int t = 0; t < nt; ++t) acc += __ldcg(a.part + ((int64_t)l * nt + t) * kFHid + col);
            a.gb[l][col] = acc;
        }
        if (tid == 0) *a.count = 0u;
    }
}

bool fused_ready() {
    static int st = -1;
    if (st < 0) {
        st = cudaFuncSetAttribute(mlp_forward_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kFSmem) == cudaSuccess &&
                     cudaFuncSetAttribute(mlp_backward_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kFSmem) == cudaSuccess
                 ? 1
                 : 0;
    }
    return st == 1;
}
}  // namespace

extern "C" int chemgen_mlp_forward_tc(const void* X, int64_t ldx, int K0, const void* const* W, const float* const* b,
                                      int B, float* const* ZT, void* const* HT, float* out, void* stream) {
    if (!X || !W || !b || !ZT || !HT || !out || B <= 0 || B % kFR || (K0 != 64 && K0 != 128) || ldx < K0)
        return CHEMGEN_ERR_INVALID_ARGUMENT;
    FwdArgs a{};
    a.X = (const bf16*)X;
    a.ldx = ldx;
    a.K0 = K0;
    a.B = B;
    a.out = out;
    for (int l = 0; l < 4; ++l) {
        if (!W[l] || !b[l] || !al16(W[l])) return W[l] && b[l] ? CHEMGEN_ERR_MISALIGNED : CHEMGEN_ERR_INVALID_ARGUMENT;
        a.W[l] = (const bf16*)W[l];
        a.b[l] = b[l];
    }
    for (int l = 0; l < 3; ++l) {
        if (!ZT[l] || !HT[l]) return CHEMGEN_ERR_INVALID_ARGUMENT;
        a.ZT[l] = ZT[l];
        a.HT[l] = (bf16*)HT[l];
    }
    if (!al16(X) || (ldx & 7) || !al16(out)) return CHEMGEN_ERR_MISALIGNED;
    if (!fused_ready()) return CHEMGEN_ERR_CUDA;
    mlp_forward_fused_kernel<<<B / kFR, kFT, kFSmem, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

extern "C" size_t chemgen_mlp_backward_tc_work_bytes(int B) {
    return B > 0 ? (size_t)3 * ((B + kFR - 1) / kFR) * kFHid * sizeof(float) + 16 : 0;
}

extern "C" int chemgen_mlp_backward_tc(const void* dout, const void* const* WT, const float* const* ZT, int B,
                                       void* const* dZT, float* const* gb, void* doutT, void* work, void* stream) {
    if (!dout || !WT || !ZT || !dZT || !gb || !doutT || !work || B <= 0 || B % kFR)
        return CHEMGEN_ERR_INVALID_ARGUMENT;
    BwdArgs a{};
    a.dout = (const bf16*)dout;
    a.B = B;
    a.doutT = (bf16*)doutT;
    a.part = (float*)work;
    a.count = (unsigned*)((char*)work + chemgen_mlp_backward_tc_work_bytes(B) - 16);
    if (!al16(work)) return CHEMGEN_ERR_MISALIGNED;
    for (int l = 1; l < 4; ++l) {
        if (!WT[l]) return CHEMGEN_ERR_INVALID_ARGUMENT;
        if (!al16(WT[l])) return CHEMGEN_ERR_MISALIGNED;
        a.WT[l] = (const bf16*)WT[l];
    }
    for (int l = 0; l < 3; ++l) {
        if (!ZT[l] || !dZT[l] || !gb[l]) return CHEMGEN_ERR_INVALID_ARGUMENT;
        a.ZT[l] = ZT[l];
        a.dZT[l] = (bf16*)dZT[l];
        a.gb[l] = gb[l];
    }
    if (!al16(dout)) return CHEMGEN_ERR_MISALIGNED;
    if (!fused_ready()) return CHEMGEN_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    mlp_backward_fused_kernel<<<B / kFR, kFT, kFSmem, s>>>(a);
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}
