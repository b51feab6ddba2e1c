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

__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

template <int NT>
__global__ void __launch_bounds__(128) mlp_gemm_tc_kernel(TcArgs g) {
    extern __shared__ __align__(1024) unsigned char sm[];
    constexpr int kABytes = kTM * kKC * 2;
    constexpr int kBBytes = NT * kKC * 2;
    constexpr int kStage = kABytes + kBBytes;
    constexpr uint32_t kCols = NT < 32 ? 32u : (uint32_t)NT;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kStages * kStage);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + kStages);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * NT;
    // this CTA's share of K (split-K: blockIdx.z of gridDim.z, whole chunks)
    const int nkc = g.K / kKC;
    const int per = (nkc + gridDim.z - 1) / gridDim.z;
    const int kc0 = blockIdx.z * per, kc1 = min(nkc, kc0 + per);
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
#pragma unroll 1
        for (int c0 = 0; c0 < NT; c0 += 16) {
            float v[16];
            um::tmem_ld16(um::tmem_lane_addr(tbase, warp, c0), v);
            const int nb = n0 + c0;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int n = nb + j;
                float x = v[j];
                if (g.epi == kStore || g.epi == kStoreT) {
                    float* c = g.epi == kStore ? g.C + (int64_t)m * g.ldc + n : g.C + (int64_t)n * g.ldc + m;
                    if (gridDim.z > 1) atomicAdd(c, x);
                    else *c = g.accumulate ? *c + x : x;
                } else {
                    if (g.epi == kGeluBack) {
                        float d;
                        gelu(g.zprev[(int64_t)m * g.ldz + n], &d);
                        x *= d;
                    } else {
                        x += g.bias[n];
                    }
                    if (g.C) g.C[(int64_t)m * g.ldc + n] = x;
                    const float h = g.epi == kBiasGelu ? gelu(x, nullptr) : x;
                    const bf16 hb = __float2bfloat16(h);
                    if (g.H) g.H[(int64_t)m * g.ldh + n] = hb;
                    if (g.HT) g.HT[(int64_t)n * g.ldt + m] = hb;
                }
            }
        }
    }
    if (!ok && lane == 0) atomicExch(&g_mlp_tc_err, 1);
    um::fence_before_sync();
    __syncthreads();
    if (warp == 0) um::tmem_dealloc(tbase, kCols);
}

template <int NT>
cudaError_t launch_tc(const TcArgs& a, cudaStream_t s) {
    const size_t smem = kStages * (size_t)(kTM * kKC * 2 + NT * kKC * 2) + 64;
    cudaError_t e = cudaFuncSetAttribute(mlp_gemm_tc_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    // long reductions (the weight gradients, K = batch) are split over up to
    // eight CTAs of at least two chunks each, which add their parts atomically
    int split = 1;
    if (a.epi == kStore || a.epi == kStoreT) split = std::max(1, std::min(8, a.K / (2 * kKC)));
    if (split > 1 && !a.accumulate) {
        // the parts add into zero
        const size_t w = (size_t)(a.epi == kStore ? a.N : a.M) * sizeof(float);
        const size_t h = (size_t)(a.epi == kStore ? a.M : a.N);
        e = cudaMemset2DAsync(a.C, (size_t)a.ldc * sizeof(float), 0, w, h, s);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((unsigned)(a.M / kTM), (unsigned)(a.N / NT), (unsigned)split);
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
