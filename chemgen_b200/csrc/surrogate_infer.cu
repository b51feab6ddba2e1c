// Fused inference of the wdot surrogate on the 5th-generation tensor cores:
// features -> 4 MLP layers -> decoded FP64 wdot in one kernel, activations
// never leaving the SM.
//
// One persistent CTA of 384 threads per SM works through tiles of 128 points,
// in two warp groups that run one tile apart:
// * feature group (warps 8-11, one thread per point): the next tile's 64
//   network inputs (1000/T, ln T, ln P/1 atm, ln X_k, zeros), centred and
//   scaled, split into BF16 hi + lo parts, written into their own
//   shared-memory A operand [128 x 128] (K-major canonical layout); then 128
//   arrivals on the "features full" mbarrier.  It writes tile j+1 only after
//   the first layer of tile j has consumed tile j ("features empty");
// * compute group (warps 0-7): per layer one thread issues K/16 tcgen05.mma
//   (M = 128, N = 256 or 64, K = 16, BF16 in, FP32 accumulate in tensor
//   memory) against the layer's weights, which a bulk asynchronous copy
//   (cp.async.bulk, no multicast) brought into shared memory while the
//   previous epilogue ran; epilogue l < 3: tcgen05.ld, bias, GELU (tanh form,
//   hardware tanh as in training), BF16, into the A operand of the next layer
//   (K = 256), in two phases of 128 columns: between them the first half of
//   the next layer's K is issued, into the other 256 tensor-memory columns,
//   so that it runs beside the second phase; epilogue l = 3:
//   w_k = (u_k + b_k) exp(c + s (L + b_L)) in FP64, stored species-major,
//   and the error estimate.  The compute group synchronises on its own named
//   barrier.
// The weights come pre-arranged in the canonical layout (chemgen_surrogate_pack),
// so every weight load is a straight 16-byte-aligned bulk copy.  Shared
// memory: 64 KB activations + 32 KB features + 128 KB weights; tensor memory:
// 512 columns (layer l accumulates in columns 256 (l % 2) ..); biases are
// read through the read-only cache.  Every mbarrier wait is bounded; a
// time-out sets the error word, and the kernel waits for every product it
// issued before freeing tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/chemgen_b200.h"
#include "umma.cuh"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kPts = 128, kCompute = 256, kThreads = kCompute + kPts;
constexpr int kDin = 64, kK1 = 2 * kDin, kHid = 256, kDout = 64;
constexpr int kW1 = kHid * kK1, kW2 = kHid * kHid, kW4 = kDout * kHid;
constexpr int kImgElems = kW1 + 2 * kW2 + kW4;
constexpr uint32_t kABytes = kPts * kHid * 2;                // hidden activations, K = 256
constexpr uint32_t kFBytes = kPts * kK1 * 2;                 // features, K = 128
constexpr uint32_t kWBytes = kHid * kHid * 2;
constexpr uint32_t kFOff = kABytes, kWOff = kFOff + kFBytes, kTailOff = kWOff + kWBytes;
constexpr uint32_t kOobOff = kTailOff + 64;                 // out-of-range flags, [tile parity][row]
constexpr size_t kSmem = (size_t)kOobOff + 2 * kPts;         // + 4 mbarriers, TMEM slot, fail words
constexpr uint32_t kCopyPiece = 16384;

__device__ int g_sur_err;

__host__ __device__ constexpr int layer_k(int l) { return l == 0 ? kK1 : kHid; }
__host__ __device__ constexpr int layer_n(int l) { return l == 3 ? kDout : kHid; }
__host__ __device__ constexpr int layer_off(int l) {
    return l == 0 ? 0 : l == 1 ? kW1 : l == 2 ? kW1 + kW2 : kW1 + 2 * kW2;
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// The network's activation exactly as in training (mlp_act.cuh: GELU in tanh
// form, 0.5 z (1 + tanh(k0 (z + k1 z^3))), the hardware tanh approximation),
// on two values with the packed FP32 instructions of sm_100 (mul/fma .f32x2):
// the same operations in the same order, so the same roundings, in half the
// issue slots; the tanh stays one MUFU operation per value.
__device__ __forceinline__ float2 gelu_fast2(float2 z) {
    const float2 k1 = make_float2(0.044715f, 0.044715f), k0 = make_float2(0.7978845608028654f, 0.7978845608028654f);
    const float2 half = make_float2(0.5f, 0.5f);
    const float2 z3 = __fmul2_rn(__fmul2_rn(k1, z), z);           // 0.044715 z z
    const float2 u = __fmul2_rn(k0, __ffma2_rn(z3, z, z));        // k0 fma(.., z, z)
    float2 t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t.x) : "f"(u.x));
    asm("tanh.approx.f32 %0, %1;" : "=f"(t.y) : "f"(u.y));
    const float2 hz = __fmul2_rn(half, z);
    return __ffma2_rn(hz, t, hz);
}

// 16 accumulators + bias -> GELU -> BF16, two 16-byte stores (8 columns each).
__device__ __forceinline__ void gelu_store16(const uint32_t* r, const float* __restrict__ b, unsigned char* dst0,
                                             unsigned char* dst1) {
    uint32_t pk[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 bb = __ldg(reinterpret_cast<const float4*>(b) + q);
        const float2 z01 = __fadd2_rn(make_float2(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1])),
                                      make_float2(bb.x, bb.y));
        const float2 z23 = __fadd2_rn(make_float2(__uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3])),
                                      make_float2(bb.z, bb.w));
        const float2 h01 = gelu_fast2(z01), h23 = gelu_fast2(z23);
        const __nv_bfloat162 p01 = __floats2bfloat162_rn(h01.x, h01.y), p23 = __floats2bfloat162_rn(h23.x, h23.y);
        pk[2 * q] = *reinterpret_cast<const uint32_t*>(&p01);
        pk[2 * q + 1] = *reinterpret_cast<const uint32_t*>(&p23);
    }
    *reinterpret_cast<uint4*>(dst0) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(dst1) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
}

__device__ __forceinline__ void issue_weights(const bf16* img, int l, unsigned char* sW, uint64_t* wbar) {
    const uint32_t bytes = (uint32_t)layer_n(l) * layer_k(l) * 2;
    um::mbar_expect_tx(wbar, bytes);
    const unsigned char* src = reinterpret_cast<const unsigned char*>(img + layer_off(l));
    for (uint32_t o = 0; o < bytes; o += kCopyPiece) um::bulk_g2s(sW + o, src + o, kCopyPiece, wbar);
}

// Feature group: the 64 inputs of point `row` of `tile`, as BF16 hi/lo parts
// into sF (K = 128 canonical layout).  All loads use clamped (valid) indices
// so that they are in flight together; absent points and padding give 0.
// Returns whether the point lies outside the training support given by
// `range` (T in [range[0], range[1]], P in [range[2], range[3]], every Y_k
// >= 0 and |sum Y - 1| < 1e-6; NaN fails); no range, no check.
__device__ __forceinline__ bool write_features(unsigned char* sF, int row, int64_t tile, int64_t ng, int ns,
                                               const double* __restrict__ P, const double* __restrict__ T,
                                               const double* __restrict__ Y, const double* __restrict__ inv_mw,
                                               const float* nrm, const double* __restrict__ range) {
    const int64_t i = tile * kPts + row;
    const bool act = i < ng;
    const int64_t ic = act ? i : ng - 1;
    float y[kDin - 3];
    double ysum = 0.0, ymin = 0.0;
#pragma unroll
    for (int k = 0; k < kDin - 3; ++k) {
        const double yd = __ldg(Y + (int64_t)min(k, ns - 1) * ng + ic);
        y[k] = (float)yd;
        if (k < ns) {
            ysum += yd;
            ymin = fmin(ymin, yd);
        }
    }
    const double t = __ldg(T + ic), pr = __ldg(P + ic);
    bool oob = false;
    if (range && act)
        oob = !(t >= __ldg(range) && t <= __ldg(range + 1) && pr >= __ldg(range + 2) && pr <= __ldg(range + 3) &&
                ymin >= 0.0 && fabs(ysum - 1.0) < 1e-6);
    const float invT = (float)(1000.0 / t), lnT = logf((float)t), lnP = logf((float)(pr / 1013250.0));
    float mix = 0.0f;
#pragma unroll
    for (int k = 0; k < kDin - 3; ++k)
        if (k < ns) mix = fmaf(fmaxf(y[k], 0.0f), (float)__ldg(inv_mw + k), mix);
    const float lmix = __logf(fmaxf(mix, 1e-37f));
#pragma unroll
    for (int g = 0; g < kDin / 8; ++g) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int u = 0; u < 8; u += 2) {
            float f[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int j = 8 * g + u + e, k = j - 3;
                float v = 0.0f;
                if (act) {
                    if (j == 0) {
                        v = (invT - nrm[0]) * nrm[1];
                    } else if (j == 1) {
                        v = (lnT - nrm[2]) * nrm[3];
                    } else if (j == 2) {
                        v = (lnP - nrm[4]) * nrm[5];
                    } else if (k < ns) {
                        // fast log: ~1e-5 absolute, below the ~2^-16 of the split inputs
                        const float lx = __logf(fmaxf(y[k], 1e-30f) * (float)__ldg(inv_mw + k)) - lmix;
                        v = fminf(fmaxf((lx - nrm[6]) * nrm[7], -6.0f), 6.0f);
                    }
                }
                f[e] = v;
            }
            const bf16 h0 = __float2bfloat16(f[0]), h1 = __float2bfloat16(f[1]);
            hi[u / 2] = pack2(h0, h1);
            lo[u / 2] = pack2(__float2bfloat16(f[0] - __bfloat162float(h0)),
                              __float2bfloat16(f[1] - __bfloat162float(h1)));
        }
        *reinterpret_cast<uint4*>(sF + um::kmajor_offset(row, 8 * g, kK1)) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(sF + um::kmajor_offset(row, kDin + 8 * g, kK1)) =
            make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
    return oob;
}

__global__ void __launch_bounds__(kThreads, 1)
    surrogate_infer_kernel(const bf16* __restrict__ img, const float* __restrict__ bias,
                           const float* __restrict__ norm, const float* __restrict__ lnorm,
                           const double* __restrict__ inv_mw, int ns, const double* __restrict__ P,
                           const double* __restrict__ T, const double* __restrict__ Y, int64_t ng,
                           double* __restrict__ W, float* __restrict__ est, const double* __restrict__ range) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* sA = sm;
    unsigned char* sF = sm + kFOff;
    unsigned char* sW = sm + kWOff;
    // [0] MMAs done, [1] weights landed, [2] features full (128 arrivals), [3] features empty,
    // [4] every product issued has completed (before tensor memory is freed)
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kTailOff);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 5);
    volatile int* wfail = reinterpret_cast<volatile int*>(tslot + 1);   // set by thread 0 before a barrier
    volatile int* mfail = wfail + 1;                                     // set after the MMA wait
    volatile int* ffail = wfail + 2;                                     // feature group gave up
    // out-of-range flag of each row, one slot per tile parity: the feature
    // group writes tile j's before "features full" of tile j and tile j+2's
    // only after "features empty" of tile j+1, which the compute group
    // signals after the decode of tile j has read them
    unsigned char* sOob = sm + kOobOff;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t ntiles = (ng + kPts - 1) / kPts;
    if (tid == 0) {
        um::mbar_init(&bars[0], 1);
        um::mbar_init(&bars[1], 1);
        um::mbar_init(&bars[2], kPts);
        um::mbar_init(&bars[3], 1);
        um::mbar_init(&bars[4], 1);
        *wfail = 0;
        *mfail = 0;
        *ffail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) um::tmem_alloc(tslot, 512);
    um::fence_before_sync();
    __syncthreads();
    um::fence_after_sync();
    const uint32_t tbase = *tslot;
    float nrm[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) nrm[q] = __ldg(norm + q);
    bool failed = false, w_pending = false;
    uint32_t mpar = 0, wpar = 0;

    if (tid >= kCompute) {
        // ------------------------------------------------------ feature group
        const int row = tid - kCompute;
        int j = 0;
        for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++j) {
            if (j > 0 && !um::mbar_wait(&bars[3], (uint32_t)((j - 1) & 1))) {
                *ffail = 1;
                break;
            }
            if (*wfail || *mfail) break;
            // the inputs of the tile after this one start moving into L2
            if (warp == kThreads / 32 - 1 && tile + gridDim.x < ntiles) {
                const int64_t n0 = (tile + gridDim.x) * kPts;
                const uint32_t bytes = (uint32_t)(min((int64_t)kPts, ng - n0) * 8) & ~15u;
                for (int r = lane; r < ns + 2 && bytes; r += 32) {
                    const double* src = r < ns ? Y + (int64_t)r * ng + n0 : (r == ns ? T + n0 : P + n0);
                    if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) um::bulk_prefetch_l2(src, bytes);
                }
            }
            sOob[(j & 1) * kPts + row] = write_features(sF, row, tile, ng, ns, P, T, Y, inv_mw, nrm, range);
            um::fence_proxy_async();
            um::mbar_arrive(&bars[2]);
        }
    } else {
        // ------------------------------------------------------ compute group
        const int g4 = warp & 3, ehalf = warp >> 2;   // TMEM lane group, column half
        const int erow = 32 * g4 + lane;
        const double lc = (double)__ldg(lnorm), ls = (double)__ldg(lnorm + 1);
        if (tid == 0) {
            issue_weights(img, 0, sW, &bars[1]);
            w_pending = true;
        }
        // Layer l accumulates in tensor-memory columns 256 (l % 2) .. + 255, so
        // that the next layer's product can start before this layer's
        // epilogue has read all of its accumulators: the epilogue of a hidden
        // layer runs in two phases (columns 0-127, then 128-255), and between
        // them thread 0 issues the first half of the next layer's K (which
        // reads only activation columns 0-127); the second half follows the
        // epilogue.
        bool half_issued = false;     // thread 0: first K half of the next layer issued
        int j = 0;
        for (int64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x, ++j) {
            for (int l = 0; l < 4; ++l) {
                const int K = layer_k(l), N = layer_n(l);
                const uint32_t tacc = tbase + 256u * (uint32_t)(l & 1);
                if (tid == 0) {
                    const uint32_t idesc = um::idesc_bf16(kPts, N);
                    if (l == 0) {
                        const bool okw = um::mbar_wait(&bars[1], wpar);
                        if (okw) {
                            wpar ^= 1u;
                            w_pending = false;
                        }
                        if (okw && um::mbar_wait(&bars[2], (uint32_t)(j & 1))) {
                            um::fence_after_sync();
                            const uint32_t a = um::smem_addr(sF), b = um::smem_addr(sW);
                            for (int ks = 0; ks < K / 16; ++ks)
                                um::mma_bf16(tacc, um::desc_kmajor(a, K, ks), um::desc_kmajor(b, K, ks), idesc,
                                             ks > 0 ? 1u : 0u);
                            um::commit(&bars[0]);
                        } else {
                            *wfail = 1;
                        }
                    } else if (half_issued) {
                        // the second half of K: activation columns 128-255
                        um::fence_after_sync();
                        const uint32_t a = um::smem_addr(sA), b = um::smem_addr(sW);
                        for (int ks = K / 32; ks < K / 16; ++ks)
                            um::mma_bf16(tacc, um::desc_kmajor(a, K, ks), um::desc_kmajor(b, K, ks), idesc, 1u);
                        um::commit(&bars[0]);
                        half_issued = false;
                    } else {
                        *wfail = 1;
                    }
                }
                um::bar_sync(1, kCompute);
                if (*wfail) {
                    failed = true;
                    break;
                }
                const bool ok = um::mbar_wait(&bars[0], mpar);
                if (!ok) {
                    *mfail = 1;
                } else {
                    mpar ^= 1u;
                }
                um::fence_after_sync();
                if (ok) {
                    // the first layer has read the features: the feature group
                    // may write the next tile's
                    if (l == 0 && tid == 0) um::mbar_arrive(&bars[3]);
                    // the weights of the next layer (or of the next tile's first
                    // layer) stream in while this epilogue runs
                    if (tid == 0 && (l < 3 || tile + gridDim.x < ntiles)) {
                        issue_weights(img, l < 3 ? l + 1 : 0, sW, &bars[1]);
                        w_pending = true;
                    }
                    if (l < 3) {
                        const float* bl = bias + kHid * l;
#pragma unroll 1
                        for (int ph = 0; ph < 2; ++ph) {
                            const int c = 128 * ph + 64 * ehalf;
                            uint32_t r[64];
                            um::tmem_ld64(um::tmem_lane_addr(tacc, g4, c), r);
#pragma unroll
                            for (int q = 0; q < 4; ++q)
                                gelu_store16(r + 16 * q, bl + c + 16 * q, sA + um::kmajor_offset(erow, c + 16 * q, kHid),
                                             sA + um::kmajor_offset(erow, c + 16 * q + 8, kHid));
                            if (ph == 0) {
                                // activation columns 0-127 are written: the next
                                // layer's first K half can run beside phase 1
                                um::fence_proxy_async();
                                um::fence_before_sync();
                                um::bar_sync(1, kCompute);
                                if (tid == 0) {
                                    const bool okw = um::mbar_wait(&bars[1], wpar);
                                    if (okw) {
                                        wpar ^= 1u;
                                        w_pending = false;
                                        um::fence_after_sync();
                                        const int K2 = layer_k(l + 1);
                                        const uint32_t idesc2 = um::idesc_bf16(kPts, layer_n(l + 1));
                                        const uint32_t a = um::smem_addr(sA), b = um::smem_addr(sW);
                                        const uint32_t t2 = tbase + 256u * (uint32_t)((l + 1) & 1);
                                        for (int ks = 0; ks < K2 / 32; ++ks)
                                            um::mma_bf16(t2, um::desc_kmajor(a, K2, ks), um::desc_kmajor(b, K2, ks),
                                                         idesc2, ks > 0 ? 1u : 0u);
                                        half_issued = true;
                                    }
                                }
                            }
                        }
                    } else {
                        const float* b4 = bias + 3 * kHid;
                        const int64_t i = tile * kPts + erow;
                        const bool act = i < ng;
                        const bool oob = sOob[(j & 1) * kPts + erow] != 0;
                        const int cL = (ns / 16) * 16;
                        float v[16];
                        um::tmem_ld16(um::tmem_lane_addr(tacc, g4, cL), v);
                        float L = 0.0f;
#pragma unroll
                        for (int q = 0; q < 16; ++q)
                            if (cL + q == ns) L = v[q];
                        const double scale = exp(lc + ls * (double)(L + __ldg(b4 + ns)));
#pragma unroll 1
                        for (int c = 32 * ehalf; c < 32 * ehalf + 32; c += 16) {
                            um::tmem_ld16(um::tmem_lane_addr(tacc, g4, c), v);
                            if (act) {
#pragma unroll
                                for (int q = 0; q < 16; ++q) {
                                    const int k = c + q;
                                    if (k < ns) W[(int64_t)k * ng + i] = (double)(v[q] + __ldg(b4 + k)) * scale;
                                    else if (k == ns + 1 && est) est[i] = oob ? INFINITY : v[q] + __ldg(b4 + k);
                                }
                            }
                        }
                    }
                } else if (l < 3) {
                    um::bar_sync(1, kCompute);     // the mid-epilogue barrier the others reach
                }
                um::fence_proxy_async();
                um::fence_before_sync();
                um::bar_sync(1, kCompute);
                um::fence_after_sync();
                if (*mfail) {
                    failed = true;
                    break;
                }
            }
            if (*ffail) failed = true;
        }
        if (failed && tid == 0) {
            // drain the weight copy this group issued (bounded)
            atomicExch(&g_sur_err, 1);
            if (w_pending) um::mbar_wait(&bars[1], wpar);
        }
        // every product issued (committed or not) completes before tensor
        // memory is freed
        if (tid == 0) {
            um::commit(&bars[4]);
            um::mbar_wait(&bars[4], 0);
        }
    }
    if (tid >= kCompute && *ffail && tid == kCompute) atomicExch(&g_sur_err, 1);
    um::fence_before_sync();
    __syncthreads();
    if (warp == 0) um::tmem_dealloc(tbase, 512);
}

// Weight image: layer l's [N_l x K_l] BF16 operand in the K-major canonical
// layout (element (n, k) at (n/8) K 8 + (k/8) 64 + (n%8) 8 + k%8), layers
// back to back; layer 0's K = 128 holds the 64 input weights twice (for the
// hi and lo parts of the inputs).
__global__ void pack_kernel(const bf16* __restrict__ W1, const bf16* __restrict__ W2, const bf16* __restrict__ W3,
                            const bf16* __restrict__ W4, bf16* __restrict__ img) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= kImgElems) return;
    const int l = d < layer_off(1) ? 0 : d < layer_off(2) ? 1 : d < layer_off(3) ? 2 : 3;
    const int K = layer_k(l), local = d - layer_off(l);
    const int rg = local / (K * 8), rem = local % (K * 8);
    const int kc = rem / 64, r8 = (rem % 64) / 8, k8 = rem % 8;
    const int n = rg * 8 + r8, k = kc * 8 + k8;
    bf16 v;
    if (l == 0) v = W1[n * kDin + (k % kDin)];
    else if (l == 1) v = W2[n * kHid + k];
    else if (l == 2) v = W3[n * kHid + k];
    else v = W4[n * kHid + k];
    img[d] = v;
}

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return n;
}

}  // namespace

extern "C" {

int chemgen_surrogate_image_elems(void) { return kImgElems; }

int chemgen_surrogate_pack(const void* W1, const void* W2, const void* W3, const void* W4, void* img, void* stream) {
    if (!W1 || !W2 || !W3 || !W4 || !img) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(img) & 15) return CHEMGEN_ERR_MISALIGNED;
    pack_kernel<<<(kImgElems + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        (const bf16*)W1, (const bf16*)W2, (const bf16*)W3, (const bf16*)W4, (bf16*)img);
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

int chemgen_surrogate_infer(const void* img, const float* bias, const float* norm, const float* lnorm,
                            const double* inv_mw, int ns, const double* P, const double* T, int64_t ng,
                            const double* Y, double* wdot, float* err_est, const double* range, void* stream) {
    if (!img || !bias || !norm || !lnorm || !inv_mw || !P || !T || !Y || !wdot || ng < 0)
        return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (ns < 1 || ns + 3 > kDin || ns + 2 > kDout) return CHEMGEN_ERR_UNSUPPORTED;
    if (reinterpret_cast<uintptr_t>(img) & 15) return CHEMGEN_ERR_MISALIGNED;
    if (ng == 0) return CHEMGEN_OK;
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (cudaFuncSetAttribute(surrogate_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem) !=
            cudaSuccess)
            return CHEMGEN_ERR_CUDA;
    }
    const int sms = sm_count();
    if (sms <= 0) return CHEMGEN_ERR_CUDA;
    const int64_t ntiles = (ng + kPts - 1) / kPts;
    const unsigned grid = (unsigned)(ntiles < sms ? ntiles : sms);
    surrogate_infer_kernel<<<grid, kThreads, kSmem, (cudaStream_t)stream>>>(
        (const bf16*)img, bias, norm, lnorm, inv_mw, ns, P, T, Y, ng, wdot, err_est, range);
    return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA;
}

int chemgen_surrogate_infer_error(int reset) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_sur_err, sizeof(int)) != cudaSuccess) return -1;
    if (reset && v) {
        const int z = 0;
        if (cudaMemcpyToSymbol(g_sur_err, &z, sizeof(int)) != cudaSuccess) return -1;
    }
    return v;
}

}  // extern "C"
