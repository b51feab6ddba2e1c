// Mixed-precision getrates with the stoichiometric contraction on the
// 5th-generation tensor cores (tcgen05).  Table-driven: one compiled kernel
// serves every mechanism loaded at run time, including 348-species /
// 2163-reaction ones.
//
// Work split.  A CTA owns a tile of 128 grid points -- one point per thread,
// one point per TMEM lane.  For every chunk of 16 reactions each thread
// computes its point's net rates of progress q (the reference's
// rr = kf prod C^nu - kb prod C^nu, reactions/standard.j2:3-19, with the
// third-body factor of third_body.j2:30 and the falloff of troe.j2:9-45)
// and writes them, split exactly into three BF16 parts q = q_hi + q_mid +
// q_lo, into shared memory as the A operand of an MMA whose B operand is
// the chunk's net stoichiometric matrix nu (exact in BF16).  One thread
// issues tcgen05.mma; the products accumulate in FP32 in tensor memory,
// D[point][species] = sum_r q_r nu_rk, which is wdot
// (reactions/standard.j2:21-27).  Two chunk buffers let the tensor core
// accumulate one chunk while the threads compute the next.
//
// Arithmetic.  Exponents are formed in FP64: ln A + b ln T - Ea/(Rc T) and
// the Gibbs sums sum nu G that give Kc (G = log2(exp(smh) Patm/(R0 T))).
// 2^f of the fractional part runs on the SFU (ex2.approx.f32); concentration
// products are FP32 on C * 2^32 (so that they stay clear of FP32 underflow);
// q is FP32 and the accumulation FP32.  PLOG reactions and reactions with
// fractional stoichiometry are evaluated in FP64 and rounded to FP32.
//
// Per-point state: C (FP32, shared memory) and G (FP64, shared memory, or a
// per-CTA slice of global scratch when the mechanism is too large).
// Every mbarrier wait is bounded; a time-out sets the error word.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "cg_math.cuh"
#include "gen_common.cuh"
#include "rates_common.cuh"
#include "umma.cuh"

namespace cg {

constexpr int kTile = 128;       // points per CTA tile (TMEM lanes)
constexpr int kChunk = 16;       // reactions per MMA chunk (MMA K)
constexpr int kABytes = kTile * kChunk * 2;   // one BF16 A split tile

// Pre-decoded record of a standard or three-body reaction with at most three
// molecules per side (the common case), built once per plan on the device:
// log2-space Arrhenius constants and the species of each molecule, padded with
// the dummy species ns (C = 1, G = 0), so that the rate needs no decoding.
struct __align__(16) TcFast {
    double l2A, b, th2;          // log2|A|, b, (Ea/Rc) log2 e
    unsigned short sr[3], sp[3]; // reactant / product molecules (species ns = none)
    unsigned char ordf, ordb;    // concentration factors of each side (M included)
    unsigned char flags;         // kFastOn | kFastRev | kFastThird | kFastNeg
    unsigned char pad0;
    int pad1[2];
};
static_assert(sizeof(TcFast) == 48, "TcFast must stay 48 bytes");
constexpr unsigned kFastOn = 1, kFastRev = 2, kFastThird = 4, kFastNeg = 8;

struct MixedPlan {
    int ns = 0, nr = 0, npad = 0, nhalf = 0, nchunk = 0;
    uint32_t tcols = 0;
    int g_smem = 0;
    size_t smem = 0;
    int grid = 0;
    int group = 4;          // chunks accumulated in FP32 before the FP64 flush
    int nt = 1;             // threads per point (blockDim = 128 nt)
    int hot = 0;            // species with FP64 accumulators in spare tensor-memory columns
    int hot_every = 8;      // chunks between the hot species' FP64 flushes
    const int* perm = nullptr;  // accumulator column -> species (-1: padding)
    void* dbuf = nullptr;
    const __nv_bfloat16* nu = nullptr;
    const TcFast* fast = nullptr;
    int* err = nullptr;
};

namespace {

constexpr double kLog2eD = 1.4426950408889634074;
constexpr float kLog2eF = 1.44269504f;
constexpr float kLog10_2F = 0.30103000f;

// 2^e for an integer e, applied in two FP32 steps so that large products
// with small scales (and the reverse) keep their value.
__device__ __forceinline__ float scale2(float m, int e) {
    const int e1 = max(-126, min(e, 127));
    const int e2 = max(-126, min(e - e1, 127));
    return m * __int_as_float((e1 + 127) << 23) * __int_as_float((e2 + 127) << 23);
}

// FP32 q = 2^a * prod * 2^eoff, a in FP64.
__device__ __forceinline__ float rate32(double a, float prod, int eoff) {
    const double magic = 6755399441055744.0;
    const double t = a + magic;
    const int n = __double2loint(t);
    const float f = (float)(a - (t - magic));
    return scale2(cgg::ex2f(f) * prod, n + eoff);
}

struct TileCtx {
    const float* C;      // C * 2^32, stride kTile
    const double* G;     // log2 Gibbs terms, stride kTile
    double T, Pv, lnT, lnT2, invT;
    float ctot32, Tf, invTf, lnT2f;
};

// log2 kf of a falloff reaction (Lindemann, Troe, SRI), in FP64 throughout
// (troe.j2:9-45 in the log2 domain).  The FP32 blend that the 53-species
// generated kernels use was measured on JetSurf 2.0 (382 Troe reactions,
// several of them each point's dominant rate): its kf errors reached 5e-6,
// mostly from FP32 exponent arguments in Fcent and the FP32 log10 Pr / f1 chain,
// which put the normwise error of wdot at 7.6e-6 over 2^18 points.  In FP64
// the blend costs about three exp and three log per falloff reaction.
__device__ double falloff_l2(int kind, int flags, const DRxn& R, const DFall& f, double x2, float Ms,
                             const TileCtx& c) {
    constexpr double kLog10_2 = 0.30102999566398119521, kLn2 = 0.69314718055994530942;
    const double ainf = (fma(R.b, c.lnT, R.lnA) - R.theta * c.invT) * kLog2eD;
    const double a0 = (fma(f.b0, c.lnT, f.lnA0) - f.theta0 * c.invT) * kLog2eD;
    const double M = (double)Ms * 2.3283064365386963e-10;   // Ms = M * 2^32
    // log2 Pr and log2 Pr/(1 + Pr), without overflow at either end
    const double l2pr = (a0 - ainf) + cgm::cg_log(M) * kLog2eD;
    const double x = cgm::cg_exp_clamped(-fabs(l2pr) * kLn2);          // min(Pr, 1/Pr)
    const double l2r = fmin(l2pr, 0.0) - cgm::cg_log(1.0 + x) * kLog2eD;
    double l2F = 0.0;
    if (kind == CG_TROE) {
        double Fc = fma(f.p[0], cgm::cg_exp_clamped(-c.T * f.p[1]), f.p[2] * cgm::cg_exp_clamped(-c.T * f.p[3]));
        if (flags & CG_F_TROE_T2) Fc += cgm::cg_exp_clamped(-x2 * c.invT);
        const double lFc = cgm::cg_log10(Fc);
        const double lp = fma(kLog10_2, l2pr, fma(-0.67, lFc, -0.4));
        const double f1 = lp * cgm::cg_rcp(fma(-0.14, lp, fma(-1.27, lFc, 0.75)));
        l2F = lFc * cgm::cg_rcp(fma(f1, f1, 1.0)) / kLog10_2;
    } else if (kind == CG_SRI) {
        const double lp = kLog10_2 * l2pr;
        const double X = cgm::cg_rcp(fma(lp, lp, 1.0));
        const double base = fma(f.p[0], cgm::cg_exp_clamped(-f.p[1] * c.invT), cgm::cg_exp_clamped(-c.T * f.p[2]));
        l2F = (cgm::cg_log(f.p[3]) + fma(X, cgm::cg_log(base), x2 * c.lnT)) * kLog2eD;
    }
    return ainf + (l2r + l2F);
}

// PLOG forward rate in FP64 (plog.j2:4-38).
__device__ double plog_kf64(const DevMech& m, int row, double P, double lnT, double invT) {
    const int l0 = __ldg(m.plog_ptr + row), l1 = __ldg(m.plog_ptr + row + 1);
    int l = l0;
    while (l < l1 && !(P < __ldg(m.plog_p + l))) ++l;
    int la, lb;
    if (l == l0) la = lb = l0;
    else if (l == l1) la = lb = l1 - 1;
    else {
        la = l - 1;
        lb = l;
    }
    double k[2] = {0.0, 0.0};
    const int lev[2] = {la, lb};
    for (int s = 0; s < (la == lb ? 1 : 2); ++s)
        for (int t = __ldg(m.plog_tptr + lev[s]); t < __ldg(m.plog_tptr + lev[s] + 1); ++t) {
            const double4 cc = m.plog_term[t];
            k[s] += cc.w * cgm::cg_exp_clamped(fma(cc.y, lnT, cc.x) - cc.z * invT);
        }
    if (la == lb) return k[0];
    const double a = __ldg(m.plog_lnp + la), b = __ldg(m.plog_lnp + lb);
    const double kl = cgm::cg_log(k[0]);
    return cgm::cg_exp_clamped(kl + (cgm::cg_log(k[1]) - kl) * (cgm::cg_log(P) - a) / (b - a));
}

// FP64 evaluation of reaction r (PLOG, non-integer stoichiometry, falloff
// with negative pre-exponential factors): kept out of line so that the
// common FP32 path keeps few registers.
__device__ __noinline__ float rate_of_progress_fp64(const DevMech& m, const DRxn& R, int kind, float Ms,
                                                    const TileCtx& c, int tid) {
    const bool compact = (R.flags & kFCompact) != 0;
    {
        double kf;
        if (kind == CG_PLOG) kf = plog_kf64(m, R.aux, c.Pv, c.lnT, c.invT);
        else if (kind <= CG_THIRD_BODY) kf = R.sgn * cgm::cg_exp_clamped(fma(R.b, c.lnT, R.lnA) - R.theta * c.invT);
        else {
            const DFall f = load_fall(m.fall + R.aux);
            kf = R.sgn * exp2(falloff_l2(kind, R.flags, R, f, __ldg(&m.fall2[R.aux].T2), Ms, c));
        }
        const double cs = 2.3283064365386963e-10;   // 2^-32
        double qf = kf, qb = 0.0, g = 0.0;
        {
            if (compact) {
                for (int j = 0; j < R.nre; ++j) {
                    const int s = slot_species(R.sp[j]);
                    qf *= ipow3((double)c.C[s * kTile + tid] * cs, slot_nu(R.sp[j]));
                    g = fma((double)slot_nu(R.sp[j]), c.G[s * kTile + tid], g);
                }
                double pb = 1.0;
                for (int j = 0; j < R.npr; ++j) {
                    const int s = slot_species(R.sp[3 + j]);
                    pb *= ipow3((double)c.C[s * kTile + tid] * cs, slot_nu(R.sp[3 + j]));
                    g = fma(-(double)slot_nu(R.sp[3 + j]), c.G[s * kTile + tid], g);
                }
                if (R.flags & CG_F_REVERSIBLE) qb = kf * exp2(g) * pb;
            } else {
                const int gr = R.gen;
                const int r0 = __ldg(m.gen_rptr + gr), r1 = __ldg(m.gen_rptr + gr + 1);
                const int p0 = __ldg(m.gen_pptr + gr), p1 = __ldg(m.gen_pptr + gr + 1);
                for (int j = r0; j < r1; ++j) {
                    const int s = __ldg(m.gen_sp + j);
                    const double nu = __ldg(m.gen_nu + j);
                    qf *= pow((double)c.C[s * kTile + tid] * cs, nu);
                    g = fma(nu, c.G[s * kTile + tid], g);
                }
                double pb = 1.0;
                for (int j = p0; j < p1; ++j) {
                    const int s = __ldg(m.gen_sp + j);
                    const double nu = __ldg(m.gen_nu + j);
                    pb *= pow((double)c.C[s * kTile + tid] * cs, nu);
                    g = fma(-nu, c.G[s * kTile + tid], g);
                }
                if (R.flags & CG_F_REVERSIBLE) qb = kf * exp2(g) * pb;
            }
        }
        double rr = qf - qb;
        if (kind == CG_THIRD_BODY) rr *= (double)Ms * cs;
        return (float)rr;
    }
}

// Ms = ctot + sum_e (eff_e - 1) C[sp_e] of reaction r (third_body.j2:18-31) in
// FP32 at point `tid`, the efficiencies taken four at a time so that their
// loads are in flight together; the sum keeps the table's order.
__device__ __forceinline__ float tc_third_body(const DevMech& m, int r, const TileCtx& c, int tid) {
    float Ms = c.ctot32;
    const int e1 = __ldg(m.eff_ptr + r + 1);
    for (int e = __ldg(m.eff_ptr + r); e < e1; e += 4) {
        int sp[4];
        float ev[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool ok = e + u < e1;
            sp[u] = ok ? __ldg(m.eff_sp + e + u) : 0;
            ev[u] = ok ? (float)__ldg(m.eff_val + e + u) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float cv = c.C[sp[u] * kTile + tid];
            if (e + u < e1) Ms = fmaf(ev[u], cv, Ms);
        }
    }
    return Ms;
}

// Net rate of progress of reaction r at point `tid` of the tile, FP32.
__device__ float rate_of_progress(const DevMech& m, int r, const TileCtx& c, int tid) {
    const DRxn R = load_rxn(m.rxn + r);
    int kind = CG_STANDARD;
    while (kind < CG_PLOG && r >= m.seg[kind + 1]) ++kind;
    float Ms = 0.0f;
    if (kind >= CG_THIRD_BODY && kind <= CG_SRI) Ms = tc_third_body(m, r, c, tid);
    const bool compact = (R.flags & kFCompact) != 0;
    const bool neg_falloff = kind >= CG_LINDEMANN && kind <= CG_SRI && (R.flags & (CG_F_A_NEG | CG_F_LOW_NEG));
    if (!compact || kind == CG_PLOG || neg_falloff) return rate_of_progress_fp64(m, R, kind, Ms, c, tid);
    double a;
    float sgn = 1.0f;
    if (kind <= CG_THIRD_BODY) {
        a = (fma(R.b, c.lnT, R.lnA) - R.theta * c.invT) * kLog2eD;
        sgn = (float)R.sgn;
    } else {
        const DFall f = load_fall(m.fall + R.aux);
        a = falloff_l2(kind, R.flags, R, f, __ldg(&m.fall2[R.aux].T2), Ms, c);
    }
    float cf = 1.0f;
    int of = 0;
    double g = 0.0;
    for (int j = 0; j < R.nre; ++j) {
        const int s = slot_species(R.sp[j]), nu = slot_nu(R.sp[j]);
        const float x = c.C[s * kTile + tid];
        cf *= (nu == 1) ? x : (nu == 2 ? x * x : x * x * x);
        of += nu;
        g = fma((double)nu, c.G[s * kTile + tid], g);
    }
    if (kind == CG_THIRD_BODY) {
        cf *= Ms;
        of += 1;
    }
    float q = rate32(a, cf, -32 * of);
    if (R.flags & CG_F_REVERSIBLE) {
        float cb = 1.0f;
        int ob = 0;
        for (int j = 0; j < R.npr; ++j) {
            const int s = slot_species(R.sp[3 + j]), nu = slot_nu(R.sp[3 + j]);
            const float x = c.C[s * kTile + tid];
            cb *= (nu == 1) ? x : (nu == 2 ? x * x : x * x * x);
            ob += nu;
            g = fma(-(double)nu, c.G[s * kTile + tid], g);
        }
        if (kind == CG_THIRD_BODY) {
            cb *= Ms;
            ob += 1;
        }
        q -= rate32(a + g, cb, -32 * ob);
    }
    return sgn * q;
}

// Net rate of progress of a pre-decoded reaction (TcFast) at point `tid`, FP32.
__device__ __forceinline__ float rate_fast(const DevMech& m, int r, const TcFast& F, const TileCtx& c, int tid) {
    const double a = fma(F.b, c.lnT2, F.l2A) - F.th2 * c.invT;
    float Ms = 1.0f;
    if (F.flags & kFastThird) Ms = tc_third_body(m, r, c, tid);
    const float cf = c.C[F.sr[0] * kTile + tid] * c.C[F.sr[1] * kTile + tid] * c.C[F.sr[2] * kTile + tid] * Ms;
    float q = rate32(a, cf, -32 * (int)F.ordf);
    if (F.flags & kFastRev) {
        const double g = (c.G[F.sr[0] * kTile + tid] + c.G[F.sr[1] * kTile + tid] + c.G[F.sr[2] * kTile + tid]) -
                         (c.G[F.sp[0] * kTile + tid] + c.G[F.sp[1] * kTile + tid] + c.G[F.sp[2] * kTile + tid]);
        const float cb = c.C[F.sp[0] * kTile + tid] * c.C[F.sp[1] * kTile + tid] * c.C[F.sp[2] * kTile + tid] * Ms;
        q -= rate32(a + g, cb, -32 * (int)F.ordb);
    }
    return (F.flags & kFastNeg) ? -q : q;
}

__device__ __forceinline__ TcFast load_fast(const TcFast* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    TcFast f;
    int4* d = reinterpret_cast<int4*>(&f);
    d[0] = __ldg(q);
    d[1] = __ldg(q + 1);
    d[2] = __ldg(q + 2);
    return f;
}

// One TcFast per reaction (flags 0 where the generic path is needed).
__global__ void build_fast_kernel(DevMech m, TcFast* out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m.nr) return;
    const DRxn R = load_rxn(m.rxn + r);
    int kind = CG_STANDARD;
    while (kind < CG_PLOG && r >= m.seg[kind + 1]) ++kind;
    TcFast f;
    f.l2A = R.lnA * kLog2eD;
    f.b = R.b;
    f.th2 = R.theta * kLog2eD;
    f.pad0 = 0;
    f.pad1[0] = f.pad1[1] = 0;
    f.flags = 0;
    f.ordf = f.ordb = 0;
    for (int j = 0; j < 3; ++j) f.sr[j] = f.sp[j] = (unsigned short)m.ns;
    bool ok = (kind == CG_STANDARD || kind == CG_THIRD_BODY) && (R.flags & kFCompact) && R.sgn != 0.0;
    int nf = 0, nb = 0;
    for (int j = 0; ok && j < R.nre; ++j)
        for (int k = 0; k < slot_nu(R.sp[j]); ++k) {
            if (nf == 3) ok = false;
            else f.sr[nf++] = (unsigned short)slot_species(R.sp[j]);
        }
    for (int j = 0; ok && j < R.npr; ++j)
        for (int k = 0; k < slot_nu(R.sp[3 + j]); ++k) {
            if (nb == 3) ok = false;
            else f.sp[nb++] = (unsigned short)slot_species(R.sp[3 + j]);
        }
    if (ok) {
        const bool third = kind == CG_THIRD_BODY;
        f.ordf = (unsigned char)(nf + (third ? 1 : 0));
        f.ordb = (unsigned char)(nb + (third ? 1 : 0));
        f.flags = (unsigned char)(kFastOn | ((R.flags & CG_F_REVERSIBLE) ? kFastRev : 0) | (third ? kFastThird : 0) |
                                  (R.sgn < 0.0 ? kFastNeg : 0));
    }
    out[r] = f;
}

// NT threads share each of the tile's 128 points (blockDim = 128 NT): they
// split the species of the prologue (their partial sums meet in shared
// memory), the 16 reactions of each chunk, and the accumulator columns of
// each flush.  The FP32 sums live in tensor memory, so extra threads cost
// no per-species registers.
template <bool GS, int NT>
__global__ void __launch_bounds__(kTile * NT, 1)
    getrates_tc_kernel(DevMech m, const __nv_bfloat16* __restrict__ nu, const TcFast* __restrict__ fast, int npad,
                       int nhalf, int nchunk, uint32_t tcols,
                       const double* __restrict__ P, const double* __restrict__ Tg, const double* __restrict__ Y,
                       double* __restrict__ wdot, int64_t ng, double* __restrict__ gscratch, int* err, int group,
                       const int* __restrict__ perm, int hot, int hot_every) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int pt = tid & (kTile - 1), sub = tid >> 7;          // point of the tile, share of its work
    const int ns = m.ns;
    unsigned char* sA = sm;                                    // [2 buffers][3 splits][128 x 16] BF16
    unsigned char* sB = sm + 6 * kABytes;                      // [2 buffers][npad x 16] BF16
    const int rows = ns + 1;                                   // species + the dummy row of TcFast
    float* sC = reinterpret_cast<float*>(sB + 2 * npad * 32);  // [rows][128]
    double* sG = GS ? reinterpret_cast<double*>(sC + rows * kTile) : gscratch + (int64_t)blockIdx.x * rows * kTile;
    double* sRed = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(sC) + rows * kTile * 4 +
                                             (GS ? rows * kTile * 8 : 0));   // [NT][128] partial sums
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sRed + NT * kTile);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);
    if (tid == 0) {
        um::mbar_init(&mbar[0], 1);
        um::mbar_init(&mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) um::tmem_alloc(tslot, tcols);
    um::fence_before_sync();
    __syncthreads();
    um::fence_after_sync();
    const uint32_t tbase = *tslot;
    uint32_t parity[2] = {0u, 0u};
    bool pending[2] = {false, false};
    bool ok = true;
    const uint32_t idesc = um::idesc_bf16(kTile, nhalf);
    const int nh = npad / nhalf;
    const int64_t ntiles = (ng + kTile - 1) / kTile;
    for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int64_t i = tile * kTile + pt;
        const bool act = i < ng;
        TileCtx c;
        c.C = sC;
        c.G = sG;
        // inputs are read once: streaming loads, so that they do not push the
        // Gibbs scratch and the stoichiometry image out of L2
        c.T = act ? __ldcs(Tg + i) : 1000.0;
        c.Pv = act ? __ldcs(P + i) : kPatm;
        c.lnT = cgm::cg_log(c.T);
        c.invT = 1.0 / c.T;
        c.lnT2 = c.lnT * kLog2eD;
        c.Tf = (float)c.T;
        c.invTf = (float)c.invT;
        c.lnT2f = (float)c.lnT2;
        // Y -> C (ytoc.j2), stored as C * 2^32 in FP32; species k is handled
        // by the thread with sub = k % NT
        double part = 0.0;
        for (int k = sub; k < ns; k += NT) {
            const double yk = (act ? __ldcs(Y + (int64_t)k * ng + i) : 1.0) * __ldg(m.inv_mw + k);
            sG[k * kTile + pt] = yk;
            part += yk;
        }
        sRed[sub * kTile + pt] = part;
        __syncthreads();
        double csum = 0.0;
        for (int q = 0; q < NT; ++q) csum += sRed[q * kTile + pt];
        const double facs = c.Pv / (kR0 * csum * c.T) * 4294967296.0;
        part = 0.0;
        for (int k = sub; k < ns; k += NT) {
            const double cc = sG[k * kTile + pt] * facs;
            sC[k * kTile + pt] = (float)cc;
            part += cc;
        }
        __syncthreads();
        sRed[sub * kTile + pt] = part;
        __syncthreads();
        double ctot = 0.0;
        for (int q = 0; q < NT; ++q) ctot += sRed[q * kTile + pt];
        c.ctot32 = (float)ctot;
        // G = log2(exp(smh) Patm/(R0 T)) (exp_g.j2), FP64
        const double lpfac2 = -6.35856916300311 - c.lnT2;   // log2(Patm/R0) - log2 T
        for (int k = sub; k < ns; k += NT)
            sG[k * kTile + pt] = fma(species_smh(m.thermo, k, c.T, c.lnT, c.invT), kLog2eD, lpfac2);
        if (sub == 0) {
            sC[ns * kTile + pt] = 1.0f;     // dummy species of TcFast: a factor 1 ...
            sG[ns * kTile + pt] = 0.0;      // ... and no Gibbs term
        }
        __syncthreads();
        bool first_group = true;
        int nhot = 0;                    // hot flushes so far in this tile
        for (int ch = 0; ch < nchunk && ok; ++ch) {
            const int buf = ch & 1;
            if (pending[buf]) {
                ok = um::mbar_wait(&mbar[buf], parity[buf]);
                parity[buf] ^= 1u;
                pending[buf] = false;
                if (!ok) break;
            }
            // the chunk's stoichiometry, B operand [npad x 16], canonical layout
            const uint4* src = reinterpret_cast<const uint4*>(nu + (int64_t)ch * npad * kChunk);
            uint4* dst = reinterpret_cast<uint4*>(sB + buf * npad * 32);
            for (int q = tid; q < npad * 2; q += kTile * NT) dst[q] = __ldg(src + q);
            // q for the chunk's reactions -> A operands (hi, mid, lo).  The
            // thread with share `sub` takes kPer consecutive reactions, so that
            // its BF16 values of a row leave in one 8- or 16-byte store per
            // split instead of one 2-byte store per reaction
            unsigned char* a0 = sA + buf * 3 * kABytes;
            constexpr int kPer = kChunk / NT, kWords = kPer / 4;
            static_assert(kChunk % NT == 0 && kPer % 4 == 0, "each share takes whole 4-reaction words");
            const int j0 = sub * kPer;
            uint64_t ph[kWords], pm[kWords], pl[kWords];
#pragma unroll
            for (int w = 0; w < kWords; ++w) ph[w] = pm[w] = pl[w] = 0ull;
#pragma unroll 1
            for (int u = 0; u < kPer; ++u) {
                const int r = ch * kChunk + j0 + u;
                float q = 0.0f;
                if (r < m.nr) {
                    const TcFast F = load_fast(fast + r);
                    // this thread's next record moves into L1 meanwhile (no registers held)
                    if (u + 1 < kPer && r + 1 < m.nr) asm volatile("prefetch.global.L1 [%0];" ::"l"(fast + r + 1));
                    q = (F.flags & kFastOn) ? rate_fast(m, r, F, c, pt) : rate_of_progress(m, r, c, pt);
                }
                if (!act) q = 0.0f;
                const __nv_bfloat16 h = __float2bfloat16_rn(q);
                const float r1 = q - __bfloat162float(h);
                const __nv_bfloat16 md = __float2bfloat16_rn(r1);
                const __nv_bfloat16 lo = __float2bfloat16_rn(r1 - __bfloat162float(md));
                const int sh = 16 * (u & 3);
#pragma unroll
                for (int w = 0; w < kWords; ++w)
                    if (w == (u >> 2)) {
                        ph[w] |= (uint64_t)__bfloat16_as_ushort(h) << sh;
                        pm[w] |= (uint64_t)__bfloat16_as_ushort(md) << sh;
                        pl[w] |= (uint64_t)__bfloat16_as_ushort(lo) << sh;
                    }
            }
#pragma unroll
            for (int w = 0; w < kWords; ++w) {
                const uint32_t off = um::kmajor_offset(pt, j0 + 4 * w, kChunk);   // 8-byte aligned
                *reinterpret_cast<uint64_t*>(a0 + off) = ph[w];
                *reinterpret_cast<uint64_t*>(a0 + kABytes + off) = pm[w];
                *reinterpret_cast<uint64_t*>(a0 + 2 * kABytes + off) = pl[w];
            }
            um::fence_proxy_async();
            um::fence_before_sync();
            __syncthreads();
            const bool group_start = (ch % group) == 0;
            if (tid == 0) {
                um::fence_after_sync();
                const uint32_t bb = um::smem_addr(sB + buf * npad * 32);
                for (int s = 0; s < 3; ++s) {
                    const uint64_t ad = um::desc_kmajor(um::smem_addr(a0 + s * kABytes), kChunk, 0);
                    for (int h = 0; h < nh; ++h)
                        um::mma_bf16(tbase + (uint32_t)(h * nhalf), ad,
                                     um::desc_kmajor(bb + (uint32_t)(h * nhalf * 32), kChunk, 0), idesc,
                                     (!group_start || s > 0) ? 1u : 0u);
                }
                um::commit(&mbar[buf]);
            }
            pending[buf] = true;
            const bool group_end = (ch % group) == group - 1 || ch == nchunk - 1;
            if (hot > 0 && !group_end && (ch % hot_every) == hot_every - 1) {
                // hot flush: the FP32 sums of the most-touched species (columns
                // 0 .. hot-1) move into their FP64 accumulators (columns npad +
                // 2j, +1) and restart from zero, so that FP32 never sums more
                // than hot_every chunks of them; tensor-memory traffic only
                for (int b = 0; b < 2; ++b)
                    if (pending[b]) {
                        ok = um::mbar_wait(&mbar[b], parity[b]) && ok;
                        parity[b] ^= 1u;
                        pending[b] = false;
                    }
                um::fence_after_sync();
                if (ok) {
                    for (int blk = warp >> 2; blk < hot / 16; blk += NT) {
                        float v[16];
                        uint32_t d[32];
                        um::tmem_ld16(um::tmem_lane_addr(tbase, warp & 3, 16 * blk), v);
                        if (nhot > 0) um::tmem_ld32(um::tmem_lane_addr(tbase, warp & 3, npad + 32 * blk), d);
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const double a = (nhot > 0 ? __hiloint2double((int)d[2 * j + 1], (int)d[2 * j]) : 0.0) +
                                             (double)v[j];
                            d[2 * j] = (uint32_t)__double2loint(a);
                            d[2 * j + 1] = (uint32_t)__double2hiint(a);
                        }
                        um::tmem_st32(um::tmem_lane_addr(tbase, warp & 3, npad + 32 * blk), d);
                        uint32_t z[16];
#pragma unroll
                        for (int j = 0; j < 16; ++j) z[j] = 0u;
                        um::tmem_st16(um::tmem_lane_addr(tbase, warp & 3, 16 * blk), z);
                    }
                    um::tmem_wait_st();
                }
                ++nhot;
                um::fence_before_sync();
                __syncthreads();
            }
            if (group_end) {
                // end of a group of reactions: wait for its MMAs, then add the
                // FP32 partial sums into the FP64 output; the NT warps that
                // share a lane quadrant split the columns
                for (int b = 0; b < 2; ++b)
                    if (pending[b]) {
                        ok = um::mbar_wait(&mbar[b], parity[b]) && ok;
                        parity[b] ^= 1u;
                        pending[b] = false;
                    }
                um::fence_after_sync();
                if (ok) {
                    for (int col = 16 * (warp >> 2); col < npad; col += 16 * NT) {
                        float v[16];
                        uint32_t d[32];
                        um::tmem_ld16(um::tmem_lane_addr(tbase, warp & 3, col), v);
                        const bool h64 = col < hot && nhot > 0;
                        if (h64) um::tmem_ld32(um::tmem_lane_addr(tbase, warp & 3, npad + 2 * col), d);
                        if (act)
                            for (int j = 0; j < 16; ++j) {
                                const int sp = __ldg(perm + col + j);
                                if (sp >= 0) {
                                    double x = (double)v[j];
                                    if (h64) x += __hiloint2double((int)d[2 * j + 1], (int)d[2 * j]);
                                    double* w = wdot + (int64_t)sp * ng + i;
                                    // first (often only) group: a streaming store, so that
                                    // wdot does not push the Gibbs scratch out of L2
                                    if (first_group) __stcs(w, x);
                                    else *w += x;
                                }
                            }
                    }
                }
                first_group = false;
                um::fence_before_sync();
                __syncthreads();
            }
        }
        um::fence_before_sync();
        __syncthreads();
    }
    if (!ok && lane == 0) atomicExch(err, 1);
    __syncthreads();
    if (warp == 0) um::tmem_dealloc(tbase, tcols);
}

const void* kernel_for(int g_smem, int nt) {
    if (g_smem) return nt == 4 ? (const void*)getrates_tc_kernel<true, 4>
                               : nt == 2 ? (const void*)getrates_tc_kernel<true, 2> : (const void*)getrates_tc_kernel<true, 1>;
    return nt == 4 ? (const void*)getrates_tc_kernel<false, 4>
                   : nt == 2 ? (const void*)getrates_tc_kernel<false, 2> : (const void*)getrates_tc_kernel<false, 1>;
}

template <bool GS, int NT>
cudaError_t launch_tc(const MixedPlan* p, const DevMech& m, const double* P, const double* T, const double* Y,
                      double* wdot, int64_t ng, double* scratch, int64_t grid, cudaStream_t s) {
    getrates_tc_kernel<GS, NT><<<(unsigned)grid, kTile * NT, p->smem, s>>>(m, p->nu, p->fast, p->npad, p->nhalf, p->nchunk,
                                                                           p->tcols, P, T, Y, wdot, ng, scratch,
                                                                           p->err, p->group, p->perm, p->hot,
                                                                           p->hot_every);
    return cudaGetLastError();
}

}  // namespace

// ---------------------------------------------------------------- host side
cudaError_t mixed_prepare(const DevMech& m, const cg_mech_view& v, int device, MixedPlan** out) {
    *out = nullptr;
    const int ns = m.ns, nr = m.nr;
    int npad = (ns + 31) / 32 * 32;
    if (npad > 512) return cudaErrorNotSupported;     // TMEM holds 512 FP32 columns per lane
    const int nhalf = npad <= 256 ? npad : npad / 2;
    uint32_t tcols = 32;
    while ((int)tcols < npad) tcols <<= 1;
    const int nchunk = (nr + kChunk - 1) / kChunk;
    // the largest share count is planned for; the [nt][128] partial-sum slots follow the state
    const size_t rows = (size_t)ns + 1;                       // + the dummy row of TcFast
    const size_t base = 6 * (size_t)kABytes + 2 * (size_t)npad * 32 + rows * kTile * 4 + 4 * kTile * 8 + 32;
    const size_t with_g = base + rows * kTile * 8;
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    const size_t limit = prop.sharedMemPerBlockOptin;
    if (base > limit) return cudaErrorNotSupported;
    MixedPlan* p = new MixedPlan();
    p->ns = ns;
    p->nr = nr;
    p->npad = npad;
    p->nhalf = nhalf;
    p->nchunk = nchunk;
    p->tcols = tcols;
    p->g_smem = with_g <= limit ? 1 : 0;
    // FP32 accumulation runs over `group` chunks (16 reactions each) before
    // the partial sums are added into the FP64 output: 64 reactions for small
    // mechanisms (GRI30 needs it for 1e-6), the whole mechanism for large
    // ones, whose output does not fit in L2 and would otherwise be read back
    // from DRAM at every flush (348/2163: 3.5e-7 with one flush)
    p->group = npad <= 128 ? 4 : nchunk;
    p->smem = p->g_smem ? with_g : base;
    // resident CTAs per SM, limited by shared memory and by 512 TMEM columns
    int per_sm = (int)(prop.sharedMemPerMultiprocessor / (p->smem + 1024));
    per_sm = std::min(per_sm, (int)(512 / tcols));
    per_sm = std::max(per_sm, 1);
    // threads per point: the most (4, 2, 1) whose registers still let per_sm
    // CTAs share the SM's register file
    p->nt = 1;
    for (int nt : {4, 2}) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, kernel_for(p->g_smem, nt)) != cudaSuccess) continue;
        if ((long)per_sm * kTile * nt * fa.numRegs <= prop.regsPerMultiprocessor &&
            per_sm * kTile * nt <= prop.maxThreadsPerMultiProcessor) {
            p->nt = nt;
            break;
        }
    }
    p->grid = prop.multiProcessorCount * per_sm;
    // nu chunks in the canonical K-major layout: B[n][k] = nu of species n in reaction 16*chunk + k
    std::vector<float> nuf((size_t)ns * nr, 0.0f);
    const int32_t* rp = (const int32_t*)v.a[CG_RPTR];
    const int32_t* pp = (const int32_t*)v.a[CG_PPTR];
    const int32_t* rsp = (const int32_t*)v.a[CG_RSP];
    const int32_t* psp = (const int32_t*)v.a[CG_PSP];
    const double* rnu = (const double*)v.a[CG_RNU];
    const double* pnu = (const double*)v.a[CG_PNU];
    for (int r = 0; r < nr; ++r) {
        for (int j = rp[r]; j < rp[r + 1]; ++j) nuf[(size_t)rsp[j] * nr + r] -= (float)rnu[j];
        for (int j = pp[r]; j < pp[r + 1]; ++j) nuf[(size_t)psp[j] * nr + r] += (float)pnu[j];
    }
    // accumulator columns: for large mechanisms (one FP64 flush per tile) the
    // species most reactions touch come first, and up to 48 of them (what the
    // spare tensor-memory columns hold as FP64, in multiples of 16) get FP64
    // accumulators flushed every hot_every chunks; otherwise file order
    std::vector<int> perm(npad, -1);
    for (int n = 0; n < ns; ++n) perm[n] = n;
    if (p->group == nchunk && nchunk > p->hot_every) {
        std::vector<int> nnz(ns, 0);
        for (int n = 0; n < ns; ++n)
            for (int r = 0; r < nr; ++r) nnz[n] += nuf[(size_t)n * nr + r] != 0.0f;
        std::stable_sort(perm.begin(), perm.begin() + ns, [&](int a, int b) { return nnz[a] > nnz[b]; });
        p->hot = std::min(48, std::min(((int)tcols - npad) / 2, ns) / 16 * 16);
    }
    std::vector<__nv_bfloat16> img((size_t)nchunk * npad * kChunk, __float2bfloat16(0.0f));
    bool exact = true;
    for (int ch = 0; ch < nchunk; ++ch)
        for (int n = 0; n < ns; ++n)
            for (int k = 0; k < kChunk; ++k) {
                const int r = ch * kChunk + k;
                if (r >= nr) continue;
                const float x = nuf[(size_t)perm[n] * nr + r];
                const __nv_bfloat16 b = __float2bfloat16(x);
                if (__bfloat162float(b) != x) exact = false;
                const size_t off = ((size_t)(n >> 3) * (kChunk * 16) + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2) / 2;
                img[(size_t)ch * npad * kChunk + off] = b;
            }
    if (!exact) {
        delete p;
        return cudaErrorNotSupported;                  // coefficients not exact in BF16
    }
    const size_t img_bytes = (img.size() * sizeof(__nv_bfloat16) + 255) / 256 * 256;
    const size_t fast_bytes = ((size_t)nr * sizeof(TcFast) + 255) / 256 * 256;
    const size_t perm_bytes = ((size_t)npad * sizeof(int) + 255) / 256 * 256;
    const size_t bytes = img_bytes + fast_bytes + perm_bytes + 256;
    e = cudaMalloc(&p->dbuf, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(p->dbuf, img.data(), img.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset((char*)p->dbuf + bytes - 256, 0, 256);
    if (e == cudaSuccess)
        e = cudaMemcpy((char*)p->dbuf + img_bytes + fast_bytes, perm.data(), perm.size() * sizeof(int),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kernel_for(p->g_smem, p->nt),
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem);
    if (e != cudaSuccess) {
        if (p->dbuf) cudaFree(p->dbuf);
        delete p;
        return e;
    }
    p->nu = (const __nv_bfloat16*)p->dbuf;
    p->fast = (const TcFast*)((char*)p->dbuf + img_bytes);
    p->perm = (const int*)((char*)p->dbuf + img_bytes + fast_bytes);
    if (nr > 0) {
        build_fast_kernel<<<(nr + 127) / 128, 128>>>(m, (TcFast*)p->fast);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            cudaFree(p->dbuf);
            delete p;
            return e;
        }
    }
    p->err = (int*)((char*)p->dbuf + bytes - 256);
    *out = p;
    return cudaSuccess;
}

void mixed_release(MixedPlan* p) {
    if (!p) return;
    if (p->dbuf) cudaFree(p->dbuf);
    delete p;
}

size_t mixed_workspace_bytes(const MixedPlan* p, int64_t ng) {
    if (!p || p->g_smem) return 0;
    int64_t tiles = (ng + kTile - 1) / kTile;
    int64_t grid = std::min<int64_t>(tiles, p->grid);
    return (size_t)grid * (p->ns + 1) * kTile * sizeof(double);
}

cudaError_t launch_getrates_mixed(const MixedPlan* p, const DevMech& m, const double* P, const double* T,
                                  const double* Y, double* wdot, int64_t ng, void* scratch, size_t scratch_bytes,
                                  cudaStream_t s) {
    if (ng <= 0) return cudaSuccess;
    int64_t tiles = (ng + kTile - 1) / kTile;
    int64_t grid = std::min<int64_t>(tiles, p->grid);
    if (!p->g_smem) {
        const int64_t fit = (int64_t)(scratch_bytes / ((size_t)(p->ns + 1) * kTile * sizeof(double)));
        grid = std::min<int64_t>(grid, fit);
        if (grid < 1 || !scratch) return cudaErrorInvalidValue;
    }
    double* gs = p->g_smem ? nullptr : (double*)scratch;
    // the kernel's shared-memory limit is this plan's, set under one lock with
    // the launch (a plan made later for a smaller mechanism sets it lower)
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    const cudaError_t e = cudaFuncSetAttribute(kernel_for(p->g_smem, p->nt),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem);
    if (e != cudaSuccess) return e;
    switch ((p->g_smem ? 10 : 0) + p->nt) {
        case 14: return launch_tc<true, 4>(p, m, P, T, Y, wdot, ng, gs, grid, s);
        case 12: return launch_tc<true, 2>(p, m, P, T, Y, wdot, ng, gs, grid, s);
        case 11: return launch_tc<true, 1>(p, m, P, T, Y, wdot, ng, gs, grid, s);
        case 4: return launch_tc<false, 4>(p, m, P, T, Y, wdot, ng, gs, grid, s);
        case 2: return launch_tc<false, 2>(p, m, P, T, Y, wdot, ng, gs, grid, s);
        default: return launch_tc<false, 1>(p, m, P, T, Y, wdot, ng, gs, grid, s);
    }
}

int mixed_error_flag(const MixedPlan* p) {
    int v = 0;
    if (!p || cudaMemcpy(&v, p->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return v;
}

}  // namespace cg
