// Plain FP64 getrates: one grid point per thread.
//
// Computes the same quantities, in the same units, as the reference's
// generated getrates (chemgen/templates/python_header.j2:25-56, ytoc.j2,
// exp_g.j2, reactions/{standard,third_body,troe,plog}.j2) and its HIP
// successor rdot_merge_kernel (reactions_hip/hip_v1_cpp.j2:15-159), with
// Lindemann and SRI falloff added.
//
// Data layout (HBM): P[ng], T[ng], Y[k*ng + i], wdot[k*ng + i] -- the
// reference's device layout (reactions_hip/device_functions_h.j2:701-719), so
// every per-species load and store of a warp is one contiguous 256-byte run.
//
// Per-point state: three arrays of ns doubles -- C (mol/cm^3), EGp = cgm::cg_exp_clamped(smh) *
// Patm/(R0 T), and the wdot accumulator -- laid out [array][species][thread]
// in shared memory (ns small enough) or in a per-block slice of a scratch
// buffer (large ns).  Each thread only ever touches its own column, so the
// kernel needs no barrier.  Folding pfac into EGp turns the reference's
// kb = kf * prod EG_r / prod EG_p / pfac^dnu (standard.j2:7-16) into
// kb = kf * prod EGp_r / prod EGp_p.
//
// Reactions are processed kind by kind (the blob stores them grouped), so the
// control flow is warp-uniform; coefficient records are read with uniform
// 16-byte loads.
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <mutex>
#include <vector>

#include "cg_math.cuh"
#include "rates_common.cuh"

namespace cg {

struct PointState {
    double* C;     // C[k * B]
    double* E;     // EGp[k * B]
    double* W;     // wdot[k * B]
};

template <int B>
__device__ __forceinline__ void scatter_compact(const DRxn& R, double rr, double* W) {
#pragma unroll
    for (int j = 0; j < kMaxCompact; ++j)
        if (j < R.nre) {
            const int s = slot_species(R.sp[j]);
            W[s * B] = fma(-(double)slot_nu(R.sp[j]), rr, W[s * B]);
        }
#pragma unroll
    for (int j = 0; j < kMaxCompact; ++j)
        if (j < R.npr) {
            const int s = slot_species(R.sp[3 + j]);
            W[s * B] = fma((double)slot_nu(R.sp[3 + j]), rr, W[s * B]);
        }
}

// kb and the net rate of progress mfac * (qf - qb) of one reaction with
// forward rate kf (reactions/standard.j2:3-19).  mfac is the third-body
// concentration for three-body reactions, 1 otherwise (third_body.j2:30-31).
// C and EGp are read with stride B.
template <int B>
__device__ __forceinline__ double net_rate(const DevMech& m, const DRxn& R, double kf, double mfac, const double* C,
                                          const double* E) {
    if (R.flags & kFCompact) {
        double qf = kf, qb = 0.0;
        if (R.flags & CG_F_REVERSIBLE) {
            double num = 1.0, den = 1.0, cp = 1.0;
#pragma unroll
            for (int j = 0; j < kMaxCompact; ++j)
                if (j < R.nre) num *= ipow3(E[slot_species(R.sp[j]) * B], slot_nu(R.sp[j]));
#pragma unroll
            for (int j = 0; j < kMaxCompact; ++j)
                if (j < R.npr) {
                    const int s = slot_species(R.sp[3 + j]), nu = slot_nu(R.sp[3 + j]);
                    den *= ipow3(E[s * B], nu);
                    cp *= ipow3(C[s * B], nu);
                }
            qb = kf * num * rcp_nr(den) * cp;
        }
#pragma unroll
        for (int j = 0; j < kMaxCompact; ++j)
            if (j < R.nre) qf *= ipow3(C[slot_species(R.sp[j]) * B], slot_nu(R.sp[j]));
        return mfac * (qf - qb);
    }
    const int g = R.gen;
    const int r0 = __ldg(m.gen_rptr + g), r1 = __ldg(m.gen_rptr + g + 1);
    const int p0 = __ldg(m.gen_pptr + g), p1 = __ldg(m.gen_pptr + g + 1);
    double qf = kf, qb = 0.0;
    for (int j = r0; j < r1; ++j) {
        const int s = __ldg(m.gen_sp + j);
        const double nu = __ldg(m.gen_nu + j);
        qf *= (nu == 1.0) ? C[s * B] : pow(C[s * B], nu);
    }
    if (R.flags & CG_F_REVERSIBLE) {
        double ratio = 1.0, cp = 1.0;
        for (int j = r0; j < r1; ++j) {
            const int s = __ldg(m.gen_sp + j);
            const double nu = __ldg(m.gen_nu + j);
            ratio *= (nu == 1.0) ? E[s * B] : pow(E[s * B], nu);
        }
        for (int j = p0; j < p1; ++j) {
            const int s = __ldg(m.gen_sp + j);
            const double nu = __ldg(m.gen_nu + j);
            ratio /= (nu == 1.0) ? E[s * B] : pow(E[s * B], nu);
            cp *= (nu == 1.0) ? C[s * B] : pow(C[s * B], nu);
        }
        qb = kf * ratio * cp;
    }
    return mfac * (qf - qb);
}

// kb, q and the scatter for one reaction with forward rate kf.  mfac
// multiplies (qf - qb): the third-body concentration for three-body
// reactions, 1 otherwise (third_body.j2:30-31).
template <int B>
__device__ __forceinline__ void finish(const DevMech& m, const DRxn& R, double kf, double mfac,
                                       const PointState& st) {
    if (R.flags & kFCompact) {
        double qf = kf, qb = 0.0;
        if (R.flags & CG_F_REVERSIBLE) {
            double num = 1.0, den = 1.0, cp = 1.0;
#pragma unroll
            for (int j = 0; j < kMaxCompact; ++j)
                if (j < R.nre) num *= ipow3(st.E[slot_species(R.sp[j]) * B], slot_nu(R.sp[j]));
#pragma unroll
            for (int j = 0; j < kMaxCompact; ++j)
                if (j < R.npr) {
                    const int s = slot_species(R.sp[3 + j]), nu = slot_nu(R.sp[3 + j]);
                    den *= ipow3(st.E[s * B], nu);
                    cp *= ipow3(st.C[s * B], nu);
                }
            qb = kf * num * rcp_nr(den) * cp;
        }
#pragma unroll
        for (int j = 0; j < kMaxCompact; ++j)
            if (j < R.nre) qf *= ipow3(st.C[slot_species(R.sp[j]) * B], slot_nu(R.sp[j]));
        scatter_compact<B>(R, mfac * (qf - qb), st.W);
        return;
    }
    // general stoichiometry (fractional nu or more than 3 species on a side)
    const int g = R.gen;
    const int r0 = __ldg(m.gen_rptr + g), r1 = __ldg(m.gen_rptr + g + 1);
    const int p0 = __ldg(m.gen_pptr + g), p1 = __ldg(m.gen_pptr + g + 1);
    double qf = kf, qb = 0.0;
    for (int j = r0; j < r1; ++j) {
        const int s = __ldg(m.gen_sp + j);
        const double nu = __ldg(m.gen_nu + j);
        qf *= (nu == 1.0) ? st.C[s * B] : pow(st.C[s * B], nu);
    }
    if (R.flags & CG_F_REVERSIBLE) {
        double ratio = 1.0, cp = 1.0;
        for (int j = r0; j < r1; ++j) {
            const int s = __ldg(m.gen_sp + j);
            const double nu = __ldg(m.gen_nu + j);
            ratio *= (nu == 1.0) ? st.E[s * B] : pow(st.E[s * B], nu);
        }
        for (int j = p0; j < p1; ++j) {
            const int s = __ldg(m.gen_sp + j);
            const double nu = __ldg(m.gen_nu + j);
            ratio /= (nu == 1.0) ? st.E[s * B] : pow(st.E[s * B], nu);
            cp *= (nu == 1.0) ? st.C[s * B] : pow(st.C[s * B], nu);
        }
        qb = kf * ratio * cp;
    }
    const double rr = mfac * (qf - qb);
    for (int j = r0; j < r1; ++j) {
        const int s = __ldg(m.gen_sp + j);
        st.W[s * B] = fma(-__ldg(m.gen_nu + j), rr, st.W[s * B]);
    }
    for (int j = p0; j < p1; ++j) {
        const int s = __ldg(m.gen_sp + j);
        st.W[s * B] = fma(__ldg(m.gen_nu + j), rr, st.W[s * B]);
    }
}

__device__ __forceinline__ double arrhenius(double lnA, double b, double theta, double sgn, const PointT& pt) {
    return sgn * cgm::cg_exp_clamped(fma(b, pt.lnT, lnA) - theta * pt.invT);
}

template <int B>
__device__ __forceinline__ double third_body_m(const DevMech& m, int r, double ctot, const PointState& st) {
    double M = ctot;
    const int e0 = __ldg(m.eff_ptr + r), e1 = __ldg(m.eff_ptr + r + 1);
    for (int e = e0; e < e1; ++e) M = fma(__ldg(m.eff_val + e), st.C[__ldg(m.eff_sp + e) * B], M);
    return M;
}

// Falloff forward rate: kinf * Pr/(1+Pr) * F (troe.j2:21-45); Lindemann F = 1,
// SRI F = d [a cgm::cg_exp_clamped(-b/T) + cgm::cg_exp_clamped(-T/c)]^X T^e with X = 1/(1 + cgm::cg_log10(Pr)^2).
__device__ __forceinline__ double falloff_kf(int kind, int flags, const DRxn& R, const DFall& f, double e_sri_or_t2,
                                             double M, const PointT& pt) {
    const double kinf = arrhenius(R.lnA, R.b, R.theta, R.sgn, pt);
    const double k0 = arrhenius(f.lnA0, f.b0, f.theta0, f.sgn0, pt);
    const double Pr = k0 * M / kinf;
    double F = 1.0;
    if (kind == CG_TROE) {
        double Fc = fma(f.p[0], cgm::cg_exp_clamped(-pt.T * f.p[1]), f.p[2] * cgm::cg_exp_clamped(-pt.T * f.p[3]));
        if (flags & CG_F_TROE_T2) Fc += cgm::cg_exp_clamped(-e_sri_or_t2 * pt.invT);
        const double lFc = cgm::cg_log10(Fc);
        const double c1 = fma(-0.67, lFc, -0.4);
        const double n1 = fma(-1.27, lFc, 0.75);
        const double lp = cgm::cg_log10(Pr) + c1;
        const double f1 = lp / fma(-0.14, lp, n1);
        F = cgm::cg_exp_clamped(2.302585092994045684 * lFc / fma(f1, f1, 1.0));
    } else if (kind == CG_SRI) {
        const double lp = cgm::cg_log10(Pr);
        const double X = 1.0 / fma(lp, lp, 1.0);
        const double base = fma(f.p[0], cgm::cg_exp_clamped(-f.p[1] * pt.invT), cgm::cg_exp_clamped(-pt.T * f.p[2]));
        F = f.p[3] * cgm::cg_exp_clamped(fma(X, cgm::cg_log(base), e_sri_or_t2 * pt.lnT));
    }
    return kinf * (Pr / (1.0 + Pr)) * F;
}

// PLOG (plog.j2:4-38): bracket P between tabulated pressures and interpolate
// ln kf linearly in ln P; below the first / above the last level the
// nearest level's rate is used.
__device__ __forceinline__ double plog_kf(const DevMech& m, int row, double P, double lnP, const PointT& pt) {
    const int l0 = __ldg(m.plog_ptr + row), l1 = __ldg(m.plog_ptr + row + 1);
    int l = l0;
    while (l < l1 && !(P < __ldg(m.plog_p + l))) ++l;
    int la, lb;
    if (l == l0) {
        la = lb = l0;
    } else if (l == l1) {
        la = lb = l1 - 1;
    } else {
        la = l - 1;
        lb = l;
    }
    double kfl = 0.0, kfh = 0.0;
    for (int t = __ldg(m.plog_tptr + la); t < __ldg(m.plog_tptr + la + 1); ++t) {
        const double4 c = m.plog_term[t];
        kfl += arrhenius(c.x, c.y, c.z, c.w, pt);
    }
    if (lb == la) return kfl;
    for (int t = __ldg(m.plog_tptr + lb); t < __ldg(m.plog_tptr + lb + 1); ++t) {
        const double4 c = m.plog_term[t];
        kfh += arrhenius(c.x, c.y, c.z, c.w, pt);
    }
    const double a = __ldg(m.plog_lnp + la), b = __ldg(m.plog_lnp + lb);
    const double lkl = cgm::cg_log(kfl);
    return cgm::cg_exp_clamped(lkl + (cgm::cg_log(kfh) - lkl) * (lnP - a) / (b - a));
}

// The whole getrates for the point handled by this thread.  `st` points at
// this thread's column of the state arrays (stride B).
template <int B>
__device__ __forceinline__ void getrates_point(const DevMech& m, bool active, int64_t i, int64_t ng, const double* P,
                                               const double* Tg, const double* Y, double* wdot, const PointState& st) {
    const int ns = m.ns;
    double T = 1000.0, Pp = kPatm;
    if (active) {
        T = Tg[i];
        Pp = P[i];
    }
    // ytoc.j2:3-18
    double csum = 0.0;
    for (int k = 0; k < ns; ++k) {
        const double c = (active ? Y[(int64_t)k * ng + i] : 1.0) * __ldg(m.inv_mw + k);
        st.C[k * B] = c;
        csum += c;
    }
    const double fac = Pp / (kR0 * csum * T);
    double ctot = 0.0;
    for (int k = 0; k < ns; ++k) {
        const double c = st.C[k * B] * fac;
        st.C[k * B] = c;
        ctot += c;
    }
    PointT pt;
    pt.T = T;
    pt.lnT = cgm::cg_log(T);
    pt.invT = 1.0 / T;
    // exp_g.j2:2-27, with pfac = Patm/(R0 T) folded in
    const double pfac = kPatm / (kR0 * T);
    for (int k = 0; k < ns; ++k) {
        st.E[k * B] = cgm::cg_exp_clamped(species_smh(m.thermo, k, T, pt.lnT, pt.invT)) * pfac;
        st.W[k * B] = 0.0;
    }
    // elementary reactions, two at a time for instruction-level parallelism
    int r = m.seg[CG_STANDARD];
    const int r_std = m.seg[CG_STANDARD + 1];
    for (; r + 1 < r_std; r += 2) {
        const DRxn R0 = load_rxn(m.rxn + r);
        const DRxn R1 = load_rxn(m.rxn + r + 1);
        const double kf0 = arrhenius(R0.lnA, R0.b, R0.theta, R0.sgn, pt);
        const double kf1 = arrhenius(R1.lnA, R1.b, R1.theta, R1.sgn, pt);
        finish<B>(m, R0, kf0, 1.0, st);
        finish<B>(m, R1, kf1, 1.0, st);
    }
    for (; r < r_std; ++r) {
        const DRxn R = load_rxn(m.rxn + r);
        finish<B>(m, R, arrhenius(R.lnA, R.b, R.theta, R.sgn, pt), 1.0, st);
    }
    // three-body
    for (r = m.seg[CG_THIRD_BODY]; r < m.seg[CG_THIRD_BODY + 1]; ++r) {
        const DRxn R = load_rxn(m.rxn + r);
        const double M = third_body_m<B>(m, r, ctot, st);
        finish<B>(m, R, arrhenius(R.lnA, R.b, R.theta, R.sgn, pt), M, st);
    }
    // falloff: Lindemann, Troe, SRI
#pragma unroll 1
    for (int kind = CG_LINDEMANN; kind <= CG_SRI; ++kind) {
        for (r = m.seg[kind]; r < m.seg[kind + 1]; ++r) {
            const DRxn R = load_rxn(m.rxn + r);
            const DFall f = load_fall(m.fall + R.aux);
            const double x2 = __ldg(&m.fall2[R.aux].T2);
            const double M = third_body_m<B>(m, r, ctot, st);
            finish<B>(m, R, falloff_kf(kind, R.flags, R, f, x2, M, pt), 1.0, st);
        }
    }
    // PLOG
    if (m.seg[CG_PLOG] < m.seg[CG_PLOG + 1]) {
        const double lnP = cgm::cg_log(Pp);
        for (r = m.seg[CG_PLOG]; r < m.seg[CG_PLOG + 1]; ++r) {
            const DRxn R = load_rxn(m.rxn + r);
            finish<B>(m, R, plog_kf(m, R.aux, Pp, lnP, pt), 1.0, st);
        }
    }
    if (active)
        for (int k = 0; k < ns; ++k) wdot[(int64_t)k * ng + i] = st.W[k * B];
}

// State in shared memory: [3][ns][B] doubles per block.
template <int B>
__global__ void __launch_bounds__(B) getrates_fp64_smem(DevMech m, const double* __restrict__ P,
                                                        const double* __restrict__ T, const double* __restrict__ Y,
                                                        double* __restrict__ wdot, int64_t ng) {
    extern __shared__ double smem[];
    const int tid = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * B + tid;
    PointState st{smem + tid, smem + m.ns * B + tid, smem + 2 * m.ns * B + tid};
    getrates_point<B>(m, i < ng, i, ng, P, T, Y, wdot, st);
}

// State in global scratch: persistent blocks, one [3][ns][B] slice each.
template <int B>
__global__ void __launch_bounds__(B) getrates_fp64_global(DevMech m, const double* __restrict__ P,
                                                          const double* __restrict__ T, const double* __restrict__ Y,
                                                          double* __restrict__ wdot, int64_t ng, double* scratch) {
    const int tid = threadIdx.x;
    double* base = scratch + (int64_t)blockIdx.x * 3 * m.ns * B + tid;
    PointState st{base, base + m.ns * B, base + 2 * m.ns * B};
    const int64_t nchunks = (ng + B - 1) / B;
    for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const int64_t i = c * B + tid;
        getrates_point<B>(m, i < ng, i, ng, P, T, Y, wdot, st);
    }
}

// ------------------------------------------------ staged large-mechanism kernel
//
// For mechanisms whose per-point state is too large for a block of points in
// shared memory with one thread per point and per-thread wdot (JetSurf-size,
// hundreds of species).  A persistent CTA owns a tile of 32 points -- one
// point per lane, so every lane of a warp works on the same reaction and no
// branch diverges -- and keeps the tile's C and EGp in shared memory.  The
// reactions run in chunks of R:
//   pass 1  warp w computes the net rates of progress of reactions w, w + W,
//           ... of the chunk for the 32 points into a staging array q[R][32];
//   pass 2  warp w owns species w, w + W, ..., whose FP64 wdot accumulators
//           sit in its registers for the whole tile, and adds
//           sum_r nu_kr q_r over the chunk from a per-chunk species -> reaction
//           list (reactions/standard.j2:21-27).
// Each species has one owner, so the sums need no atomics and wdot is
// written once per point, and nothing is kept in global scratch: DRAM traffic
// is the inputs and outputs.

// Pre-decoded record of a standard or three-body reaction with at most three
// molecules a side, built once per mechanism: the rate needs no decoding,
// no loop and no power; unused molecule slots name the dummy species ns,
// whose C and EGp are 1.
struct __align__(16) StFast {
    double lnA, b, theta;        // ln|A|, b, Ea/Rc
    unsigned short sr[3], sp[3]; // reactant / product molecules
    unsigned int flags;          // kStOn | kStRev | kStThird | kStNeg
    int pad[2];
};
static_assert(sizeof(StFast) == 48, "StFast must stay 48 bytes");
constexpr unsigned kStOn = 1, kStRev = 2, kStThird = 4, kStNeg = 8;

struct StagedPlan {
    int W = 16;                 // warps per CTA
    int kpw = 0;                // accumulator slots per warp (template instance)
    int R = 0;                  // reactions per chunk
    int nchunk = 0;
    size_t smem = 0;
    int grid = 0;
    const int* ptr = nullptr;   // [nchunk][ns + 1] into the entries
    const int* er = nullptr;    // reaction of each entry, within its chunk
    const double* enu = nullptr;  // net stoichiometric coefficient of each entry
    const StFast* fast = nullptr;   // [nr]
    void* dbuf = nullptr;
};

constexpr int kStTile = 32;

__device__ __forceinline__ StFast load_stfast(const StFast* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    StFast f;
    int4* d = reinterpret_cast<int4*>(&f);
    d[0] = __ldg(q);
    d[1] = __ldg(q + 1);
    d[2] = __ldg(q + 2);
    return f;
}

// M = ctot + sum_e (eff_e - 1) C[sp_e] of reaction r (third_body.j2:18-31), the
// efficiencies taken four at a time so that their loads are in flight
// together; the sum keeps the table's order.
__device__ __forceinline__ double staged_m(const DevMech& m, int r, double ctot, const double* C) {
    double M = ctot;
    const int e1 = __ldg(m.eff_ptr + r + 1);
    for (int e = __ldg(m.eff_ptr + r); e < e1; e += 4) {
        int sp[4];
        double ev[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool ok = e + u < e1;
            sp[u] = ok ? __ldg(m.eff_sp + e + u) : 0;
            ev[u] = ok ? __ldg(m.eff_val + e + u) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double cv = C[sp[u] * kStTile];
            if (e + u < e1) M = fma(ev[u], cv, M);
        }
    }
    return M;
}

template <int W, int KPW>
__global__ void __launch_bounds__(32 * W, 1)
    getrates_fp64_staged(DevMech m, int R, int nchunk, const int* __restrict__ cptr, const int* __restrict__ cer,
                         const double* __restrict__ cnu, const StFast* __restrict__ fast,
                         const double* __restrict__ P, const double* __restrict__ Tg,
                         const double* __restrict__ Y, double* __restrict__ wdot, int64_t ng,
                         const unsigned long long* __restrict__ count) {
    extern __shared__ double smem[];
    const int ns = m.ns;
    // the arrays' stride is ng; with a device-side count only its first
    // min(*count, ng) points are computed
    const int64_t npts = count ? min(ng, (int64_t)*count) : ng;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* sC = smem;                       // [ns + 1][32] (row ns: the dummy species, 1)
    double* sE = sC + (ns + 1) * kStTile;    // [ns + 1][32]
    double* sQ = sE + (ns + 1) * kStTile;    // [R][32]
    double* sRed = sQ + R * kStTile;         // [W][32]
    const int64_t ntiles = (npts + kStTile - 1) / kStTile;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t i = tile * kStTile + lane;
        const bool act = i < npts;
        const double T = act ? Tg[i] : 1000.0;
        const double Pp = act ? P[i] : kPatm;
        // ytoc.j2:3-18; species k handled by warp k % W, sums met in shared memory
        double part = 0.0;
        for (int k = warp; k < ns; k += W) {
            const double c = (act ? Y[(int64_t)k * ng + i] : 1.0) * __ldg(m.inv_mw + k);
            sC[k * kStTile + lane] = c;
            part += c;
        }
        sRed[warp * kStTile + lane] = part;
        __syncthreads();
        double csum = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) csum += sRed[w * kStTile + lane];
        const double fac = Pp / (kR0 * csum * T);
        part = 0.0;
        for (int k = warp; k < ns; k += W) {
            const double c = sC[k * kStTile + lane] * fac;
            sC[k * kStTile + lane] = c;
            part += c;
        }
        PointT pt;
        pt.T = T;
        pt.lnT = cgm::cg_log(T);
        pt.invT = 1.0 / T;
        // exp_g.j2:2-27 with pfac = Patm/(R0 T) folded in
        const double pfac = kPatm / (kR0 * T);
        for (int k = warp; k < ns; k += W)
            sE[k * kStTile + lane] = cgm::cg_exp_clamped(species_smh(m.thermo, k, T, pt.lnT, pt.invT)) * pfac;
        if (warp == 0) {
            sC[ns * kStTile + lane] = 1.0;
            sE[ns * kStTile + lane] = 1.0;
        }
        __syncthreads();                     // csum read by every warp before sRed is reused
        sRed[warp * kStTile + lane] = part;
        __syncthreads();
        double ctot = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) ctot += sRed[w * kStTile + lane];
        const double lnP = cgm::cg_log(Pp);
        double acc[KPW];
#pragma unroll
        for (int j = 0; j < KPW; ++j) acc[j] = 0.0;
        const double* C = sC + lane;
        const double* E = sE + lane;
        for (int c = 0; c < nchunk; ++c) {
            // pass 1: net rates of progress of this warp's reactions of the chunk
            for (int rl = warp; rl < R; rl += W) {
                const int r = c * R + rl;
                double q = 0.0;
                const StFast F = load_stfast(fast + (r < m.nr ? r : 0));
                // the warp's next record moves into L1 while this one is evaluated
                // (a prefetch: no registers held)
                if (r + W < m.nr) asm volatile("prefetch.global.L1 [%0];" ::"l"(fast + r + W));
                if (r < m.nr && (F.flags & kStOn)) {
                    const double kf = cgm::cg_exp_clamped(fma(F.b, pt.lnT, F.lnA) - F.theta * pt.invT);
                    q = kf * C[F.sr[0] * kStTile] * C[F.sr[1] * kStTile] * C[F.sr[2] * kStTile];
                    if (F.flags & kStRev) {
                        const double num = E[F.sr[0] * kStTile] * E[F.sr[1] * kStTile] * E[F.sr[2] * kStTile];
                        const double den = E[F.sp[0] * kStTile] * E[F.sp[1] * kStTile] * E[F.sp[2] * kStTile];
                        q -= kf * num * rcp_nr(den) * C[F.sp[0] * kStTile] * C[F.sp[1] * kStTile] *
                             C[F.sp[2] * kStTile];
                    }
                    if (F.flags & kStThird) q *= staged_m(m, r, ctot, C);
                    if (F.flags & kStNeg) q = -q;
                } else if (r < m.nr) {
                    const DRxn Rx = load_rxn(m.rxn + r);
                    int kind = CG_STANDARD;
                    while (kind < CG_PLOG && r >= m.seg[kind + 1]) ++kind;
                    if (kind == CG_STANDARD) {
                        q = net_rate<kStTile>(m, Rx, arrhenius(Rx.lnA, Rx.b, Rx.theta, Rx.sgn, pt), 1.0, C, E);
                    } else if (kind == CG_THIRD_BODY) {
                        const double M = staged_m(m, r, ctot, C);
                        q = net_rate<kStTile>(m, Rx, arrhenius(Rx.lnA, Rx.b, Rx.theta, Rx.sgn, pt), M, C, E);
                    } else if (kind == CG_PLOG) {
                        q = net_rate<kStTile>(m, Rx, plog_kf(m, Rx.aux, Pp, lnP, pt), 1.0, C, E);
                    } else {
                        const DFall f = load_fall(m.fall + Rx.aux);
                        const double x2 = __ldg(&m.fall2[Rx.aux].T2);
                        const double M = staged_m(m, r, ctot, C);
                        q = net_rate<kStTile>(m, Rx, falloff_kf(kind, Rx.flags, Rx, f, x2, M, pt), 1.0, C, E);
                    }
                }
                sQ[rl * kStTile + lane] = q;
            }
            __syncthreads();
            // pass 2: this warp's species accumulate the chunk's contributions
            const int* cp = cptr + (int64_t)c * (ns + 1);
#pragma unroll
            for (int j = 0; j < KPW; ++j) {
                const int k = warp + j * W;
                if (k < ns) {
                    // entries four at a time, their loads in flight together;
                    // the sum keeps the list's order
                    const int e1 = __ldg(cp + k + 1);
                    for (int e = __ldg(cp + k); e < e1; e += 4) {
                        int ix[4];
                        double nu[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const bool ok = e + u < e1;
                            ix[u] = ok ? __ldg(cer + e + u) : 0;
                            nu[u] = ok ? __ldg(cnu + e + u) : 0.0;
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const double qv = sQ[ix[u] * kStTile + lane];
                            if (e + u < e1) acc[j] = fma(nu[u], qv, acc[j]);
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (act) {
#pragma unroll
            for (int j = 0; j < KPW; ++j) {
                const int k = warp + j * W;
                if (k < ns) wdot[(int64_t)k * ng + i] = acc[j];
            }
        }
    }
}

template <int W, int KPW>
static const void* staged_fn() {
    return (const void*)getrates_fp64_staged<W, KPW>;
}

static const void* staged_kernel(int kpw) {
    switch (kpw) {
        case 8: return staged_fn<16, 8>();
        case 16: return staged_fn<16, 16>();
        case 24: return staged_fn<16, 24>();
        case 32: return staged_fn<16, 32>();
        default: return nullptr;
    }
}

cudaError_t staged_prepare(const DevMech& m, const cg_mech_view& v, int device, StagedPlan** out) {
    *out = nullptr;
    const int ns = m.ns, nr = m.nr;
    StagedPlan pl;
    pl.W = 16;
    const int need = (ns + pl.W - 1) / pl.W;
    pl.kpw = need <= 8 ? 8 : need <= 16 ? 16 : need <= 24 ? 24 : need <= 32 ? 32 : 0;
    if (!pl.kpw || nr == 0) return cudaErrorNotSupported;
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    const size_t limit = prop.sharedMemPerBlockOptin;
    const size_t fixed = (size_t)2 * (ns + 1) * kStTile * 8 + (size_t)pl.W * kStTile * 8;
    if (fixed + (size_t)pl.W * kStTile * 8 > limit) return cudaErrorNotSupported;
    int R = (int)((limit - fixed) / (kStTile * 8));
    R = std::min(R, 256) / pl.W * pl.W;
    R = std::min(R, (nr + pl.W - 1) / pl.W * pl.W);
    if (R < pl.W) return cudaErrorNotSupported;
    pl.R = R;
    pl.nchunk = (nr + R - 1) / R;
    pl.smem = fixed + (size_t)R * kStTile * 8;
    // per-chunk species -> (reaction, net nu) lists, reactions in kernel order
    const int32_t* rp = (const int32_t*)v.a[CG_RPTR];
    const int32_t* pp = (const int32_t*)v.a[CG_PPTR];
    const int32_t* rsp = (const int32_t*)v.a[CG_RSP];
    const int32_t* psp = (const int32_t*)v.a[CG_PSP];
    const double* rnu = (const double*)v.a[CG_RNU];
    const double* pnu = (const double*)v.a[CG_PNU];
    std::vector<int> ptr((size_t)pl.nchunk * (ns + 1), 0);
    std::vector<int> er;
    std::vector<double> enu;
    std::vector<double> net(ns, 0.0);
    std::vector<std::vector<std::pair<int, double>>> lists(ns);
    for (int c = 0; c < pl.nchunk; ++c) {
        for (auto& l : lists) l.clear();
        for (int r = c * R; r < std::min(nr, (c + 1) * R); ++r) {
            for (int j = rp[r]; j < rp[r + 1]; ++j) net[rsp[j]] -= rnu[j];
            for (int j = pp[r]; j < pp[r + 1]; ++j) net[psp[j]] += pnu[j];
            for (int j = rp[r]; j < rp[r + 1]; ++j)
                if (net[rsp[j]] != 0.0) {
                    lists[rsp[j]].push_back({r - c * R, net[rsp[j]]});
                    net[rsp[j]] = 0.0;
                }
            for (int j = pp[r]; j < pp[r + 1]; ++j)
                if (net[psp[j]] != 0.0) {
                    lists[psp[j]].push_back({r - c * R, net[psp[j]]});
                    net[psp[j]] = 0.0;
                }
            for (int j = rp[r]; j < rp[r + 1]; ++j) net[rsp[j]] = 0.0;
        }
        int* cp = ptr.data() + (size_t)c * (ns + 1);
        cp[0] = (int)er.size();
        for (int k = 0; k < ns; ++k) {
            for (const auto& x : lists[k]) {
                er.push_back(x.first);
                enu.push_back(x.second);
            }
            cp[k + 1] = (int)er.size();
        }
    }
    // fast records: standard and three-body reactions, integer stoichiometry,
    // at most three molecules a side, A != 0
    const double* karh = (const double*)v.a[CG_KARH];
    const double* arh = (const double*)v.a[CG_ARH];
    const int32_t* rflags = (const int32_t*)v.a[CG_FLAGS];
    const int n_std = (int)v.s[CG_S_NSTD], n_3b = (int)v.s[CG_S_N3B];
    std::vector<StFast> fr(nr);
    for (int r = 0; r < nr; ++r) {
        StFast f{};
        f.lnA = karh[4 * r];
        f.b = karh[4 * r + 1];
        f.theta = karh[4 * r + 2];
        for (int j = 0; j < 3; ++j) f.sr[j] = f.sp[j] = (unsigned short)ns;
        bool ok = r < n_std + n_3b && arh[3 * r] != 0.0 && (rflags[r] & CG_F_INT_NU);
        int nf = 0, nb = 0;
        for (int j = rp[r]; ok && j < rp[r + 1]; ++j)
            for (int k = 0; k < (int)rnu[j]; ++k) {
                if (nf == 3) ok = false;
                else f.sr[nf++] = (unsigned short)rsp[j];
            }
        for (int j = pp[r]; ok && j < pp[r + 1]; ++j)
            for (int k = 0; k < (int)pnu[j]; ++k) {
                if (nb == 3) ok = false;
                else f.sp[nb++] = (unsigned short)psp[j];
            }
        if (ok)
            f.flags = kStOn | ((rflags[r] & CG_F_REVERSIBLE) ? kStRev : 0) | (r >= n_std ? kStThird : 0) |
                      (karh[4 * r + 3] < 0.0 ? kStNeg : 0);
        else
            f.flags = 0;
        fr[r] = f;
    }
    const size_t b_ptr = (ptr.size() * sizeof(int) + 255) / 256 * 256;
    const size_t b_er = (std::max<size_t>(er.size(), 1) * sizeof(int) + 255) / 256 * 256;
    const size_t b_nu = (std::max<size_t>(enu.size(), 1) * sizeof(double) + 255) / 256 * 256;
    const size_t b_fast = (size_t)nr * sizeof(StFast);
    StagedPlan* p = new StagedPlan(pl);
    e = cudaMalloc(&p->dbuf, b_ptr + b_er + b_nu + b_fast);
    char* d = (char*)p->dbuf;
    if (e == cudaSuccess) e = cudaMemcpy(d, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !er.empty()) e = cudaMemcpy(d + b_ptr, er.data(), er.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !enu.empty())
        e = cudaMemcpy(d + b_ptr + b_er, enu.data(), enu.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d + b_ptr + b_er + b_nu, fr.data(), b_fast, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(staged_kernel(p->kpw), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem);
    if (e != cudaSuccess) {
        if (p->dbuf) cudaFree(p->dbuf);
        delete p;
        return e;
    }
    p->ptr = (const int*)d;
    p->er = (const int*)(d + b_ptr);
    p->enu = (const double*)(d + b_ptr + b_er);
    p->fast = (const StFast*)(d + b_ptr + b_er + b_nu);
    p->grid = prop.multiProcessorCount;
    *out = p;
    return cudaSuccess;
}

void staged_release(StagedPlan* p) {
    if (!p) return;
    if (p->dbuf) cudaFree(p->dbuf);
    delete p;
}

cudaError_t launch_getrates_staged(const StagedPlan* p, const DevMech& m, const double* P, const double* T,
                                   const double* Y, double* wdot, int64_t ng, cudaStream_t s,
                                   const unsigned long long* count) {
    if (ng <= 0) return cudaSuccess;
    const int64_t tiles = (ng + kStTile - 1) / kStTile;
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, p->grid);
    const unsigned threads = 32u * (unsigned)p->W;
    // Every plan of the same kernel instance (one per handle) sets the
    // instance's shared-memory limit to its own size: set it and launch
    // under one lock, so that a handle made later for a smaller mechanism
    // cannot leave the limit below this plan's.
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    cudaError_t e = cudaFuncSetAttribute(staged_kernel(p->kpw), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)p->smem);
    if (e != cudaSuccess) return e;
#define CG_STAGED_LAUNCH(K)                                                                                  \
    getrates_fp64_staged<16, K><<<grid, threads, p->smem, s>>>(m, p->R, p->nchunk, p->ptr, p->er, p->enu, p->fast, \
                                                               P, T, Y, wdot, ng, count)
    switch (p->kpw) {
        case 8: CG_STAGED_LAUNCH(8); break;
        case 16: CG_STAGED_LAUNCH(16); break;
        case 24: CG_STAGED_LAUNCH(24); break;
        case 32: CG_STAGED_LAUNCH(32); break;
        default: return cudaErrorInvalidValue;
    }
#undef CG_STAGED_LAUNCH
    return cudaGetLastError();
}

// ---------------------------------------------------------------- launchers
template <int B>
static cudaError_t launch_smem(const DevMech& m, const double* P, const double* T, const double* Y, double* wdot,
                               int64_t ng, cudaStream_t s) {
    const size_t smem = (size_t)3 * m.ns * B * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(getrates_fp64_smem<B>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t blocks = (ng + B - 1) / B;
    getrates_fp64_smem<B><<<(unsigned)blocks, B, smem, s>>>(m, P, T, Y, wdot, ng);
    return cudaGetLastError();
}

// Shared-memory footprint of one point's state.
static inline size_t point_bytes(int ns) { return (size_t)3 * ns * sizeof(double); }

// Points per block for the shared-memory variant, chosen to maximise resident
// points per SM; 0 when the state does not fit.
// Block size (32, 64 or 128 points) of the one-thread-per-point kernel with
// the most resident points per SM, or 0 when none fits; *pts_per_sm (may be
// NULL) receives that number of points.
int fp64_smem_block(int ns, size_t smem_per_sm, size_t smem_per_block, long* pts_per_sm) {
    int best_b = 0;
    long best_pts = 0;
    const int cands[3] = {32, 64, 128};
    for (int c = 0; c < 3; ++c) {
        const int b = cands[c];
        const size_t need = point_bytes(ns) * b;
        if (need > smem_per_block) continue;
        long blocks = (long)(smem_per_sm / (need + 1024));
        if (blocks > 2048 / b) blocks = 2048 / b;
        const long pts = blocks * b;
        if (pts >= best_pts) {
            best_pts = pts;
            best_b = b;
        }
    }
    if (pts_per_sm) *pts_per_sm = best_pts;
    return best_pts >= 64 ? best_b : 0;
}

cudaError_t launch_getrates_fp64(const DevMech& m, const double* P, const double* T, const double* Y, double* wdot,
                                 int64_t ng, int block, double* scratch, int64_t scratch_blocks, cudaStream_t s) {
    if (ng <= 0) return cudaSuccess;
    switch (block) {
        case 32: return launch_smem<32>(m, P, T, Y, wdot, ng, s);
        case 64: return launch_smem<64>(m, P, T, Y, wdot, ng, s);
        case 128: return launch_smem<128>(m, P, T, Y, wdot, ng, s);
        default: break;
    }
    // global-state variant, 64 points per block
    int64_t grid = (ng + 63) / 64;
    if (grid > scratch_blocks) grid = scratch_blocks;
    if (grid <= 0 || scratch == nullptr) return cudaErrorInvalidValue;
    getrates_fp64_global<64><<<(unsigned)grid, 64, 0, s>>>(m, P, T, Y, wdot, ng, scratch);
    return cudaGetLastError();
}

size_t fp64_global_slice_bytes(int ns) { return point_bytes(ns) * 64; }

}  // namespace cg

namespace cg {
int fp64_global_blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, getrates_fp64_global<64>, 64, 0) != cudaSuccess || n < 1)
        n = 4;
    return n;
}
}  // namespace cg
