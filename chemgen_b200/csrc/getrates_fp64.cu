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
int fp64_smem_block(int ns, size_t smem_per_sm, size_t smem_per_block) {
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
