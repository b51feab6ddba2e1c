// Analytic derivatives of getrates: the dense Jacobian d wdot / d(T, Y) and
// the adjoint (vector-Jacobian product), table-driven so that one compiled
// kernel serves every mechanism.
//
// The reference has no derivative code (its torch prototype
// chemgen/chemistry_nn.py:15-85 never ran); these kernels differentiate the
// rate law of reactions/*.j2:
//     wdot_k = sum_r nu_kr q_r,   q_r = m_r (qf_r - qb_r),   C = C(T, Y)
// with
//     dC_m/dY_j  = (ctot delta_mj - C_m) / (W_j S),  S = sum_j Y_j / W_j,
//     dC_m/dT    = -C_m / T,   dM/dC_m = 1 + (eff_m - 1),
//     d ln kf/dT = (b + theta/T) / T   (theta = Ea/Rc),
//     d ln kb/dT = d ln kf/dT + sum nu_r dE_r - sum nu_p dE_p,
//     dE_k       = d ln(exp(smh_k) Patm/(R0 T))/dT = d smh_k/dT - 1/T,
//     falloff:   d ln kf = d ln kinf + g (d ln k0 - d ln kinf + d ln M) + d ln F|_Pr,
//                g = 1/(1 + Pr) + d ln F / d ln Pr.
// Mass-action derivatives use the product of the other factors, so species
// at zero concentration keep exact derivatives.
//
// Layouts: J[(k*(ns+1) + c)*ng + i], column c = 0 for T and 1 + j for Y_j;
// adjoint outputs gT[i], gY[j*ng + i], gP[i].  Per-point state (C, EGp, dE
// and, for the Jacobian, the dense-M vector A) lives in a scratch buffer of
// 4*ns*ng doubles laid out [array][species][point].
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>

#include "cg_math.cuh"
#include "rates_common.cuh"

namespace cg {
namespace {

constexpr double kLn10 = 2.302585092994045684;

struct DState {
    double* C;
    double* E;
    double* D;
    double* A;
    int64_t s;       // stride between species (ng)
};

__device__ __forceinline__ double arr_ln(double lnA, double b, double theta, const PointT& pt) {
    return fma(b, pt.lnT, lnA) - theta * pt.invT;
}
__device__ __forceinline__ double arr_dln(double b, double theta, const PointT& pt) {
    return fma(theta, pt.invT, b) * pt.invT;
}

// Forward rate constant of a falloff reaction and its derivatives:
// dlkf = d ln kf/dT at fixed M, gM = d ln kf/dM.
__device__ void falloff_d(int kind, int flags, const DRxn& R, const DFall& f, double x2, double M, const PointT& pt,
                          double& kf, double& dlkf, double& gM) {
    const double lkinf = arr_ln(R.lnA, R.b, R.theta, pt);
    const double lr = arr_ln(f.lnA0, f.b0, f.theta0, pt) - lkinf;
    const double Pr = cgm::cg_exp_clamped(lr) * M * (f.sgn0 * R.sgn);
    const double dlkinf = arr_dln(R.b, R.theta, pt);
    const double dlPr = arr_dln(f.b0, f.theta0, pt) - dlkinf;
    const double ipr = cgm::cg_rcp(1.0 + Pr);
    double lnF = 0.0, gpr = ipr, dlF_T = 0.0;
    if (kind == CG_TROE) {
        const double e3 = cgm::cg_exp_clamped(-pt.T * f.p[1]);
        const double e1 = cgm::cg_exp_clamped(-pt.T * f.p[3]);
        double Fc = fma(f.p[0], e3, f.p[2] * e1);
        double dFc = fma(-f.p[0] * f.p[1], e3, -f.p[2] * f.p[3] * e1);
        if (flags & CG_F_TROE_T2) {
            const double e2 = cgm::cg_exp_clamped(-x2 * pt.invT);
            Fc += e2;
            dFc = fma(x2 * pt.invT * pt.invT, e2, dFc);
        }
        const double lFc = cgm::cg_log10(Fc);
        const double u = fma(lr, 1.0 / kLn10, cgm::cg_log10(M)) + fma(-0.67, lFc, -0.4);
        const double nn = fma(-1.27, lFc, 0.75);
        const double den = fma(-0.14, u, nn);
        const double iden = cgm::cg_rcp(den);
        const double f1 = u * iden;
        const double q1 = cgm::cg_rcp(fma(f1, f1, 1.0));
        lnF = kLn10 * lFc * q1;
        const double dF_df1 = -2.0 * lFc * f1 * q1 * q1;
        const double dF_dlpr = dF_df1 * nn * iden * iden;
        const double df1_dlfc = (-0.67 * den + 1.1762 * u) * iden * iden;
        const double dF_dlfc = fma(dF_df1, df1_dlfc, q1);
        gpr = ipr + dF_dlpr;
        dlF_T = dF_dlfc * dFc * cgm::cg_rcp(Fc);
    } else if (kind == CG_SRI) {
        const double lp = fma(lr, 1.0 / kLn10, cgm::cg_log10(M));
        const double X = cgm::cg_rcp(fma(lp, lp, 1.0));
        const double eb = cgm::cg_exp_clamped(-f.p[1] * pt.invT);
        const double ec = cgm::cg_exp_clamped(-pt.T * f.p[2]);
        const double base = fma(f.p[0], eb, ec);
        const double dbase = fma(f.p[0] * f.p[1] * pt.invT * pt.invT, eb, -f.p[2] * ec);
        const double lb = cgm::cg_log(base);
        lnF = cgm::cg_log(f.p[3]) + fma(X, lb, x2 * pt.lnT);
        gpr = ipr - 2.0 * lp * X * X * lb / kLn10;
        dlF_T = fma(X, dbase * cgm::cg_rcp(base), x2 * pt.invT);
    }
    kf = R.sgn * cgm::cg_exp_clamped(lkinf + lnF) * (Pr * ipr);
    dlkf = fma(gpr, dlPr, dlkinf) + dlF_T;
    gM = gpr * cgm::cg_rcp(M);
}

// PLOG forward rate, d ln kf/dT and d ln kf/d ln P (plog.j2:4-38).
__device__ void plog_d(const DevMech& m, int row, double P, double lnP, const PointT& pt, double& kf, double& dlkf,
                       double& dlkf_lnP) {
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
    double k[2] = {0.0, 0.0}, d[2] = {0.0, 0.0};
    const int lev[2] = {la, lb};
    for (int s = 0; s < 2; ++s) {
        for (int t = __ldg(m.plog_tptr + lev[s]); t < __ldg(m.plog_tptr + lev[s] + 1); ++t) {
            const double4 c = m.plog_term[t];
            const double x = c.w * cgm::cg_exp_clamped(arr_ln(c.x, c.y, c.z, pt));
            k[s] += x;
            d[s] = fma(x, arr_dln(c.y, c.z, pt), d[s]);
        }
        d[s] *= cgm::cg_rcp(k[s]);
    }
    if (la == lb) {
        kf = k[0];
        dlkf = d[0];
        dlkf_lnP = 0.0;
        return;
    }
    const double a = __ldg(m.plog_lnp + la), b = __ldg(m.plog_lnp + lb);
    const double w = (lnP - a) / (b - a);
    const double kl = cgm::cg_log(k[0]), kh = cgm::cg_log(k[1]);
    kf = cgm::cg_exp_clamped(kl + (kh - kl) * w);
    dlkf = fma(w, d[1] - d[0], d[0]);
    dlkf_lnP = (kh - kl) / (b - a);
}

// One side of a reaction: species, coefficients (compact or general rows).
// NMAX = 3 holds the compact form only; its loops unroll, so the arrays stay
// in registers.
template <int NMAX>
struct SideT {
    int n;
    int sp[NMAX];
    double nu[NMAX];
};
using Side = SideT<16>;

__device__ __forceinline__ void load_sides3(const DRxn& R, SideT<3>& re, SideT<3>& pr) {
    re.n = R.nre;
    pr.n = R.npr;
#pragma unroll
    for (int j = 0; j < kMaxCompact; ++j) {
        re.sp[j] = slot_species(R.sp[j]);
        re.nu[j] = slot_nu(R.sp[j]);
        pr.sp[j] = slot_species(R.sp[3 + j]);
        pr.nu[j] = slot_nu(R.sp[3 + j]);
    }
}

__device__ __forceinline__ void load_sides(const DevMech& m, const DRxn& R, Side& re, Side& pr) {
    if (R.flags & kFCompact) {
        re.n = R.nre;
        pr.n = R.npr;
        for (int j = 0; j < kMaxCompact; ++j) {
            re.sp[j] = slot_species(R.sp[j]);
            re.nu[j] = slot_nu(R.sp[j]);
            pr.sp[j] = slot_species(R.sp[3 + j]);
            pr.nu[j] = slot_nu(R.sp[3 + j]);
        }
        return;
    }
    const int g = R.gen;
    const int r0 = __ldg(m.gen_rptr + g), r1 = __ldg(m.gen_rptr + g + 1);
    const int p0 = __ldg(m.gen_pptr + g), p1 = __ldg(m.gen_pptr + g + 1);
    re.n = min(r1 - r0, 16);
    pr.n = min(p1 - p0, 16);
    for (int j = 0; j < re.n; ++j) {
        re.sp[j] = __ldg(m.gen_sp + r0 + j);
        re.nu[j] = __ldg(m.gen_nu + r0 + j);
    }
    for (int j = 0; j < pr.n; ++j) {
        pr.sp[j] = __ldg(m.gen_sp + p0 + j);
        pr.nu[j] = __ldg(m.gen_nu + p0 + j);
    }
}

__device__ __forceinline__ double powi(double x, double nu) {
    if (nu == 1.0) return x;
    if (nu == 2.0) return x * x;
    if (nu == 3.0) return x * x * x;
    return pow(x, nu);
}

// d(c^nu)/dc
__device__ __forceinline__ double dpowi(double x, double nu) {
    if (nu == 1.0) return 1.0;
    if (nu == 2.0) return 2.0 * x;
    if (nu == 3.0) return 3.0 * x * x;
    return nu * pow(x, nu - 1.0);
}

// Derivative of prod_i c_i^nu_i with respect to factor j (product of the others).
template <int NMAX>
__device__ __forceinline__ double dprod(const SideT<NMAX>& s, const double* c, int j) {
    double p = dpowi(c[j], s.nu[j]);
#pragma unroll(NMAX == 3 ? 3 : 1)
    for (int i = 0; i < NMAX; ++i)
        if (i < s.n && i != j) p *= powi(c[i], s.nu[i]);
    return p;
}

// Rate of progress of reaction r at one point and its derivatives: dqdT at
// fixed C, dqdM (three-body and falloff), and dq/dC_j over the reaction's own
// species (dsp[0..nd)); re/pr are its sides.  State C, EGp and dE are read
// with stride st.s.
template <int NMAX>
struct RxnGradT {
    int kind;
    bool usesM;
    double qnet, dqdT, dqdM, dlkf_lnP;
    int nd;
    int dsp[2 * NMAX];
    double dqc[2 * NMAX];
};
using RxnGrad = RxnGradT<16>;

// The rate constants of reaction r at one point: kf and its d ln kf/dT,
// kb, and for three-body and falloff reactions M and d ln kf/dM (gM).  The
// row-owner Jacobian computes them once per reaction and tile (KC = 5
// values, stride 32 apart, in `kc`); reaction_grad can take them from there.
// per-reaction slots of the row-owner kernel's tile cache: a compact
// reaction's derivatives (dq/dT, dq/dM, dq/dC of its six slots), or another
// reaction's five rate constants (kf, kb, dlkf, gM, M)
constexpr int kDC = 8;

__device__ __forceinline__ void reaction_k(const DevMech& m, int r, const DRxn& R, int kind, const PointT& pt,
                                           double ctot, double Pv, double lnP, const DState& st, double& kf,
                                           double& kb, double& dlkf, double& gM, double& M, double& dlkf_lnP) {
    M = 0.0;
    gM = 0.0;
    dlkf_lnP = 0.0;
    if (kind != CG_STANDARD && kind != CG_PLOG) {
        M = ctot;
        for (int e = __ldg(m.eff_ptr + r); e < __ldg(m.eff_ptr + r + 1); ++e)
            M = fma(__ldg(m.eff_val + e), st.C[__ldg(m.eff_sp + e) * st.s], M);
    }
    if (kind == CG_STANDARD || kind == CG_THIRD_BODY) {
        kf = R.sgn * cgm::cg_exp_clamped(arr_ln(R.lnA, R.b, R.theta, pt));
        dlkf = arr_dln(R.b, R.theta, pt);
    } else if (kind == CG_PLOG) {
        plog_d(m, R.aux, Pv, lnP, pt, kf, dlkf, dlkf_lnP);
    } else {
        const DFall f = load_fall(m.fall + R.aux);
        falloff_d(kind, R.flags, R, f, __ldg(&m.fall2[R.aux].T2), M, pt, kf, dlkf, gM);
    }
    kb = 0.0;
    if (R.flags & CG_F_REVERSIBLE) {
        double num = 1.0, den = 1.0;
        if (R.flags & kFCompact) {
#pragma unroll
            for (int j = 0; j < kMaxCompact; ++j) {
                if (j < R.nre) num *= ipow3(st.E[slot_species(R.sp[j]) * st.s], slot_nu(R.sp[j]));
                if (j < R.npr) den *= ipow3(st.E[slot_species(R.sp[3 + j]) * st.s], slot_nu(R.sp[3 + j]));
            }
        } else {
            const int g = R.gen;
            for (int j = __ldg(m.gen_rptr + g); j < __ldg(m.gen_rptr + g + 1); ++j)
                num *= powi(st.E[__ldg(m.gen_sp + j) * st.s], __ldg(m.gen_nu + j));
            for (int j = __ldg(m.gen_pptr + g); j < __ldg(m.gen_pptr + g + 1); ++j)
                den *= powi(st.E[__ldg(m.gen_sp + j) * st.s], __ldg(m.gen_nu + j));
        }
        kb = kf * num * cgm::cg_rcp(den);
    }
}

// NMAX = 3: compact reactions only (the caller checks kFCompact).  With
// CACHED the rate constants come from kc (reaction_k's values).
template <int NMAX, bool CACHED = false>
__device__ __forceinline__ void reaction_grad(const DevMech& m, int r, const DRxn& R, const PointT& pt, double ctot,
                                              double Pv, double lnP, const DState& st, SideT<NMAX>& re,
                                              SideT<NMAX>& pr, RxnGradT<NMAX>& g, const double* kc = nullptr) {
    int kind = CG_STANDARD;
    while (kind < CG_PLOG && r >= m.seg[kind + 1]) ++kind;
    if constexpr (NMAX == 3) load_sides3(R, re, pr);
    else load_sides(m, R, re, pr);
    double M, kf, kb_c, dlkf, gM, dlkf_lnP = 0.0;
    if constexpr (CACHED) {
        kf = kc[0];
        kb_c = kc[32];
        dlkf = kc[64];
        gM = kc[96];
        M = kc[128];
    } else {
        reaction_k(m, r, R, kind, pt, ctot, Pv, lnP, st, kf, kb_c, dlkf, gM, M, dlkf_lnP);
    }
    double cr[NMAX], cp[NMAX];
    double pf = 1.0;
#pragma unroll(NMAX == 3 ? 3 : 1)
    for (int j = 0; j < NMAX; ++j)
        if (j < re.n) {
            cr[j] = st.C[re.sp[j] * st.s];
            pf *= powi(cr[j], re.nu[j]);
        }
    const double qf = kf * pf;
    double kb = 0.0, qb = 0.0, dlKc = 0.0;
    if (R.flags & CG_F_REVERSIBLE) {
        double pb_ = 1.0;
#pragma unroll(NMAX == 3 ? 3 : 1)
        for (int j = 0; j < NMAX; ++j)
            if (j < re.n) dlKc = fma(re.nu[j], st.D[re.sp[j] * st.s], dlKc);
#pragma unroll(NMAX == 3 ? 3 : 1)
        for (int j = 0; j < NMAX; ++j)
            if (j < pr.n) {
                cp[j] = st.C[pr.sp[j] * st.s];
                pb_ *= powi(cp[j], pr.nu[j]);
                dlKc = fma(-pr.nu[j], st.D[pr.sp[j] * st.s], dlKc);
            }
        kb = kb_c;
        qb = kb * pb_;
    }
    const double mfac = (kind == CG_THIRD_BODY) ? M : 1.0;
    g.kind = kind;
    g.qnet = qf - qb;
    g.dlkf_lnP = dlkf_lnP;
    g.dqdT = mfac * fma(qf, dlkf, -qb * (dlkf + dlKc));
    g.dqdM = (kind == CG_THIRD_BODY) ? (qf - qb) : ((kind >= CG_LINDEMANN && kind <= CG_SRI) ? (qf - qb) * gM : 0.0);
    g.usesM = kind >= CG_THIRD_BODY && kind <= CG_SRI;
    const bool rev = (R.flags & CG_F_REVERSIBLE) != 0;
    if constexpr (NMAX == 3) {
        // fixed slots: 0..2 reactants, 3..5 products (unused: zero derivative
        // on species 0), so that every loop over the slots unrolls
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const bool on = j < re.n;
            g.dsp[j] = on ? re.sp[j] : 0;
            g.dqc[j] = on ? mfac * kf * dprod(re, cr, j) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const bool on = rev && j < pr.n;
            g.dsp[3 + j] = on ? pr.sp[j] : 0;
            g.dqc[3 + j] = on ? -mfac * kb * dprod(pr, cp, j) : 0.0;
        }
        g.nd = 6;
    } else {
        int nd = 0;
        for (int j = 0; j < re.n; ++j) {
            g.dsp[nd] = re.sp[j];
            g.dqc[nd++] = mfac * kf * dprod(re, cr, j);
        }
        if (rev)
            for (int j = 0; j < pr.n; ++j) {
                g.dsp[nd] = pr.sp[j];
                g.dqc[nd++] = -mfac * kb * dprod(pr, cp, j);
            }
        g.nd = nd;
    }
}

template <bool JAC, typename JT>
__global__ void __launch_bounds__(128) deriv_kernel(DevMech m, const double* __restrict__ P, const double* __restrict__ Tg,
                                                    const double* __restrict__ Y, const double* __restrict__ G,
                                                    JT* __restrict__ J, double* __restrict__ gT, double* __restrict__ gY,
                                                    double* __restrict__ gP, double* __restrict__ scratch, int64_t ng) {
    const int ns = m.ns;
    const int64_t ncol = ns + 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += (int64_t)gridDim.x * blockDim.x) {
        DState st{scratch + i, scratch + (int64_t)ns * ng + i, scratch + (int64_t)2 * ns * ng + i,
                  scratch + (int64_t)3 * ns * ng + i, ng};
        const double T = Tg[i], Pv = P[i];
        PointT pt;
        pt.T = T;
        pt.lnT = cgm::cg_log(T);
        pt.invT = 1.0 / T;
        double S = 0.0;
        for (int k = 0; k < ns; ++k) {
            const double c = Y[(int64_t)k * ng + i] * __ldg(m.inv_mw + k);
            st.C[k * st.s] = c;
            S += c;
        }
        const double fac = Pv / (kR0 * S * T);
        double ctot = 0.0;
        for (int k = 0; k < ns; ++k) {
            const double c = st.C[k * st.s] * fac;
            st.C[k * st.s] = c;
            ctot += c;
        }
        const double pfac = kPatm / (kR0 * T);
        for (int k = 0; k < ns; ++k) {
            const double* th = m.thermo + 16 * k;
            const double* c = (T < __ldg(th)) ? th + 1 : th + 8;
            double cc[7];
            for (int j = 0; j < 7; ++j) cc[j] = __ldg(c + j);
            const double smh = smh_poly(cc, T, pt.lnT, pt.invT);
            st.E[k * st.s] = cgm::cg_exp_clamped(smh) * pfac;
            // d smh/dT - 1/T
            const double dp = fma(fma(fma(4.0 * cc[5], T, 3.0 * cc[4]), T, 2.0 * cc[3]), T, cc[2]);
            st.D[k * st.s] = dp + fma(cc[6], pt.invT, cc[1]) * pt.invT - pt.invT;
            st.A[k * st.s] = 0.0;
        }
        if (JAC) {
            JT* Jp = J + i;
            for (int64_t c = 0; c < (int64_t)ns * ncol; ++c) Jp[c * ng] = (JT)0;
        } else {
            for (int k = 0; k < ns; ++k) gY[(int64_t)k * ng + i] = 0.0;   // holds C-bar until the end
        }
        double tb = 0.0, ab = 0.0, pb = 0.0;
        const double lnP = cgm::cg_log(Pv);
        for (int r = 0; r < m.nr; ++r) {
            Side re, pr;
            RxnGrad rg;
            const DRxn R = load_rxn(m.rxn + r);
            reaction_grad<16>(m, r, R, pt, ctot, Pv, lnP, st, re, pr, rg);
            const int kind = rg.kind, nd = rg.nd;
            const double dqdT = rg.dqdT, dqdM = rg.dqdM;
            const bool usesM = rg.usesM;
            const int* dsp = rg.dsp;
            const double* dqc = rg.dqc;
            if (JAC) {
                JT* Jp = J + i;
                // rows: every species of the reaction with its net coefficient contribution
                for (int side = 0; side < 2; ++side) {
                    const Side& s = side ? pr : re;
                    const double sg = side ? 1.0 : -1.0;
                    for (int kk = 0; kk < s.n; ++kk) {
                        const int k = s.sp[kk];
                        const double nu = sg * s.nu[kk];
                        Jp[(int64_t)(k * ncol) * ng] += (JT)(nu * dqdT);
                        for (int j = 0; j < nd; ++j) Jp[(int64_t)(k * ncol + 1 + dsp[j]) * ng] += (JT)(nu * dqc[j]);
                        if (usesM) {
                            st.A[k * st.s] = fma(nu, dqdM, st.A[k * st.s]);
                            for (int e = __ldg(m.eff_ptr + r); e < __ldg(m.eff_ptr + r + 1); ++e)
                                Jp[(int64_t)(k * ncol + 1 + __ldg(m.eff_sp + e)) * ng] +=
                                    (JT)(nu * __ldg(m.eff_val + e) * dqdM);
                        }
                    }
                }
            } else {
                double gq = 0.0;
                for (int j = 0; j < re.n; ++j) gq = fma(-re.nu[j], G[(int64_t)re.sp[j] * ng + i], gq);
                for (int j = 0; j < pr.n; ++j) gq = fma(pr.nu[j], G[(int64_t)pr.sp[j] * ng + i], gq);
                tb = fma(gq, dqdT, tb);
                for (int j = 0; j < nd; ++j) gY[(int64_t)dsp[j] * ng + i] = fma(gq, dqc[j], gY[(int64_t)dsp[j] * ng + i]);
                if (usesM) {
                    ab = fma(gq, dqdM, ab);
                    for (int e = __ldg(m.eff_ptr + r); e < __ldg(m.eff_ptr + r + 1); ++e) {
                        const int64_t o = (int64_t)__ldg(m.eff_sp + e) * ng + i;
                        gY[o] = fma(gq * dqdM, __ldg(m.eff_val + e), gY[o]);
                    }
                }
                if (kind == CG_PLOG) pb = fma(gq, rg.qnet * rg.dlkf_lnP / Pv, pb);
            }
        }
        const double iS = 1.0 / S;
        if (JAC) {
            JT* Jp = J + i;
            for (int k = 0; k < ns; ++k) {
                const double ak = st.A[k * st.s];
                double rk = ak * ctot;
                for (int j = 0; j < ns; ++j) rk = fma((double)Jp[(int64_t)(k * ncol + 1 + j) * ng], st.C[j * st.s], rk);
                Jp[(int64_t)(k * ncol) * ng] = (JT)((double)Jp[(int64_t)(k * ncol) * ng] - rk * pt.invT);
                for (int j = 0; j < ns; ++j) {
                    const int64_t o = (int64_t)(k * ncol + 1 + j) * ng;
                    Jp[o] = (JT)(fma(ctot, (double)Jp[o] + ak, -rk) * __ldg(m.inv_mw + j) * iS);
                }
            }
        } else {
            double rho = 0.0;
            for (int k = 0; k < ns; ++k) {
                const double cb = gY[(int64_t)k * ng + i] + ab;
                gY[(int64_t)k * ng + i] = cb;
                rho = fma(cb, st.C[k * st.s], rho);
            }
            for (int k = 0; k < ns; ++k) {
                const int64_t o = (int64_t)k * ng + i;
                gY[o] = fma(ctot, gY[o], -rho) * __ldg(m.inv_mw + k) * iS;
            }
            gT[i] = tb - rho * pt.invT;
            if (gP) gP[i] = fma(rho, 1.0 / Pv, pb);
        }
    }
}

// ------------------------------------------------ row-owner Jacobian kernel
//
// J written once.  A persistent CTA owns a tile of 32 points (one per lane,
// so every lane of a warp evaluates the same reaction and nothing diverges)
// and keeps the tile's C, EGp and dE in shared memory.  Warp w owns the rows
// k = w, w + W, ...: for row k it walks the reactions that change species k
// (a per-species list of (reaction, net nu), built once per mechanism),
// evaluates each reaction's rate derivatives for its 32 points and adds
// nu * dq into the row, held in a [ns + 1][32] shared-memory buffer of its
// own; then it applies the chain rule through C(T, Y) (file header) and
// stores the row's ns + 1 columns, one coalesced 32-point store each.  A
// reaction is evaluated once per species it changes (about four times), in
// exchange for J never being read back from memory.
constexpr int kJTile = 32;
constexpr int kJMaxWarps = 8;

template <typename JT>
__global__ void __launch_bounds__(32 * kJMaxWarps, 1)
    jac_rows_kernel(DevMech m, const int* __restrict__ lptr, const int* __restrict__ lrx,
                    const double* __restrict__ lnu, const int* __restrict__ lrow, const double* __restrict__ P,
                    const double* __restrict__ Tg,
                    const double* __restrict__ Y, JT* __restrict__ J, int64_t ng, double* __restrict__ kcache) {
    extern __shared__ double smem[];
    const int ns = m.ns, ncol = ns + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double* sC = smem;
    double* sE = sC + ns * kJTile;
    double* sD = sE + ns * kJTile;
    double* sRed = sD + ns * kJTile;                               // [kJMaxWarps][32]
    double* row = sRed + kJMaxWarps * kJTile + (size_t)warp * ncol * kJTile + lane;   // this warp's [ncol][32]
    const int64_t ntiles = (ng + kJTile - 1) / kJTile;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t i = tile * kJTile + lane;
        const bool act = i < ng;
        const double T = act ? Tg[i] : 1000.0;
        const double Pv = act ? P[i] : kPatm;
        PointT pt;
        pt.T = T;
        pt.lnT = cgm::cg_log(T);
        pt.invT = 1.0 / T;
        double part = 0.0;
        for (int k = warp; k < ns; k += nw) {
            const double c = (act ? Y[(int64_t)k * ng + i] : 1.0) * __ldg(m.inv_mw + k);
            sC[k * kJTile + lane] = c;
            part += c;
        }
        sRed[warp * kJTile + lane] = part;
        __syncthreads();
        double S = 0.0;
        for (int w = 0; w < nw; ++w) S += sRed[w * kJTile + lane];
        const double fac = Pv / (kR0 * S * T);
        const double pfac = kPatm / (kR0 * T);
        part = 0.0;
        for (int k = warp; k < ns; k += nw) {
            const double c = sC[k * kJTile + lane] * fac;
            sC[k * kJTile + lane] = c;
            part += c;
            const double* th = m.thermo + 16 * k;
            const double* cf = (T < __ldg(th)) ? th + 1 : th + 8;
            double cc[7];
#pragma unroll
            for (int j = 0; j < 7; ++j) cc[j] = __ldg(cf + j);
            sE[k * kJTile + lane] = cgm::cg_exp_clamped(smh_poly(cc, T, pt.lnT, pt.invT)) * pfac;
            const double dp = fma(fma(fma(4.0 * cc[5], T, 3.0 * cc[4]), T, 2.0 * cc[3]), T, cc[2]);
            sD[k * kJTile + lane] = dp + fma(cc[6], pt.invT, cc[1]) * pt.invT - pt.invT;
        }
        __syncthreads();                     // S read by every warp before sRed is reused
        sRed[warp * kJTile + lane] = part;
        __syncthreads();
        double ctot = 0.0;
        for (int w = 0; w < nw; ++w) ctot += sRed[w * kJTile + lane];
        const double lnP = cgm::cg_log(Pv);
        const DState st{sC + lane, sE + lane, sD + lane, nullptr, kJTile};
        const double iS = 1.0 / S;
        // phase 1: every reaction once, into this CTA's slice [nr][kDC][32]
        // (a few hundred KB: it stays in L2): a compact reaction's rate
        // derivatives, which the rows then only gather, or another reaction's
        // rate constants, from which each row that needs it evaluates them
        double* kc = kcache + (int64_t)blockIdx.x * m.nr * kDC * kJTile;
        for (int r = warp; r < m.nr; r += nw) {
            const DRxn R = load_rxn(m.rxn + r);
            double* o = kc + (int64_t)r * kDC * kJTile + lane;
            if (R.flags & kFCompact) {
                SideT<3> re, pr;
                RxnGradT<3> g;
                reaction_grad<3>(m, r, R, pt, ctot, Pv, lnP, st, re, pr, g);
                o[0] = g.dqdT;
                o[32] = g.dqdM;
#pragma unroll
                for (int j = 0; j < 6; ++j) o[(2 + j) * kJTile] = g.dqc[j];
                continue;
            }
            int kind = CG_STANDARD;
            while (kind < CG_PLOG && r >= m.seg[kind + 1]) ++kind;
            double kf, kb, dlkf, gM, M, dlp;
            reaction_k(m, r, R, kind, pt, ctot, Pv, lnP, st, kf, kb, dlkf, gM, M, dlp);
            o[0] = kf;
            o[32] = kb;
            o[64] = dlkf;
            o[96] = gM;
            o[128] = M;
        }
        __syncthreads();
        // rows t = warp, warp + nw, ...: species lrow[t], dealt out so that the
        // warps' lists are about equally long and reach the barrier together
        for (int t = warp; t < ns; t += nw) {
            const int k = __ldg(lrow + t);
            for (int c = 0; c < ncol; ++c) row[c * kJTile] = 0.0;
            double ak = 0.0;
            const int e1 = __ldg(lptr + k + 1);
            for (int e = __ldg(lptr + k); e < e1; ++e) {
                const int r = __ldg(lrx + e);
                const double nu = __ldg(lnu + e);
                const DRxn R = load_rxn(m.rxn + r);
                double dqdT, dqdM;
                bool usesM;
                const double* kr = kc + (int64_t)r * kDC * kJTile + lane;
                if (R.flags & kFCompact) {
                    // the derivatives from phase 1; the slots' species as
                    // reaction_grad<3> lays them out
                    SideT<3> re, pr;
                    load_sides3(R, re, pr);
                    const bool rev = (R.flags & CG_F_REVERSIBLE) != 0;
                    int dsp[6];
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        dsp[j] = j < re.n ? re.sp[j] : 0;
                        dsp[3 + j] = (rev && j < pr.n) ? pr.sp[j] : 0;
                    }
                    double dq[6];
#pragma unroll
                    for (int j = 0; j < 6; ++j) dq[j] = kr[(2 + j) * kJTile];
#pragma unroll
                    for (int j = 0; j < 6; ++j) row[(1 + dsp[j]) * kJTile] = fma(nu, dq[j], row[(1 + dsp[j]) * kJTile]);
                    dqdT = kr[0];
                    dqdM = kr[32];
                    int kind = CG_STANDARD;
                    while (kind < CG_PLOG && r >= m.seg[kind + 1]) ++kind;
                    usesM = kind >= CG_THIRD_BODY && kind <= CG_SRI;
                } else {
                    Side re, pr;
                    RxnGrad g;
                    reaction_grad<16, true>(m, r, R, pt, ctot, Pv, lnP, st, re, pr, g, kr);
                    for (int j = 0; j < g.nd; ++j)
                        row[(1 + g.dsp[j]) * kJTile] = fma(nu, g.dqc[j], row[(1 + g.dsp[j]) * kJTile]);
                    dqdT = g.dqdT;
                    dqdM = g.dqdM;
                    usesM = g.usesM;
                }
                row[0] = fma(nu, dqdT, row[0]);
                if (usesM) {
                    // dM/dC_j = 1 + (eff_j - 1): the 1 goes to every column (ak), the rest is sparse
                    ak = fma(nu, dqdM, ak);
                    for (int f = __ldg(m.eff_ptr + r); f < __ldg(m.eff_ptr + r + 1); ++f)
                        row[(1 + __ldg(m.eff_sp + f)) * kJTile] =
                            fma(nu * __ldg(m.eff_val + f), dqdM, row[(1 + __ldg(m.eff_sp + f)) * kJTile]);
                }
            }
            // chain rule through C(T, Y): rk = sum_j dwdot_k/dC_j C_j
            double rk = ak * ctot;
            for (int j = 0; j < ns; ++j) rk = fma(row[(1 + j) * kJTile], sC[j * kJTile + lane], rk);
            if (act) {
                // streaming stores: J is never read back, so its lines go
                // first when L2 needs room and the tile's rate-constant cache
                // stays resident instead of being written back to DRAM
                JT* Jr = J + (int64_t)k * ncol * ng + i;
                __stcs(Jr, (JT)(row[0] - rk * pt.invT));
                for (int j = 0; j < ns; ++j)
                    __stcs(Jr + (int64_t)(1 + j) * ng,
                           (JT)(fma(ctot, row[(1 + j) * kJTile] + ak, -rk) * __ldg(m.inv_mw + j) * iS));
            }
        }
        __syncthreads();                     // the tile's state stays until every row is done
    }
}

// ------------------------------------------------ tile VJP kernel
//
// dL/d(T, Y, P) from the cotangent G = dL/dwdot without J and without global
// scratch.  A persistent CTA owns a tile of 32 points (one per lane) and keeps
// the tile's C, EGp, dEGp/dT and G in shared memory.  Warp w evaluates the
// rate derivatives of reactions w, w + W, ... and adds their contributions
// into dL/dC accumulators [ns][32] of its own (shared memory, no atomics); at
// the end of the tile the W copies are added in warp order, so the result
// does not depend on scheduling.  The chain rule through C(T, Y) then follows
// the in-place kernel's (file header).
constexpr int kVMaxWarps = 16;

__global__ void __launch_bounds__(32 * kVMaxWarps, 1)
    vjp_tile_kernel(DevMech m, const double* __restrict__ P, const double* __restrict__ Tg,
                    const double* __restrict__ Y, const double* __restrict__ G, double* __restrict__ gT,
                    double* __restrict__ gY, double* __restrict__ gP, int64_t ng) {
    extern __shared__ double smem[];
    const int ns = m.ns;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double* sC = smem;
    double* sE = sC + ns * kJTile;
    double* sD = sE + ns * kJTile;
    double* sG = sD + ns * kJTile;
    double* sRed = sG + ns * kJTile;                                   // [3][kVMaxWarps][32]
    double* sAcc = sRed + 3 * kVMaxWarps * kJTile;                     // [nw][ns][32]
    double* acc = sAcc + (size_t)warp * ns * kJTile + lane;            // this warp's dL/dC
    const int64_t ntiles = (ng + kJTile - 1) / kJTile;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t i = tile * kJTile + lane;
        const bool act = i < ng;
        const double T = act ? Tg[i] : 1000.0;
        const double Pv = act ? P[i] : kPatm;
        PointT pt;
        pt.T = T;
        pt.lnT = cgm::cg_log(T);
        pt.invT = 1.0 / T;
        double part = 0.0;
        for (int k = warp; k < ns; k += nw) {
            const double c = (act ? Y[(int64_t)k * ng + i] : 1.0) * __ldg(m.inv_mw + k);
            sC[k * kJTile + lane] = c;
            sG[k * kJTile + lane] = act ? G[(int64_t)k * ng + i] : 0.0;
            part += c;
        }
        for (int k = 0; k < ns; ++k) acc[k * kJTile] = 0.0;
        sRed[warp * kJTile + lane] = part;
        __syncthreads();
        double S = 0.0;
        for (int w = 0; w < nw; ++w) S += sRed[w * kJTile + lane];
        const double fac = Pv / (kR0 * S * T);
        const double pfac = kPatm / (kR0 * T);
        part = 0.0;
        for (int k = warp; k < ns; k += nw) {
            const double c = sC[k * kJTile + lane] * fac;
            sC[k * kJTile + lane] = c;
            part += c;
            const double* th = m.thermo + 16 * k;
            const double* cf = (T < __ldg(th)) ? th + 1 : th + 8;
            double cc[7];
#pragma unroll
            for (int j = 0; j < 7; ++j) cc[j] = __ldg(cf + j);
            sE[k * kJTile + lane] = cgm::cg_exp_clamped(smh_poly(cc, T, pt.lnT, pt.invT)) * pfac;
            const double dp = fma(fma(fma(4.0 * cc[5], T, 3.0 * cc[4]), T, 2.0 * cc[3]), T, cc[2]);
            sD[k * kJTile + lane] = dp + fma(cc[6], pt.invT, cc[1]) * pt.invT - pt.invT;
        }
        __syncthreads();                     // S read by every warp before sRed is reused
        sRed[warp * kJTile + lane] = part;
        __syncthreads();
        double ctot = 0.0;
        for (int w = 0; w < nw; ++w) ctot += sRed[w * kJTile + lane];
        const double lnP = cgm::cg_log(Pv);
        const DState st{sC + lane, sE + lane, sD + lane, nullptr, kJTile};
        const double* Gl = sG + lane;
        double tb = 0.0, ab = 0.0, pb = 0.0;
        for (int r = warp; r < m.nr; r += nw) {
            const DRxn R = load_rxn(m.rxn + r);
            double gq = 0.0, dqdT, dqdM, plog_term = 0.0;
            bool usesM;
            if (R.flags & kFCompact) {
                SideT<3> re, pr;
                RxnGradT<3> g;
                reaction_grad<3>(m, r, R, pt, ctot, Pv, lnP, st, re, pr, g);
                for (int j = 0; j < re.n; ++j) gq = fma(-re.nu[j], Gl[re.sp[j] * kJTile], gq);
                for (int j = 0; j < pr.n; ++j) gq = fma(pr.nu[j], Gl[pr.sp[j] * kJTile], gq);
                for (int j = 0; j < g.nd; ++j) acc[g.dsp[j] * kJTile] = fma(gq, g.dqc[j], acc[g.dsp[j] * kJTile]);
                dqdT = g.dqdT;
                dqdM = g.dqdM;
                usesM = g.usesM;
                if (g.kind == CG_PLOG) plog_term = g.qnet * g.dlkf_lnP / Pv;
            } else {
                Side re, pr;
                RxnGrad g;
                reaction_grad<16>(m, r, R, pt, ctot, Pv, lnP, st, re, pr, g);
                for (int j = 0; j < re.n; ++j) gq = fma(-re.nu[j], Gl[re.sp[j] * kJTile], gq);
                for (int j = 0; j < pr.n; ++j) gq = fma(pr.nu[j], Gl[pr.sp[j] * kJTile], gq);
                for (int j = 0; j < g.nd; ++j) acc[g.dsp[j] * kJTile] = fma(gq, g.dqc[j], acc[g.dsp[j] * kJTile]);
                dqdT = g.dqdT;
                dqdM = g.dqdM;
                usesM = g.usesM;
                if (g.kind == CG_PLOG) plog_term = g.qnet * g.dlkf_lnP / Pv;
            }
            tb = fma(gq, dqdT, tb);
            if (usesM) {
                ab = fma(gq, dqdM, ab);
                for (int e = __ldg(m.eff_ptr + r); e < __ldg(m.eff_ptr + r + 1); ++e) {
                    double* o = acc + __ldg(m.eff_sp + e) * kJTile;
                    *o = fma(gq * dqdM, __ldg(m.eff_val + e), *o);
                }
            }
            pb = fma(gq, plog_term, pb);
        }
        sRed[warp * kJTile + lane] = tb;
        sRed[(kVMaxWarps + warp) * kJTile + lane] = ab;
        sRed[(2 * kVMaxWarps + warp) * kJTile + lane] = pb;
        __syncthreads();
        tb = ab = pb = 0.0;
        for (int w = 0; w < nw; ++w) {
            tb += sRed[w * kJTile + lane];
            ab += sRed[(kVMaxWarps + w) * kJTile + lane];
            pb += sRed[(2 * kVMaxWarps + w) * kJTile + lane];
        }
        // dL/dC_k = sum over the warps' copies (in warp order) + dL/dM; this
        // warp's species' share of rho = sum_k dL/dC_k C_k
        double rpart = 0.0;
        for (int k = warp; k < ns; k += nw) {
            double cb = 0.0;
            for (int w = 0; w < nw; ++w) cb += sAcc[((size_t)w * ns + k) * kJTile + lane];
            cb += ab;
            sG[k * kJTile + lane] = cb;          // G is no longer needed
            rpart = fma(cb, sC[k * kJTile + lane], rpart);
        }
        __syncthreads();                     // tb, ab, pb read before sRed is reused
        sRed[warp * kJTile + lane] = rpart;
        __syncthreads();
        double rho = 0.0;
        for (int w = 0; w < nw; ++w) rho += sRed[w * kJTile + lane];
        const double iS = 1.0 / S;
        if (act) {
            for (int k = warp; k < ns; k += nw)
                gY[(int64_t)k * ng + i] = fma(ctot, sG[k * kJTile + lane], -rho) * __ldg(m.inv_mw + k) * iS;
            if (warp == 0) {
                gT[i] = tb - rho * pt.invT;
                if (gP) gP[i] = fma(rho, 1.0 / Pv, pb);
            }
        }
        __syncthreads();                     // the tile's state stays until every warp is done
    }
}

}  // namespace

// Row-owner Jacobian plan: per-species (reaction, net nu) lists.
struct JacPlan {
    int warps = 0;
    size_t smem = 0;
    int grid = 0;
    const int* lptr = nullptr;
    const int* lrx = nullptr;
    const double* lnu = nullptr;
    const int* lrow = nullptr;  // species of row slot t (warp t % warps)
    void* dbuf = nullptr;
};

cudaError_t jac_prepare(const DevMech& m, const cg_mech_view& v, int device, JacPlan** out) {
    *out = nullptr;
    const int ns = m.ns, nr = m.nr;
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    const size_t fixed = (size_t)3 * ns * kJTile * 8 + (size_t)kJMaxWarps * kJTile * 8;
    const size_t per_warp = (size_t)(ns + 1) * kJTile * 8;
    if (fixed + 2 * per_warp > prop.sharedMemPerBlockOptin) return cudaErrorNotSupported;
    const int warps = (int)std::min<size_t>(kJMaxWarps, (prop.sharedMemPerBlockOptin - fixed) / per_warp);
    const int32_t* rp = (const int32_t*)v.a[CG_RPTR];
    const int32_t* pp = (const int32_t*)v.a[CG_PPTR];
    const int32_t* rsp = (const int32_t*)v.a[CG_RSP];
    const int32_t* psp = (const int32_t*)v.a[CG_PSP];
    const double* rnu = (const double*)v.a[CG_RNU];
    const double* pnu = (const double*)v.a[CG_PNU];
    std::vector<std::vector<std::pair<int, double>>> lists(ns);
    std::vector<double> net(ns, 0.0);
    for (int r = 0; r < nr; ++r) {
        for (int j = rp[r]; j < rp[r + 1]; ++j) net[rsp[j]] -= rnu[j];
        for (int j = pp[r]; j < pp[r + 1]; ++j) net[psp[j]] += pnu[j];
        for (int j = rp[r]; j < rp[r + 1]; ++j)
            if (net[rsp[j]] != 0.0) {
                lists[rsp[j]].push_back({r, net[rsp[j]]});
                net[rsp[j]] = 0.0;
            }
        for (int j = pp[r]; j < pp[r + 1]; ++j)
            if (net[psp[j]] != 0.0) {
                lists[psp[j]].push_back({r, net[psp[j]]});
                net[psp[j]] = 0.0;
            }
    }
    std::vector<int> lptr(ns + 1, 0), lrx;
    std::vector<double> lnu;
    for (int k = 0; k < ns; ++k) {
        for (const auto& x : lists[k]) {
            lrx.push_back(x.first);
            lnu.push_back(x.second);
        }
        lptr[k + 1] = (int)lrx.size();
    }
    // row slots: warp w takes slots w, w + warps, ...; species dealt out
    // longest list first, each to the warp with the least work so far among
    // those with a free slot (a row costs its list plus the chain rule)
    std::vector<int> order(ns);
    for (int k = 0; k < ns; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return lists[a].size() > lists[b].size(); });
    std::vector<std::vector<int>> warp_rows(warps);
    std::vector<long> load(warps, 0);
    for (int k : order) {
        int best = -1;
        for (int w = 0; w < warps; ++w) {
            const int cap = (ns - w + warps - 1) / warps;
            if ((int)warp_rows[w].size() < cap && (best < 0 || load[w] < load[best])) best = w;
        }
        warp_rows[best].push_back(k);
        load[best] += (long)lists[k].size() + ns;
    }
    std::vector<int> lrow(ns);
    for (int w = 0; w < warps; ++w)
        for (size_t j = 0; j < warp_rows[w].size(); ++j) lrow[j * warps + w] = warp_rows[w][j];
    const size_t b_ptr = ((ns + 1) * sizeof(int) + 255) / 256 * 256;
    const size_t b_rx = (std::max<size_t>(lrx.size(), 1) * sizeof(int) + 255) / 256 * 256;
    const size_t b_nu = (std::max<size_t>(lnu.size(), 1) * sizeof(double) + 255) / 256 * 256;
    const size_t b_row = (size_t)ns * sizeof(int);
    JacPlan* p = new JacPlan();
    p->warps = warps;
    p->smem = fixed + (size_t)warps * per_warp;
    p->grid = prop.multiProcessorCount;
    e = cudaMalloc(&p->dbuf, b_ptr + b_rx + b_nu + b_row);
    char* d = (char*)p->dbuf;
    if (e == cudaSuccess) e = cudaMemcpy(d, lptr.data(), lptr.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !lrx.empty()) e = cudaMemcpy(d + b_ptr, lrx.data(), lrx.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !lnu.empty())
        e = cudaMemcpy(d + b_ptr + b_rx, lnu.data(), lnu.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d + b_ptr + b_rx + b_nu, lrow.data(), b_row, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(jac_rows_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(jac_rows_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem);
    if (e != cudaSuccess) {
        if (p->dbuf) cudaFree(p->dbuf);
        delete p;
        return e;
    }
    p->lptr = (const int*)d;
    p->lrx = (const int*)(d + b_ptr);
    p->lnu = (const double*)(d + b_ptr + b_rx);
    p->lrow = (const int*)(d + b_ptr + b_rx + b_nu);
    *out = p;
    return cudaSuccess;
}

void jac_release(JacPlan* p) {
    if (!p) return;
    if (p->dbuf) cudaFree(p->dbuf);
    delete p;
}

size_t jac_rows_workspace_bytes(const JacPlan* p, const DevMech& m, int64_t ng) {
    const int64_t tiles = (ng + kJTile - 1) / kJTile;
    const int64_t grid = std::min<int64_t>(tiles, p->grid);
    return (size_t)grid * m.nr * kDC * kJTile * sizeof(double);
}

cudaError_t launch_jacobian_rows(const JacPlan* p, const DevMech& m, int precision, const double* P, const double* T,
                                 const double* Y, void* J, int64_t ng, double* scratch, size_t scratch_bytes,
                                 cudaStream_t s) {
    if (ng <= 0) return cudaSuccess;
    const int64_t tiles = (ng + kJTile - 1) / kJTile;
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, p->grid);
    if (!scratch || scratch_bytes < jac_rows_workspace_bytes(p, m, ng)) return cudaErrorInvalidValue;
    const unsigned threads = 32u * (unsigned)p->warps;
    // the kernel's shared-memory limit is this plan's, set under one lock with
    // the launch (a plan made later for a smaller mechanism sets it lower)
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    cudaError_t e = precision == 0 ? cudaFuncSetAttribute(jac_rows_kernel<double>,
                                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem)
                                   : cudaFuncSetAttribute(jac_rows_kernel<float>,
                                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem);
    if (e != cudaSuccess) return e;
    if (precision == 0)
        jac_rows_kernel<double><<<grid, threads, p->smem, s>>>(m, p->lptr, p->lrx, p->lnu, p->lrow, P, T, Y,
                                                               (double*)J, ng, scratch);
    else
        jac_rows_kernel<float><<<grid, threads, p->smem, s>>>(m, p->lptr, p->lrx, p->lnu, p->lrow, P, T, Y,
                                                              (float*)J, ng, scratch);
    return cudaGetLastError();
}

size_t deriv_workspace_bytes(int ns, int64_t ng) { return (size_t)4 * ns * ng * sizeof(double); }

cudaError_t launch_jacobian(const DevMech& m, int precision, const double* P, const double* T, const double* Y,
                            void* J, int64_t ng, double* scratch, int sm_count, cudaStream_t s) {
    if (ng <= 0) return cudaSuccess;
    int64_t blocks = (ng + 127) / 128;
    if (blocks > (int64_t)sm_count * 16) blocks = (int64_t)sm_count * 16;
    if (precision == 0)
        deriv_kernel<true, double><<<(unsigned)blocks, 128, 0, s>>>(m, P, T, Y, nullptr, (double*)J, nullptr, nullptr,
                                                                   nullptr, scratch, ng);
    else
        deriv_kernel<true, float><<<(unsigned)blocks, 128, 0, s>>>(m, P, T, Y, nullptr, (float*)J, nullptr, nullptr,
                                                                  nullptr, scratch, ng);
    return cudaGetLastError();
}

// Warps per CTA of the tile VJP kernel for ns species (its shared memory
// holds 4 + W arrays of [ns][32] doubles), or 0 when fewer than 4 fit.
int vjp_tile_warps(int ns, size_t smem_optin) {
    const size_t arr = (size_t)ns * kJTile * 8, fixed = 4 * arr + (size_t)3 * kVMaxWarps * kJTile * 8;
    if (fixed + 4 * arr > smem_optin) return 0;
    const size_t w = (smem_optin - fixed) / arr;
    return (int)std::min<size_t>(w, kVMaxWarps);
}

cudaError_t launch_vjp(const DevMech& m, const double* P, const double* T, const double* Y, const double* G, double* gT,
                       double* gY, double* gP, int64_t ng, double* scratch, int sm_count, cudaStream_t s) {
    if (ng <= 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    int optin = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const int w = vjp_tile_warps(m.ns, (size_t)optin);
    if (w >= 4) {
        const size_t smem = (size_t)(4 + w) * m.ns * kJTile * 8 + (size_t)3 * kVMaxWarps * kJTile * 8;
        static std::mutex mu;
        std::lock_guard<std::mutex> lk(mu);
        e = cudaFuncSetAttribute(vjp_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int64_t tiles = (ng + kJTile - 1) / kJTile;
        const unsigned grid = (unsigned)std::min<int64_t>(tiles, sm_count);
        vjp_tile_kernel<<<grid, 32u * (unsigned)w, smem, s>>>(m, P, T, Y, G, gT, gY, gP, ng);
        return cudaGetLastError();
    }
    int64_t blocks = (ng + 127) / 128;
    if (blocks > (int64_t)sm_count * 16) blocks = (int64_t)sm_count * 16;
    deriv_kernel<false, double><<<(unsigned)blocks, 128, 0, s>>>(m, P, T, Y, G, nullptr, gT, gY, gP, scratch, ng);
    return cudaGetLastError();
}

}  // namespace cg
