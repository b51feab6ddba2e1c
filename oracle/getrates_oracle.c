/*
 * ORACLE -- test infrastructure only.  A plain-C FP64 restatement of the
 * getrates that the reference generates (chemgen/templates/python_header.j2,
 * ytoc.j2, exp_g.j2, reactions/{standard,third_body,troe,plog}.j2).  It is
 * the checker for the CUDA library and the timed CPU baseline of bench.py;
 * nothing in the product links or calls it.
 *
 * Every expression keeps the reference's operand order (Python evaluates left
 * to right), reactions are applied in file order, and the constants come from
 * the same packed blob the CUDA library reads (include/chemgen_mech.h), which
 * rounds them exactly as the reference prints them ("%.15e").
 *
 * Lindemann and SRI falloff are not expressible by the reference (its parser
 * drops them, chemgen/parser.py:146-147); they follow the Troe template
 * (reactions/troe.j2) with F = 1 and with the Chemkin SRI form
 * F = d [a exp(-b/T) + exp(-T/c)]^X T^e, X = 1/(1 + log10(Pr)^2).
 *
 * Layouts: Y and wdot are species-major, Y[k*ng + i] (the reference's GPU
 * layout, chemgen/templates/reactions_hip/device_functions_h.j2:701-719).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/chemgen_mech.h"

/* chemgen/chemistry.py:204-206 */
static const double RC = 1.9872155832;
static const double R0 = 8.314510e+07;
static const double PATM = 1013250.0;

typedef struct {
    cg_mech_view v;
    int64_t* kidx;        /* file index -> kernel index */
    int64_t* fidx;        /* kernel index -> falloff row, or -1 */
    int64_t* pidx;        /* kernel index -> plog row, or -1 */
    int has_m;
} oracle_mech;

static int oracle_open(const void* blob, size_t n, oracle_mech* m) {
    memset(m, 0, sizeof(*m));
    int rc = cg_mech_parse(blob, n, &m->v);
    if (rc) return rc;
    int64_t nr = m->v.s[CG_S_NR];
    m->kidx = (int64_t*)malloc(sizeof(int64_t) * (nr + 1));
    m->fidx = (int64_t*)malloc(sizeof(int64_t) * (nr + 1));
    m->pidx = (int64_t*)malloc(sizeof(int64_t) * (nr + 1));
    const int32_t* orig = (const int32_t*)m->v.a[CG_ORIG];
    int64_t f0 = cg_kind_begin(&m->v, CG_LINDEMANN), f1 = cg_kind_begin(&m->v, CG_PLOG);
    for (int64_t k = 0; k < nr; ++k) {
        m->kidx[orig[k]] = k;
        m->fidx[k] = (k >= f0 && k < f1) ? k - f0 : -1;
        m->pidx[k] = (k >= f1) ? k - f1 : -1;
    }
    m->has_m = (m->v.s[CG_S_N3B] + m->v.s[CG_S_NLIND] + m->v.s[CG_S_NTROE] + m->v.s[CG_S_NSRI]) > 0;
    return 0;
}

static void oracle_close(oracle_mech* m) {
    free(m->kidx);
    free(m->fidx);
    free(m->pidx);
}

static inline int kind_of(const cg_mech_view* v, int64_t k) {
    int64_t o = 0;
    for (int kind = 0; kind < CG_NKINDS; ++kind) {
        o += v->s[CG_S_NSTD + kind];
        if (k < o) return kind;
    }
    return -1;
}

/* A * T**b * exp(-Ea/(Rc*T)) -- reactions/standard.j2:4 (b == 0 drops T**b) */
static inline double arrhenius(double A, double b, double Ea, double T) {
    double k = A;
    if (b != 0.0) k = k * pow(T, b);
    return k * exp((-1.0 * Ea) / (RC * T));
}

/* One point.  C and EG are scratch of length ns.  Optional per-reaction
 * outputs (file order): kf, kb, qf (kf*prod C_r [*M]), qb. */
static void point(const oracle_mech* m, double P, double T, const double* Y, int64_t ystride,
                  double* wdot, int64_t wstride, double* C, double* EG,
                  double* kf_out, double* kb_out, double* qf_out, double* qb_out) {
    const cg_mech_view* v = &m->v;
    const int64_t ns = v->s[CG_S_NS], nr = v->s[CG_S_NR];
    const double* mw = (const double*)v->a[CG_MW];
    const double* tmid = (const double*)v->a[CG_TMID];
    const double* lo = (const double*)v->a[CG_SMH_LO];
    const double* hi = (const double*)v->a[CG_SMH_HI];
    const int32_t* flags = (const int32_t*)v->a[CG_FLAGS];
    const int32_t* rp = (const int32_t*)v->a[CG_RPTR];
    const int32_t* pq = (const int32_t*)v->a[CG_PPTR];
    const int32_t* rsp = (const int32_t*)v->a[CG_RSP];
    const int32_t* psp = (const int32_t*)v->a[CG_PSP];
    const double* rnu = (const double*)v->a[CG_RNU];
    const double* pnu = (const double*)v->a[CG_PNU];
    const double* dnu = (const double*)v->a[CG_DNU];
    const double* arh = (const double*)v->a[CG_ARH];
    const int32_t* ep = (const int32_t*)v->a[CG_EFF_PTR];
    const int32_t* es = (const int32_t*)v->a[CG_EFF_SP];
    const double* ev = (const double*)v->a[CG_EFF_VAL];
    const double* fall = (const double*)v->a[CG_FALL];
    const int32_t* pp = (const int32_t*)v->a[CG_PLOG_PTR];
    const double* plp = (const double*)v->a[CG_PLOG_P];
    const double* pllnp = (const double*)v->a[CG_PLOG_LNP];
    const int32_t* ptp = (const int32_t*)v->a[CG_PLOG_TPTR];
    const double* pterm = (const double*)v->a[CG_PLOG_TERM];

    for (int64_t k = 0; k < ns; ++k) wdot[k * wstride] = 0.0;
    /* python_header.j2:56 */
    const double pfac = PATM / (R0 * T);
    /* ytoc.j2:3-18 */
    for (int64_t k = 0; k < ns; ++k) C[k] = Y[k * ystride] / mw[k];
    double ctot = 0.0;
    for (int64_t k = 0; k < ns; ++k) ctot = ctot + C[k];
    for (int64_t k = 0; k < ns; ++k) C[k] = C[k] * P / (R0 * ctot * T);
    if (m->has_m) {
        ctot = 0.0;
        for (int64_t k = 0; k < ns; ++k) ctot = ctot + C[k];
    }
    /* exp_g.j2:2-27 */
    const double lnT = log(T);
    for (int64_t k = 0; k < ns; ++k) {
        const double* c = (T < tmid[k]) ? lo + 7 * k : hi + 7 * k;
        double smh = c[0] + c[1] * lnT + c[2] * T + c[3] * pow(T, 2.0) + c[4] * pow(T, 3.0) +
                     c[5] * pow(T, 4.0) - c[6] / T;
        EG[k] = exp(smh);
    }
    for (int64_t f = 0; f < nr; ++f) {
        const int64_t r = m->kidx[f];
        const int kind = kind_of(v, r);
        const int32_t fl = flags[r];
        double kf = 0.0, M = 1.0;
        if (kind != CG_STANDARD && kind != CG_PLOG) {
            /* third_body.j2:18-28, troe.j2:10-18 */
            M = ctot;
            for (int32_t e = ep[r]; e < ep[r + 1]; ++e) M = M + ev[e] * C[es[e]];
        }
        if (kind == CG_STANDARD || kind == CG_THIRD_BODY) {
            kf = arrhenius(arh[3 * r], arh[3 * r + 1], arh[3 * r + 2], T);
        } else if (kind == CG_PLOG) {
            /* plog.j2:4-38 */
            const int64_t pr = m->pidx[r];
            const int32_t l0 = pp[pr], l1 = pp[pr + 1];
            int32_t la, lb;
            double logPl, logPh;
            int32_t l = l0;
            while (l < l1 && !(P < plp[l])) ++l;
            if (l == l0) {
                la = lb = l0; logPl = 1.0e0; logPh = pllnp[l0];
            } else if (l == l1) {
                la = lb = l1 - 1; logPl = pllnp[l1 - 1]; logPh = 100.0e0;
            } else {
                la = l - 1; lb = l; logPl = pllnp[l - 1]; logPh = pllnp[l];
            }
            double kfl = 0.0, kfh = 0.0;
            for (int32_t t = ptp[la]; t < ptp[la + 1]; ++t)
                kfl = kfl + (pterm[3 * t] * pow(T, pterm[3 * t + 1]) * exp((-1.0 * pterm[3 * t + 2]) / (RC * T)));
            if (lb == la) kfh = kfl;
            else
                for (int32_t t = ptp[lb]; t < ptp[lb + 1]; ++t)
                    kfh = kfh + (pterm[3 * t] * pow(T, pterm[3 * t + 1]) * exp((-1.0 * pterm[3 * t + 2]) / (RC * T)));
            kf = exp(log(kfl) + (log(kfh) - log(kfl)) * (log(P) - logPl) / (logPh - logPl));
        } else {
            /* troe.j2:21-45 */
            const double* fr = fall + 8 * m->fidx[r];
            double k0 = arrhenius(fr[0], fr[1], fr[2], T);
            double kinf = arrhenius(arh[3 * r], arh[3 * r + 1], arh[3 * r + 2], T);
            double Pr = (k0 * M) / kinf;
            double F = 1.0;
            if (kind == CG_TROE) {
                double Fcent = fr[7] * exp(-T / fr[4]) + fr[3] * exp(-T / fr[5]);
                if (fl & CG_F_TROE_T2) Fcent = Fcent + exp((-fr[6]) / T);
                double C1 = -0.4 - 0.67 * log10(Fcent);
                double N1 = 0.75 - 1.27 * log10(Fcent);
                double f1 = (log10(Pr) + C1) / (N1 - 0.14 * (log10(Pr) + C1));
                F = pow(10.0, log10(Fcent) / (1.0 + pow(f1, 2.0)));
            } else if (kind == CG_SRI) {
                double X = 1.0 / (1.0 + pow(log10(Pr), 2.0));
                F = fr[6] * pow(fr[3] * exp(-fr[4] / T) + exp(-T / fr[5]), X) * pow(T, fr[7]);
            }
            kf = kinf * (Pr / (1.0 + Pr)) * F;
            M = 1.0;       /* falloff: M only enters through Pr */
        }
        /* standard.j2:7-16 */
        double kb = 0.0;
        if (fl & CG_F_REVERSIBLE) {
            kb = kf;
            for (int32_t j = rp[r]; j < rp[r + 1]; ++j) {
                double nu = rnu[j];
                double e = EG[rsp[j]];
                kb = kb * (nu != 1.0 ? pow(e, nu) : e);
            }
            for (int32_t j = pq[r]; j < pq[r + 1]; ++j) {
                double nu = pnu[j];
                double e = EG[psp[j]];
                kb = kb / (nu != 1.0 ? pow(e, nu) : e);
            }
            if (dnu[r] != 0.0) kb = kb / pow(pfac, dnu[r]);
        }
        /* standard.j2:18-19 */
        double qf = kf, qb = kb;
        for (int32_t j = rp[r]; j < rp[r + 1]; ++j) {
            double nu = rnu[j];
            double c = C[rsp[j]];
            qf = qf * (nu != 1.0 ? pow(c, nu) : c);
        }
        for (int32_t j = pq[r]; j < pq[r + 1]; ++j) {
            double nu = pnu[j];
            double c = C[psp[j]];
            qb = qb * (nu != 1.0 ? pow(c, nu) : c);
        }
        double rr = (kind == CG_THIRD_BODY) ? M * (qf - qb) : qf - qb;
        if (kf_out) {
            kf_out[f] = kf;
            kb_out[f] = kb;
            qf_out[f] = (kind == CG_THIRD_BODY) ? M * qf : qf;
            qb_out[f] = (kind == CG_THIRD_BODY) ? M * qb : qb;
        }
        /* standard.j2:21-27 */
        for (int32_t j = rp[r]; j < rp[r + 1]; ++j) {
            double nu = rnu[j];
            int32_t s = rsp[j];
            wdot[s * wstride] = wdot[s * wstride] - (nu != 1.0 ? rr * nu : rr);
        }
        for (int32_t j = pq[r]; j < pq[r + 1]; ++j) {
            double nu = pnu[j];
            int32_t s = psp[j];
            wdot[s * wstride] = wdot[s * wstride] + (nu != 1.0 ? rr * nu : rr);
        }
    }
}

/* wdot[ns*ng] for ng points, species-major.  Returns 0 or a blob error. */
int oracle_getrates(const void* blob, size_t nbytes, int64_t ng, const double* P, const double* T,
                    const double* Y, double* wdot, int nthreads) {
    oracle_mech m;
    int rc = oracle_open(blob, nbytes, &m);
    if (rc) return rc;
    const int64_t ns = m.v.s[CG_S_NS];
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
    {
        double* C = (double*)malloc(sizeof(double) * ns);
        double* EG = (double*)malloc(sizeof(double) * ns);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t i = 0; i < ng; ++i) point(&m, P[i], T[i], Y + i, ng, wdot + i, ng, C, EG, 0, 0, 0, 0);
        free(C);
        free(EG);
    }
    (void)nthreads;
    oracle_close(&m);
    return 0;
}

/* Per-reaction diagnostics for ng points: kf, kb, qf, qb as [nr*ng]
 * reaction-major (file order), plus the gross rate S[k*ng+i] =
 * sum_r |nu_kr| (|qf_r| + |qb_r|), the scale against which cancellation-robust
 * errors are measured.  Any output pointer may be NULL. */
int oracle_rates(const void* blob, size_t nbytes, int64_t ng, const double* P, const double* T,
                 const double* Y, double* wdot, double* kf, double* kb, double* qf, double* qb,
                 double* S, int nthreads) {
    oracle_mech m;
    int rc = oracle_open(blob, nbytes, &m);
    if (rc) return rc;
    const cg_mech_view* v = &m.v;
    const int64_t ns = v->s[CG_S_NS], nr = v->s[CG_S_NR];
    const int32_t* rp = (const int32_t*)v->a[CG_RPTR];
    const int32_t* pq = (const int32_t*)v->a[CG_PPTR];
    const int32_t* rsp = (const int32_t*)v->a[CG_RSP];
    const int32_t* psp = (const int32_t*)v->a[CG_PSP];
    const double* rnu = (const double*)v->a[CG_RNU];
    const double* pnu = (const double*)v->a[CG_PNU];
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
    {
        double* C = (double*)malloc(sizeof(double) * ns);
        double* EG = (double*)malloc(sizeof(double) * ns);
        double* w = (double*)malloc(sizeof(double) * ns);
        double* a = (double*)malloc(sizeof(double) * 4 * nr);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t i = 0; i < ng; ++i) {
            point(&m, P[i], T[i], Y + i, ng, w, 1, C, EG, a, a + nr, a + 2 * nr, a + 3 * nr);
            for (int64_t k = 0; k < ns; ++k) {
                if (wdot) wdot[k * ng + i] = w[k];
                if (S) S[k * ng + i] = 0.0;
            }
            for (int64_t f = 0; f < nr; ++f) {
                if (kf) kf[f * ng + i] = a[f];
                if (kb) kb[f * ng + i] = a[nr + f];
                if (qf) qf[f * ng + i] = a[2 * nr + f];
                if (qb) qb[f * ng + i] = a[3 * nr + f];
                if (S) {
                    int64_t r = m.kidx[f];
                    double g = fabs(a[2 * nr + f]) + fabs(a[3 * nr + f]);
                    for (int32_t j = rp[r]; j < rp[r + 1]; ++j) S[rsp[j] * ng + i] += rnu[j] * g;
                    for (int32_t j = pq[r]; j < pq[r + 1]; ++j) S[psp[j] * ng + i] += pnu[j] * g;
                }
            }
        }
        free(C);
        free(EG);
        free(w);
        free(a);
    }
    (void)nthreads;
    oracle_close(&m);
    return 0;
}

/* Parse check used by tests: returns cg_mech_parse's code. */
int oracle_check_blob(const void* blob, size_t nbytes) {
    cg_mech_view v;
    return cg_mech_parse(blob, nbytes, &v);
}
