/*
 * Packed mechanism tables ("mechanism blob"): the one input format shared by
 * the CUDA library (chemgen_create) and every host tool.
 *
 * The reference spreads these constants over generated Fortran modules and
 * HIP __constant__ symbols (chemgen/write_constants.py:14-347,
 * chemgen/constants.py:53-240); here they travel as one relocatable blob
 * written by chemgen_b200/pack.py.
 *
 * Layout: "CGB200M1" magic, CG_NSCALARS int64 scalars, then CG_NARRAYS
 * (offset, count) int64 pairs, then the arrays (64-byte aligned).  Reactions
 * are stored in kernel order: grouped by kind (standard, third_body,
 * lindemann, troe, sri, plog), file order within a kind; CG_ORIG maps a kernel
 * index back to the file index.
 */
#ifndef CHEMGEN_MECH_H
#define CHEMGEN_MECH_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define CG_MAGIC "CGB200M1"
#define CG_VERSION 1

enum cg_kind { CG_STANDARD = 0, CG_THIRD_BODY, CG_LINDEMANN, CG_TROE, CG_SRI, CG_PLOG, CG_NKINDS };

/* reaction flag bits */
#define CG_F_REVERSIBLE 1     /* kb from Kc; otherwise kb = 0 */
#define CG_F_INT_NU     2     /* every stoichiometric coefficient is 1, 2 or 3 */
#define CG_F_TROE_T2    4     /* Troe with the exp(-T2/T) term */
#define CG_F_A_NEG      8     /* negative pre-exponential factor */
#define CG_F_LOW_NEG   16     /* negative low-pressure pre-exponential factor */

enum cg_scalar {
    CG_S_VERSION = 0, CG_S_NS, CG_S_NR,
    CG_S_NSTD, CG_S_N3B, CG_S_NLIND, CG_S_NTROE, CG_S_NSRI, CG_S_NPLOG,
    CG_S_NEFF, CG_S_NPLEV, CG_S_NPTERM, CG_S_FLAGS, CG_S_MAXNU_INT,
    CG_S_NRT, CG_S_NPT,          /* reactant / product entries (CSR lengths) */
    CG_NSCALARS
};

enum cg_array {
    /* species (ns) */
    CG_MW = 0,          /* double[ns] g/mol */
    CG_INV_MW,          /* double[ns] */
    CG_TMID,            /* double[ns] K */
    CG_SMH_LO,          /* double[ns*7] c0..c6: smh = c0 + c1 lnT + c2 T + c3 T^2 + c4 T^3 + c5 T^4 - c6/T, T < Tmid */
    CG_SMH_HI,          /* double[ns*7] same, T >= Tmid */
    CG_NASA_LO,         /* double[ns*7] raw a1..a7 */
    CG_NASA_HI,         /* double[ns*7] */
    /* reactions (nr, kernel order) */
    CG_ORIG,            /* int32[nr]  file index */
    CG_FLAGS,           /* int32[nr]  CG_F_* */
    CG_RPTR,            /* int32[nr+1] CSR into the reactant entries */
    CG_PPTR,            /* int32[nr+1] CSR into the product entries */
    CG_RSP,             /* int32[nrt]  reactant species */
    CG_PSP,             /* int32[npt]  product species */
    CG_RNU,             /* double[nrt] reactant coefficients */
    CG_PNU,             /* double[npt] product coefficients */
    CG_DNU,             /* double[nr] sum(nu_p) - sum(nu_r) */
    CG_ARH,             /* double[nr*3] A (cgs), b, Ea (cal/mol); kinf for falloff; unused for plog */
    CG_KARH,            /* double[nr*4] ln|A|, b, Ea/Rc (K), sign(A) */
    CG_EFF_PTR,         /* int32[nr+1] CSR over kernel order */
    CG_EFF_SP,          /* int32[neff] */
    CG_EFF_VAL,         /* double[neff] efficiency - 1 */
    CG_FALL,            /* double[nfall*8] per falloff reaction: A0, b0, Ea0, p0..p4 (Troe a,T3,T1,T2 | SRI a,b,c,d,e) */
    CG_KFALL,           /* double[nfall*4] ln|A0|, b0, Ea0/Rc, sign(A0) */
    CG_PLOG_PTR,        /* int32[nplog+1] into pressure levels */
    CG_PLOG_P,          /* double[nlev] pressure, dyne/cm^2, ascending within a reaction */
    CG_PLOG_LNP,        /* double[nlev] ln(pressure) */
    CG_PLOG_TPTR,       /* int32[nlev+1] into terms */
    CG_PLOG_TERM,       /* double[nterm*3] A, b, Ea */
    CG_KPLOG_TERM,      /* double[nterm*4] ln|A|, b, Ea/Rc, sign(A) */
    CG_NARRAYS
};

typedef struct cg_mech_view {
    int64_t s[CG_NSCALARS];
    const void* a[CG_NARRAYS];
    int64_t count[CG_NARRAYS];
    size_t nbytes;
} cg_mech_view;

/* first kernel index of each kind */
static inline int64_t cg_kind_begin(const cg_mech_view* v, int kind) {
    int64_t o = 0;
    for (int k = 0; k < kind; ++k) o += v->s[CG_S_NSTD + k];
    return o;
}

static inline size_t cg_elem_size(int array) {
    switch (array) {
    case CG_ORIG: case CG_FLAGS: case CG_RPTR: case CG_PPTR: case CG_RSP: case CG_PSP:
    case CG_EFF_PTR: case CG_EFF_SP: case CG_PLOG_PTR: case CG_PLOG_TPTR:
        return 4;
    default:
        return 8;
    }
}

/* Parse a blob; returns 0 on success, a negative code on a malformed blob. */
static inline int cg_mech_parse(const void* blob, size_t n, cg_mech_view* v) {
    const unsigned char* p = (const unsigned char*)blob;
    size_t head = 8 + 8 * (size_t)CG_NSCALARS + 16 * (size_t)CG_NARRAYS;
    if (!blob || n < head) return -1;
    if (memcmp(p, CG_MAGIC, 8) != 0) return -2;
    memcpy(v->s, p + 8, 8 * (size_t)CG_NSCALARS);
    if (v->s[CG_S_VERSION] != CG_VERSION) return -3;
    const unsigned char* tab = p + 8 + 8 * (size_t)CG_NSCALARS;
    for (int i = 0; i < CG_NARRAYS; ++i) {
        int64_t off, cnt;
        memcpy(&off, tab + 16 * (size_t)i, 8);
        memcpy(&cnt, tab + 16 * (size_t)i + 8, 8);
        if (off < (int64_t)head || cnt < 0 || (size_t)off > n) return -4;
        if ((size_t)off + (size_t)cnt * cg_elem_size(i) > n) return -4;
        if (off % 8) return -5;
        v->a[i] = p + off;
        v->count[i] = cnt;
    }
    int64_t ns = v->s[CG_S_NS], nr = v->s[CG_S_NR];
    if (ns <= 0 || nr < 0) return -6;
    int64_t sum = 0;
    for (int k = 0; k < CG_NKINDS; ++k) sum += v->s[CG_S_NSTD + k];
    if (sum != nr) return -7;
    if (v->count[CG_MW] != ns || v->count[CG_SMH_LO] != 7 * ns || v->count[CG_ORIG] != nr ||
        v->count[CG_RPTR] != nr + 1 || v->count[CG_PPTR] != nr + 1 || v->count[CG_EFF_PTR] != nr + 1)
        return -8;
    v->nbytes = n;
    /* every index a kernel will use must stay in range */
    const int32_t* rp = (const int32_t*)v->a[CG_RPTR];
    const int32_t* pq = (const int32_t*)v->a[CG_PPTR];
    const int32_t* rsp = (const int32_t*)v->a[CG_RSP];
    const int32_t* psp = (const int32_t*)v->a[CG_PSP];
    const int32_t* ep = (const int32_t*)v->a[CG_EFF_PTR];
    const int32_t* es = (const int32_t*)v->a[CG_EFF_SP];
    int64_t neff = v->s[CG_S_NEFF], nrt = v->s[CG_S_NRT], npt = v->s[CG_S_NPT];
    if (v->count[CG_EFF_SP] != neff || v->count[CG_RSP] != nrt || v->count[CG_PSP] != npt ||
        v->count[CG_RNU] != nrt || v->count[CG_PNU] != npt)
        return -9;
    if (rp[0] != 0 || pq[0] != 0 || rp[nr] != nrt || pq[nr] != npt) return -10;
    for (int64_t r = 0; r < nr; ++r) {
        if (rp[r + 1] <= rp[r] || pq[r + 1] <= pq[r]) return -10;
        if (ep[r] < 0 || ep[r + 1] < ep[r] || ep[r + 1] > neff) return -12;
    }
    for (int64_t j = 0; j < nrt; ++j)
        if (rsp[j] < 0 || rsp[j] >= ns) return -11;
    for (int64_t j = 0; j < npt; ++j)
        if (psp[j] < 0 || psp[j] >= ns) return -11;
    if (ep[0] != 0) return -12;
    for (int64_t e = 0; e < neff; ++e)
        if (es[e] < 0 || es[e] >= ns) return -13;
    int64_t nfall = v->s[CG_S_NLIND] + v->s[CG_S_NTROE] + v->s[CG_S_NSRI];
    if (v->count[CG_FALL] != 8 * nfall || v->count[CG_KFALL] != 4 * nfall) return -14;
    int64_t nplog = v->s[CG_S_NPLOG], nlev = v->s[CG_S_NPLEV], nterm = v->s[CG_S_NPTERM];
    const int32_t* pp = (const int32_t*)v->a[CG_PLOG_PTR];
    const int32_t* tp = (const int32_t*)v->a[CG_PLOG_TPTR];
    if (v->count[CG_PLOG_PTR] != nplog + 1 || v->count[CG_PLOG_TPTR] != nlev + 1 ||
        v->count[CG_PLOG_P] != nlev || v->count[CG_KPLOG_TERM] != 4 * nterm)
        return -15;
    if (pp[0] != 0 || pp[nplog] != nlev || tp[0] != 0 || tp[nlev] != nterm) return -15;
    for (int64_t i = 0; i < nplog; ++i)
        if (pp[i + 1] <= pp[i]) return -15;
    for (int64_t i = 0; i < nlev; ++i)
        if (tp[i + 1] <= tp[i]) return -15;
    return 0;
}

#endif /* CHEMGEN_MECH_H */
