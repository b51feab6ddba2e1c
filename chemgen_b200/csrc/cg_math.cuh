// FP64 exp and log used by the getrates kernels, written from textbook methods
// so that they are branch-free and cheap in issue slots:
//
// cg_exp(x): Cody-Waite argument reduction x = k ln2 + r, |r| <= ln2/2, with
//   ln2 split into a 32-bit head (k * head is exact for |k| < 2^20) and a
//   tail; e^r from its Taylor series to degree 12 (truncation error
//   < |r|^13/13! < 2e-16 relative); 2^k applied through the exponent field.
//   Valid for |x| < 708.  cg_exp_clamped clamps x to [-746, 710] first.  At
//   the ends 2^k is built from a biased exponent clamped to [0, 2047], so
//   x <= -1022.5 ln2 (about -708.75, results below 2^-1022.5) flushes to zero,
//   and x >= 1023.5 ln2 (about 709.44, results above 2^1023.5 = 1.3e308)
//   gives +inf although e^x stays finite up to x = 709.78: the kernels treat
//   rates that large as an overflow.
// cg_log(x): x = 2^e m with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
//   s = (m-1)/(m+1), |s| <= 0.1716, from the odd series of atanh to s^21
//   (truncation < 3e-17); ln x = e ln2 + ln m.  Non-positive, infinite and
//   subnormal inputs fall back to the library log.
// The coefficients are the exact series terms 1/n! and 1/(2n+1).
#pragma once

namespace cgm {

constexpr double kLn2Hi = 0.6931471803691238;      // ln 2 rounded to 32 significant bits
constexpr double kLn2Lo = 1.9082149292705877e-10;   // ln 2 - kLn2Hi
constexpr double kLog2e = 1.4426950408889634;
constexpr double kRound = 6755399441055744.0;       // 1.5 * 2^52

__device__ __forceinline__ double cg_exp(double x) {
    const double t = fma(x, kLog2e, kRound);
    const double k = t - kRound;
    double r = fma(k, -kLn2Hi, x);
    r = fma(k, -kLn2Lo, r);
    double p = 2.08767569878681e-09;                 // 1/12!
    p = fma(p, r, 2.505210838544172e-08);            // 1/11!
    p = fma(p, r, 2.755731922398589e-07);            // 1/10!
    p = fma(p, r, 2.7557319223985893e-06);           // 1/9!
    p = fma(p, r, 2.48015873015873e-05);             // 1/8!
    p = fma(p, r, 0.0001984126984126984);            // 1/7!
    p = fma(p, r, 0.001388888888888889);             // 1/6!
    p = fma(p, r, 0.008333333333333333);             // 1/5!
    p = fma(p, r, 0.041666666666666664);             // 1/4!
    p = fma(p, r, 0.16666666666666666);              // 1/3!
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    int e = __double2loint(t) + 1023;                // biased exponent of 2^k
    e = max(0, min(e, 2047));
    const double s = __hiloint2double(e << 20, 0);   // 2^k, 0 or +inf at the ends
    return p * s;
}

__device__ __forceinline__ double cg_exp_clamped(double x) { return cg_exp(fmin(fmax(x, -746.0), 710.0)); }

// Out-of-line copies, for straight-line kernels whose code size (instruction
// fetch) matters more than a call per use.
static __device__ __noinline__ double cg_exp_ool(double x) { return cg_exp(x); }
static __device__ __noinline__ double cg_exp_clamped_ool(double x) { return cg_exp_clamped(x); }

__device__ __forceinline__ double cg_rcp(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

// Non-positive, infinite, NaN and subnormal arguments: the library log, kept
// out of line so that the straight-line generated kernels do not carry a copy
// of it at every call site.
static __device__ __noinline__ double cg_log_special(double x) { return log(x); }

__device__ __forceinline__ double cg_log(double x) {
    const int hi = __double2hiint(x);
    const int lo = __double2loint(x);
    // normal, finite, positive: biased exponent in [1, 2046], sign clear
    if (hi < 0x00100000 || hi >= 0x7ff00000) return cg_log_special(x);
    int e = (hi >> 20) - 1023;
    int mh = (hi & 0x000fffff) | 0x3ff00000;          // m in [1, 2)
    if (mh > 0x3ff6a09e) {                            // m > sqrt(2): use m/2
        mh -= 0x00100000;
        e += 1;
    }
    const double m = __hiloint2double(mh, lo);
    const double s = (m - 1.0) * cg_rcp(m + 1.0);
    const double z = s * s;
    double p = 0.047619047619047616;                  // 1/21
    p = fma(p, z, 0.05263157894736842);               // 1/19
    p = fma(p, z, 0.058823529411764705);              // 1/17
    p = fma(p, z, 0.06666666666666667);               // 1/15
    p = fma(p, z, 0.07692307692307693);               // 1/13
    p = fma(p, z, 0.09090909090909091);               // 1/11
    p = fma(p, z, 0.1111111111111111);                // 1/9
    p = fma(p, z, 0.14285714285714285);               // 1/7
    p = fma(p, z, 0.2);                               // 1/5
    p = fma(p, z, 0.3333333333333333);                // 1/3
    const double lm = fma(2.0 * s * z, p, 2.0 * s);   // 2 s (1 + z p)
    const double de = (double)e;
    return fma(de, kLn2Hi, fma(de, kLn2Lo, lm));
}

__device__ __forceinline__ double cg_log10(double x) { return cg_log(x) * 0.4342944819032518; }

}  // namespace cgm
