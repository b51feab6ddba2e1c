// Shared per-point pieces of the getrates kernels: the Y -> C prologue
// (chemgen/templates/ytoc.j2:3-18), NASA-7 Gibbs (exp_g.j2:2-27), falloff
// blending (reactions/troe.j2:21-45) and the stoichiometric scatter
// (reactions/standard.j2:21-27).
#pragma once

#include "dev_mech.cuh"

namespace cg {

__device__ __forceinline__ DRxn load_rxn(const DRxn* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    DRxn r;
    int4* d = reinterpret_cast<int4*>(&r);
    d[0] = __ldg(q);
    d[1] = __ldg(q + 1);
    d[2] = __ldg(q + 2);
    d[3] = __ldg(q + 3);
    return r;
}

__device__ __forceinline__ DFall load_fall(const DFall* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    DFall f;
    double2* d = reinterpret_cast<double2*>(&f);
    d[0] = __ldg(q);
    d[1] = __ldg(q + 1);
    d[2] = __ldg(q + 2);
    d[3] = __ldg(q + 3);
    return f;
}

__device__ __forceinline__ int slot_species(unsigned short s) { return s & 0x3fff; }
__device__ __forceinline__ int slot_nu(unsigned short s) { return s >> 14; }

// x^nu for nu in {1, 2, 3}
__device__ __forceinline__ double ipow3(double x, int nu) {
    double y = x;
    if (nu >= 2) y *= x;
    if (nu == 3) y *= x;
    return y;
}

// Reciprocal by Newton-Raphson refinement of the hardware's approximate
// reciprocal (two iterations of r <- r (2 - x r) reach double precision).
__device__ __forceinline__ double rcp_nr(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    return r;
}

// Per-point temperature functions shared by every reaction.
struct PointT {
    double T, lnT, invT;
};

// smh = s/R - h/RT from the 7 rounded coefficients (exp_g.j2:8-24):
// c0 + c1 lnT + c2 T + c3 T^2 + c4 T^3 + c5 T^4 - c6/T
__device__ __forceinline__ double smh_poly(const double* c, double T, double lnT, double invT) {
    double p = fma(c[5], T, c[4]);
    p = fma(p, T, c[3]);
    p = fma(p, T, c[2]);
    return fma(p, T, fma(c[1], lnT, c[0])) - c[6] * invT;
}

// Select the coefficient range per point (T < Tmid -> low) with uniform loads.
__device__ __forceinline__ double species_smh(const double* thermo, int k, double T, double lnT, double invT) {
    const double2* th = reinterpret_cast<const double2*>(thermo + 16 * k);
    double c[16];
    double2* cc = reinterpret_cast<double2*>(c);
#pragma unroll
    for (int j = 0; j < 8; ++j) cc[j] = __ldg(th + j);
    const bool low = T < c[0];
    double sel[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) sel[j] = low ? c[1 + j] : c[8 + j];
    return smh_poly(sel, T, lnT, invT);
}

}  // namespace cg
