// Device-side mechanism tables, built once per handle from the packed blob.
//
// The reference keeps its coefficients in per-mechanism __constant__ symbols
// uploaded by copyConstantsToDevice (chemgen/constants.py:53-240), which ties
// a process to one mechanism.  Here every handle owns one device buffer with
// the tables below, so any number of mechanisms coexist; kernels read them
// with warp-uniform loads (every lane of a warp works on the same reaction at
// the same time, so each load is one broadcast transaction served from L1).
#pragma once

#include <cstdint>

#include "../../include/chemgen_mech.h"

namespace cg {

// chemgen/chemistry.py:204-206
constexpr double kRc = 1.9872155832;
constexpr double kR0 = 8.314510e+07;
constexpr double kPatm = 1013250.0;

// extra device flag: stoichiometry stored in the compact slots of DRxn
constexpr int kFCompact = 1 << 8;
constexpr int kMaxCompact = 3;         // species per side in the compact form

// One reaction, 64 bytes: four 16-byte loads.
struct __align__(16) DRxn {
    double lnA;          // ln|A| (kinf for falloff); unused for PLOG
    double b;
    double theta;        // Ea / Rc, kelvin
    double sgn;          // sign of A (0 when A == 0)
    int flags;           // CG_F_* | kFCompact
    int aux;             // falloff row or PLOG row
    unsigned short sp[6];  // compact slots: reactants 0..2, products 3..5; species | nu << 14
    unsigned char nre, npr;
    int gen;             // general-stoichiometry row (when not compact), else -1
    int pad;
};
static_assert(sizeof(DRxn) == 64, "DRxn must stay 64 bytes");

// Falloff parameters, 64 bytes.
struct __align__(16) DFall {
    double lnA0, b0, theta0, sgn0;
    double p[4];         // Troe: 1-a, 1/T3, a, 1/T1 ; SRI: a, b, 1/c, d (e in pe)
};
struct __align__(16) DFall2 {
    double T2;           // Troe T2 (flag CG_F_TROE_T2), SRI e
    double pad;
};

struct DevMech {
    int ns, nr;
    int seg[CG_NKINDS + 1];     // kernel-order boundaries of each kind
    int has_m;
    int n_general;
    const double* inv_mw;       // [ns]
    const double* thermo;       // [ns*16]: Tmid, lo c0..c6, hi c0..c6, pad
    const DRxn* rxn;            // [nr]
    const int* eff_ptr;         // [nr+1]
    const int* eff_sp;          // [neff]
    const double* eff_val;      // [neff]
    const DFall* fall;          // [nfall]
    const DFall2* fall2;        // [nfall]
    const int* gen_rptr;        // [n_general+1]
    const int* gen_pptr;        // [n_general+1]
    const int* gen_sp;          // reactant then product entries
    const double* gen_nu;
    const int* plog_ptr;        // [nplog+1] into levels
    const double* plog_p;       // [nlev]
    const double* plog_lnp;     // [nlev]
    const int* plog_tptr;       // [nlev+1]
    const double4* plog_term;   // [nterm]: ln|A|, b, Ea/Rc, sign
};

}  // namespace cg
