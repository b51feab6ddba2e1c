"""Algorithmic operation inventory of getrates for one mechanism.

Counts, per grid point, the arithmetic the rate law requires (the work the
reference's generated code spells out, chemgen/templates/reactions/*.j2):
additions, multiplications, fused multiply-adds, reciprocals, exp and log.
The roofline of a kernel uses

    FLOP-equivalents / point = add + mul + 2 fma + c_rcp rcp + c_exp exp + c_log log

where c_x is the measured cost of one transcendental in FP64 FMA issue slots
(x2 flops), from chemgen_probe_fp64, and bytes / point = (2 + 2 ns) * 8
(P, T, Y in; wdot out).
"""
from __future__ import annotations

from typing import Dict

from .mechanism import Mechanism


def inventory(mech: Mechanism) -> Dict[str, int]:
    ns = mech.ns
    c = dict(add=0, mul=0, fma=0, rcp=0, exp=0, log=0)

    def add(**kw):
        for k, v in kw.items():
            c[k] += v

    # Y -> C (ytoc.j2): Y/W, sum, scale, sum again; ln T, 1/T, pfac
    add(mul=2 * ns + 2, add=2 * ns, rcp=2, log=1)
    # Gibbs (exp_g.j2): polynomial in T and ln T, exp, times pfac
    add(fma=5 * ns, mul=2 * ns, add=ns, exp=ns)
    for r in mech.reactions:
        nre = sum(int(round(v)) for v in r.reactants.values())
        npr = sum(int(round(v)) for v in r.products.values())
        nr_sp, np_sp = len(r.reactants), len(r.products)
        if r.kind == "plog":
            add(fma=2, mul=2, add=4, exp=3, log=3, rcp=1)          # two levels + interpolation
        else:
            add(fma=1, mul=2, add=1, exp=1)                        # A T^b exp(-E/RT) = exp(lnA + b lnT - E/RT)
        if r.is_falloff:
            add(fma=1, mul=2, add=1, exp=1)                        # k0
            add(mul=2, rcp=1)                                      # Pr = k0 M / kinf
            if r.kind == "troe":
                add(fma=2, mul=2, exp=2 + (1 if r.troe and len(r.troe) == 4 else 0), log=2)
                add(fma=4, add=2, mul=2, rcp=2, exp=1)             # C, N, f1, F
            elif r.kind == "sri":
                add(fma=3, mul=3, exp=3, log=2, rcp=1)
            add(add=1, mul=2, rcp=1)                               # Pr/(1+Pr) F kinf
        if r.uses_m:
            add(fma=len(r.efficiencies))                           # M = ctot + sum (eff-1) C
        if r.reversible:
            add(mul=max(nre - 1, 0) + max(npr - 1, 0) + 2, rcp=1)  # kf prod EGp_r / prod EGp_p
            add(mul=npr)                                           # qb
        add(mul=nre, add=1)                                        # qf, qf - qb
        if r.kind == "third_body":
            add(mul=1)
        add(fma=nr_sp + np_sp)                                     # scatter into wdot
    return c


def flop_equivalents(inv: Dict[str, int], c_exp: float, c_log: float, c_rcp: float) -> float:
    """FLOPs with transcendentals weighted by their measured FMA-slot cost (2 flops per slot)."""
    return (inv["add"] + inv["mul"] + 2 * inv["fma"] + 2 * c_rcp * inv["rcp"] + 2 * c_exp * inv["exp"]
            + 2 * c_log * inv["log"])


def bytes_per_point(ns: int) -> int:
    return (2 + 2 * ns) * 8
