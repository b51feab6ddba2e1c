"""ORACLE -- test infrastructure only.  A torch FP64 restatement of the
reference's generated getrates (chemgen/templates/python_header.j2, ytoc.j2,
exp_g.j2, reactions/{standard,third_body,troe,plog}.j2), vectorised over
points, so that torch.autograd can differentiate it.  It is the second
checker of the analytic Jacobian and adjoint kernels (the first being central
finite differences); nothing in the product imports it.

Lindemann and SRI follow reactions/troe.j2 with F = 1 and the Chemkin SRI
form; the coefficients are rounded as the reference prints them (%.15e).
"""
from __future__ import annotations

import math

import torch

from chemgen_b200.mechanism import Mechanism
from chemgen_b200.pack import r15, smh_coefs

RC = 1.9872155832
R0 = 8.314510e07
PATM = 1013250.0


def getrates(mech: Mechanism, P: torch.Tensor, T: torch.Tensor, Y: torch.Tensor) -> torch.Tensor:
    """wdot [ns, ng] from P [ng], T [ng], Y [ns, ng] (float64, any device)."""
    idx = mech.species_index()
    mw = torch.tensor([r15(w) for w in mech.mw()], dtype=Y.dtype, device=Y.device)
    pfac = PATM / (R0 * T)
    C = Y / mw[:, None]                                       # ytoc.j2
    ctot = C.sum(dim=0)
    C = C * P / (R0 * ctot * T)
    ctot = C.sum(dim=0)
    EG = []
    for sp in mech.species:                                   # exp_g.j2
        lo, hi = smh_coefs(sp.nasa_low), smh_coefs(sp.nasa_high)

        def poly(c):
            return (c[0] + c[1] * torch.log(T) + c[2] * T + c[3] * T ** 2 + c[4] * T ** 3 + c[5] * T ** 4
                    - c[6] / T)
        EG.append(torch.exp(torch.where(T < sp.t_ranges[1], poly(lo), poly(hi))))
    EG = torch.stack(EG)
    wdot = torch.zeros_like(C)

    def arr(A, b, Ea):
        A, Ea = r15(A), r15(Ea)
        k = A * torch.ones_like(T)
        if b != 0.0:
            k = k * T ** b
        return k * torch.exp((-1.0 * Ea) / (RC * T))

    for r in mech.reactions:
        M = None
        if r.uses_m:
            M = ctot.clone()
            for sp, e in r.efficiencies.items():
                M = M + r15(e) * C[idx[sp]]
        if r.kind in ("standard", "third_body"):
            kf = arr(*r.arh)
        elif r.kind == "plog":
            levels = {}
            for (p, A, b, Ea) in r.plog:
                levels.setdefault(r15(p), []).append((A, b, Ea))
            ps = sorted(levels)
            ks = [sum(arr(A, b, Ea) for (A, b, Ea) in levels[p]) for p in ps]
            lnP = torch.log(P)
            kf = ks[0]
            for j in range(1, len(ps)):
                lo, hi = ps[j - 1], ps[j]
                llo, lhi = r15(math.log(lo)), r15(math.log(hi))
                # weight clamped to [0, 1]: equal inside the bracket, and keeps the
                # unselected branches of torch.where finite for autograd
                w = torch.clamp((lnP - llo) / (lhi - llo), 0.0, 1.0)
                interp = torch.exp(torch.log(ks[j - 1]) + (torch.log(ks[j]) - torch.log(ks[j - 1])) * w)
                kf = torch.where(P >= lo, torch.where(P < hi, interp, kf), kf)
            kf = torch.where(P >= ps[-1], ks[-1], kf)
        else:
            k0 = arr(*r.low)
            kinf = arr(*r.arh)
            Pr = k0 * M / kinf
            if r.kind == "troe":
                a, T3, T1 = (r15(x) for x in r.troe[:3])
                Fc = r15(1.0 - a) * torch.exp(-T / T3) + a * torch.exp(-T / T1)
                if len(r.troe) == 4 and r.troe[3] != 0.0:
                    Fc = Fc + torch.exp(-r15(r.troe[3]) / T)
                C1 = -0.4 - 0.67 * torch.log10(Fc)
                N1 = 0.75 - 1.27 * torch.log10(Fc)
                f1 = (torch.log10(Pr) + C1) / (N1 - 0.14 * (torch.log10(Pr) + C1))
                F = 10.0 ** (torch.log10(Fc) / (1.0 + f1 ** 2))
            elif r.kind == "sri":
                s = list(r.sri) + ([1.0, 0.0] if len(r.sri) == 3 else [])
                X = 1.0 / (1.0 + torch.log10(Pr) ** 2)
                F = s[3] * (s[0] * torch.exp(-s[1] / T) + torch.exp(-T / s[2])) ** X * T ** s[4]
            else:
                F = torch.ones_like(T)
            kf = kinf * (Pr / (1.0 + Pr)) * F
        qf = kf
        for sp, nu in r.reactants.items():
            qf = qf * C[idx[sp]] ** nu
        if r.reversible:
            kb = kf
            for sp, nu in r.reactants.items():
                kb = kb * EG[idx[sp]] ** nu
            for sp, nu in r.products.items():
                kb = kb / EG[idx[sp]] ** nu
            if r.dnu != 0.0:
                kb = kb / pfac ** r.dnu
            qb = kb
            for sp, nu in r.products.items():
                qb = qb * C[idx[sp]] ** nu
        else:
            qb = torch.zeros_like(qf)
        rr = qf - qb
        if r.kind == "third_body":
            rr = M * rr
        upd = torch.zeros_like(C)
        for sp, nu in r.reactants.items():
            upd[idx[sp]] = upd[idx[sp]] - nu * rr
        for sp, nu in r.products.items():
            upd[idx[sp]] = upd[idx[sp]] + nu * rr
        wdot = wdot + upd
    return wdot
