"""Mechanism -> packed tables (the blob format of ``include/chemgen_mech.h``).

Numeric constants are rounded through ``"%.15e"`` exactly as the reference
prints them into generated code (``chemgen/templates/exp_g.j2:8-24``,
``chemgen/templates/reactions/standard.j2:4``, ``troe.j2:9-38``,
``ytoc.j2:4``), so the tables hold the same doubles the reference's generated
getrates computes with.
"""
from __future__ import annotations

import dataclasses
import math
import struct
from typing import Dict, List

import numpy as np

from .mechanism import RC_CAL, REACTION_KINDS, Mechanism, Reaction

MAGIC = b"CGB200M1"
VERSION = 1
F_REVERSIBLE, F_INT_NU, F_TROE_T2, F_A_NEG, F_LOW_NEG = 1, 2, 4, 8, 16

SCALARS = ["VERSION", "NS", "NR", "NSTD", "N3B", "NLIND", "NTROE", "NSRI", "NPLOG", "NEFF", "NPLEV",
           "NPTERM", "FLAGS", "MAXNU_INT", "NRT", "NPT"]
ARRAYS = [
    ("MW", "f8"), ("INV_MW", "f8"), ("TMID", "f8"), ("SMH_LO", "f8"), ("SMH_HI", "f8"),
    ("NASA_LO", "f8"), ("NASA_HI", "f8"),
    ("ORIG", "i4"), ("FLAGS", "i4"), ("RPTR", "i4"), ("PPTR", "i4"), ("RSP", "i4"), ("PSP", "i4"),
    ("RNU", "f8"), ("PNU", "f8"), ("DNU", "f8"), ("ARH", "f8"), ("KARH", "f8"),
    ("EFF_PTR", "i4"), ("EFF_SP", "i4"), ("EFF_VAL", "f8"), ("FALL", "f8"), ("KFALL", "f8"),
    ("PLOG_PTR", "i4"), ("PLOG_P", "f8"), ("PLOG_LNP", "f8"), ("PLOG_TPTR", "i4"), ("PLOG_TERM", "f8"),
    ("KPLOG_TERM", "f8"),
]


def r15(x: float) -> float:
    """A double as the reference writes it into source: ``"%.15e" % x``."""
    return float("%.15e" % x)


def smh_coefs(a) -> List[float]:
    """NASA-7 a1..a7 -> c0..c6 of smh = c0 + c1 lnT + c2 T + c3 T^2 + c4 T^3 + c5 T^4 - c6/T
    (s/R - h/RT), rounded as chemgen/templates/exp_g.j2:8-24 prints them."""
    return [r15(a[6] - a[0]), r15(a[0]), r15(a[1] / 2.0), r15(a[2] / 6.0), r15(a[3] / 12.0),
            r15(a[4] / 20.0), r15(a[5])]


def _karh(A: float, b: float, Ea: float):
    return [math.log(abs(A)) if A != 0.0 else -745.0, b, Ea / RC_CAL, -1.0 if A < 0 else 1.0]


@dataclasses.dataclass
class Packed:
    mech: Mechanism
    scalars: Dict[str, int]
    arrays: Dict[str, np.ndarray]
    kernel_order: List[int]          # kernel index -> file index

    @property
    def ns(self) -> int:
        return self.scalars["NS"]

    @property
    def nr(self) -> int:
        return self.scalars["NR"]

    def to_blob(self) -> bytes:
        head = 8 + 8 * len(SCALARS) + 16 * len(ARRAYS)
        off = (head + 63) // 64 * 64
        table = []
        chunks = []
        for name, dt in ARRAYS:
            arr = np.ascontiguousarray(self.arrays[name], dtype=dt)
            table.append((off, arr.size))
            data = arr.tobytes()
            chunks.append((off, data))
            off = (off + len(data) + 63) // 64 * 64
        buf = bytearray(off + 64)
        buf[0:8] = MAGIC
        struct.pack_into("<%dq" % len(SCALARS), buf, 8, *[int(self.scalars[s]) for s in SCALARS])
        for i, (o, c) in enumerate(table):
            struct.pack_into("<qq", buf, 8 + 8 * len(SCALARS) + 16 * i, o, c)
        for o, data in chunks:
            buf[o:o + len(data)] = data
        return bytes(buf)


def _kind_order(mech: Mechanism) -> List[int]:
    order = []
    for kind in REACTION_KINDS:
        order += [i for i, r in enumerate(mech.reactions) if r.kind == kind]
    return order


def pack(mech: Mechanism) -> Packed:
    mech.validate()
    ns, nr = mech.ns, mech.nr
    idx = mech.species_index()
    sp = mech.species
    A: Dict[str, np.ndarray] = {}
    A["MW"] = np.array([r15(s.mw) for s in sp])
    A["INV_MW"] = 1.0 / A["MW"]
    A["TMID"] = np.array([s.t_ranges[1] for s in sp])
    A["SMH_LO"] = np.array([smh_coefs(s.nasa_low) for s in sp]).reshape(-1)
    A["SMH_HI"] = np.array([smh_coefs(s.nasa_high) for s in sp]).reshape(-1)
    A["NASA_LO"] = np.array([s.nasa_low for s in sp], dtype=float).reshape(-1)
    A["NASA_HI"] = np.array([s.nasa_high for s in sp], dtype=float).reshape(-1)

    order = _kind_order(mech)
    rx: List[Reaction] = [mech.reactions[i] for i in order]
    flags = np.zeros(nr, np.int32)
    rptr = [0]; pptr = [0]; rsp: List[int] = []; psp: List[int] = []
    rnu: List[float] = []; pnu: List[float] = []
    dnu = np.zeros(nr)
    arh = np.zeros((nr, 3)); karh = np.zeros((nr, 4))
    eff_ptr = [0]; eff_sp: List[int] = []; eff_val: List[float] = []
    fall: List[List[float]] = []; kfall: List[List[float]] = []
    plog_ptr = [0]; plog_p: List[float] = []; plog_lnp: List[float] = []; plog_tptr = [0]; plog_term: List[List[float]] = []
    kplog: List[List[float]] = []
    maxnu_int = 0
    for k, r in enumerate(rx):
        f = F_REVERSIBLE if r.reversible else 0
        nus = list(r.reactants.values()) + list(r.products.values())
        if all(n in (1.0, 2.0, 3.0) for n in nus):
            f |= F_INT_NU
            maxnu_int = max(maxnu_int, int(max(nus)))
        for s_, n in r.reactants.items():
            rsp.append(idx[s_]); rnu.append(n)
        for s_, n in r.products.items():
            psp.append(idx[s_]); pnu.append(n)
        rptr.append(len(rsp)); pptr.append(len(psp))
        dnu[k] = r.dnu
        if r.kind != "plog":
            Aa, b, Ea = r.arh
            arh[k] = (r15(Aa), b, r15(Ea))
            karh[k] = _karh(arh[k, 0], b, arh[k, 2])
            if Aa < 0:
                f |= F_A_NEG
        if r.uses_m:
            for s_, e in r.efficiencies.items():
                eff_sp.append(idx[s_]); eff_val.append(r15(e))
        eff_ptr.append(len(eff_sp))
        if r.is_falloff:
            A0, b0, Ea0 = r.low
            row = [r15(A0), b0, r15(Ea0)]
            if r.kind == "troe":
                a, T3, T1 = r.troe[:3]
                T2 = r.troe[3] if len(r.troe) == 4 else 0.0
                if len(r.troe) == 4 and T2 != 0.0:
                    f |= F_TROE_T2
                # chemgen/templates/reactions/troe.j2:35-36 prints 1-a, T3, a, T1, -T2
                row += [r15(a), r15(T3), r15(T1), r15(T2), r15(1.0 - a)]
            elif r.kind == "sri":
                s5 = list(r.sri) + ([1.0, 0.0] if len(r.sri) == 3 else [])
                row += [float(v) for v in s5]
            else:
                row += [0.0] * 5
            fall.append(row)
            kfall.append(_karh(row[0], b0, row[2]))
            if A0 < 0:
                f |= F_LOW_NEG
        if r.kind == "plog":
            # chemgen/chemistry.py:309-316 groups the entries by pressure
            levels: Dict[float, List] = {}
            for (p, Ap, bp, Eap) in r.plog:
                levels.setdefault(p, []).append((Ap, bp, Eap))
            for p in sorted(levels):
                # chemgen/templates/reactions/plog.j2:7-16 prints p and log(p) with %.15e
                plog_p.append(r15(p))
                plog_lnp.append(r15(math.log(p)))
                for (Ap, bp, Eap) in levels[p]:
                    plog_term.append([r15(Ap), bp, r15(Eap)])
                    kplog.append(_karh(r15(Ap), bp, r15(Eap)))
                plog_tptr.append(len(plog_term))
            plog_ptr.append(len(plog_p))
        flags[k] = f
    A["ORIG"] = np.array(order, np.int32)
    A["FLAGS"] = flags
    A["RPTR"], A["PPTR"] = np.array(rptr, np.int32), np.array(pptr, np.int32)
    A["RSP"], A["PSP"] = np.array(rsp, np.int32), np.array(psp, np.int32)
    A["RNU"], A["PNU"] = np.array(rnu, float), np.array(pnu, float)
    A["DNU"] = dnu
    A["ARH"], A["KARH"] = arh.reshape(-1), karh.reshape(-1)
    A["EFF_PTR"] = np.array(eff_ptr, np.int32)
    A["EFF_SP"] = np.array(eff_sp, np.int32)
    A["EFF_VAL"] = np.array(eff_val, float)
    A["FALL"] = np.array(fall, float).reshape(-1)
    A["KFALL"] = np.array(kfall, float).reshape(-1)
    A["PLOG_PTR"] = np.array(plog_ptr, np.int32)
    A["PLOG_P"] = np.array(plog_p, float)
    A["PLOG_LNP"] = np.array(plog_lnp, float)
    A["PLOG_TPTR"] = np.array(plog_tptr, np.int32)
    A["PLOG_TERM"] = np.array(plog_term, float).reshape(-1)
    A["KPLOG_TERM"] = np.array(kplog, float).reshape(-1)
    counts = mech.counts()
    S = {s: 0 for s in SCALARS}
    S.update(VERSION=VERSION, NS=ns, NR=nr, NSTD=counts["standard"], N3B=counts["third_body"],
             NLIND=counts["lindemann"], NTROE=counts["troe"], NSRI=counts["sri"], NPLOG=counts["plog"],
             NEFF=len(eff_sp), NPLEV=len(plog_p), NPTERM=len(plog_term), MAXNU_INT=maxnu_int, NRT=len(rsp), NPT=len(psp))
    return Packed(mech=mech, scalars=S, arrays=A, kernel_order=order)


def nu_matrix(mech: Mechanism) -> np.ndarray:
    """Dense net stoichiometry nu[ns, nr] (file order): products minus reactants."""
    idx = mech.species_index()
    nu = np.zeros((mech.ns, mech.nr))
    for j, r in enumerate(mech.reactions):
        for s, n in r.reactants.items():
            nu[idx[s], j] -= n
        for s, n in r.products.items():
            nu[idx[s], j] += n
    return nu
