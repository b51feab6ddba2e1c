"""``--language cuda``: emit mechanism-specialised sm_100a getrates kernels.

The reference renders one Jinja template per reaction into straight-line
Python/Fortran/HIP (``chemgen/chemistry.py:269-321``).  This emitter does the
same for CUDA: every reaction becomes a few lines with its coefficients and
species slots as compile-time constants, so the kernel carries no table
lookups or index arithmetic, and the per-species wdot accumulators are
registers.  Two kernels are written per mechanism:

* ``fp64``  -- the reference's arithmetic in FP64 (reactions/*.j2);
* ``mixed`` -- exponents (Arrhenius, Gibbs differences -> Kc) and the wdot
  sums in FP64, 2^f / concentration products / falloff blending in FP32.

The module registers itself with libchemgen_b200.so at load time under the
64-bit FNV-1a fingerprint of the mechanism's packed blob, after which
``chemgen_create`` on the same blob dispatches to it.
"""
from __future__ import annotations

import hashlib
import math
import os
import subprocess
from typing import Dict, List, Optional, Tuple

from .mechanism import RC_CAL, Mechanism, Reaction
from .pack import pack, r15, smh_coefs

LOG2E = 1.4426950408889634074
LN10 = 2.302585092994045684
LOG10_2 = 0.30102999566398119521
CSCALE_LOG2 = 32          # mixed: concentrations are stored as C * 2^32 in FP32
# register-resident wdot accumulators up to this many species
MAX_REG_SPECIES = 72
SYNC_EVERY = 96           # reactions between block barriers, FP64 kernel (B200 sweeps at 53/325: 2..128, 0)
# FP64 kernel: consecutive reactions whose tensor-memory values load behind one wait
# (B200 at 53/325, 2^20 points: 1 -> 509-530, 3 -> 541-554 Mpts/s with barriers every 64-96
# reactions or none; 2, 4 and 6 gained less)
EGP_GROUP = 3
SYNC_EVERY_MIXED = 96     # mixed kernel (B200 sweeps at 53/325, 16 warps, streaming I/O: 12..96 and
                          # none within 3 %; 24 was best at 11 warps before the streaming hints)
SMEM_BUDGET = 220 * 1024  # dynamic shared memory per block
REG_FILE = 65536          # 32-bit registers per SM
MAX_BLOCK = 512           # 16 warps; beyond this the 53-species kernels spill heavily


def fingerprint(blob: bytes) -> int:
    """64-bit FNV-1a of the packed blob (same function as capi.cu)."""
    h = 0xcbf29ce484222325
    for b in blob:
        h ^= b
        h = (h * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    return h


def reaction_order(mech: Mechanism) -> List[int]:
    """An order of the reactions that keeps few wdot accumulators live.

    The generated kernels hold one FP64 accumulator per species in registers
    from the first reaction that touches the species to the last, after which
    its wdot is stored.  Reactions are independent, so any order gives the
    same sums (up to rounding); this one is built greedily -- next comes the
    reaction that opens the fewest new species net of those it closes, ties
    to the one that closes more, then to file order -- which at 53 species /
    325 reactions brings the peak from 44 live accumulators in file order to
    about 30, leaving the registers to overlap the reactions' arithmetic."""
    idx = mech.species_index()
    S = [frozenset(idx[x] for x in list(r.reactants) + list(r.products)) for r in mech.reactions]
    remaining_uses = [0] * mech.ns
    for sp in S:
        for k in sp:
            remaining_uses[k] += 1
    opened = set()
    left = list(range(len(S)))
    order: List[int] = []
    while left:
        best, key = None, None
        for r in left:
            new = sum(1 for k in S[r] if k not in opened)
            close = sum(1 for k in S[r] if remaining_uses[k] == 1)
            kk = (new - close, -close, r)
            if key is None or kk < key:
                best, key = r, kk
        order.append(best)
        left.remove(best)
        for k in S[best]:
            remaining_uses[k] -= 1
            opened.add(k)
    return order


def live_accumulators(mech: Mechanism, order: List[int]) -> int:
    """Peak number of species whose accumulator is live under `order`."""
    idx = mech.species_index()
    first, last = {}, {}
    for p, j in enumerate(order):
        r = mech.reactions[j]
        for sp in list(r.reactants) + list(r.products):
            first.setdefault(idx[sp], p)
            last[idx[sp]] = p
    live = [0] * (len(order) + 1)
    for k, f in first.items():
        live[f] += 1
        live[last[k] + 1] -= 1
    best = cur = 0
    for x in live:
        cur += x
        best = max(best, cur)
    return best


def _d(x: float) -> str:
    """A double literal that round-trips."""
    if x == 0.0:
        return "0.0"
    if math.isinf(x):
        return "(1.0/0.0)" if x > 0 else "(-1.0/0.0)"
    return repr(float(x))


def _f(x: float) -> str:
    return repr(float(x)) + "f"


class _Emitter:
    def __init__(self, mech: Mechanism, block: int, sync_every: int = SYNC_EVERY, tmem: bool = False,
                 live_order: bool = True, exp_noinline: bool = False, tm_prefetch: bool = False,
                 egp_group: int = 1, stream_io: bool = False):
        self.sync_every = sync_every
        # FP64 tensor-memory mode: the values of egp_group consecutive
        # reactions load behind one wait, so that their arithmetic can overlap
        self.egp_group = egp_group if (tmem and not tm_prefetch) else 1
        self._egp_ready = False
        # P, T, Y read and wdot written with streaming cache hints (evict first):
        # the inputs and outputs (0.9 GB per 2^20 points at 53 species) then
        # leave L2 before the kernel's own straight-line code (~0.5 MB, fetched
        # by every block of every wave), which otherwise they evict.  On B200
        # at 53/325, 2^20 points: FP64 515 -> 713, mixed 790 -> 832 Mpts/s.
        self.stream_io = stream_io
        # reactions call out-of-line copies of the FP64 exp (shorter code)
        self.exp_noinline = exp_noinline
        # tensor-memory mode: a reversible reaction's values are loaded while
        # the previous reversible reaction computes (split issue / wait)
        self.tm_prefetch = tm_prefetch and tmem
        # register accumulators: reactions in live-range order, each wdot
        # stored right after the last reaction that touches its species
        self.live_order = live_order and mech.ns <= MAX_REG_SPECIES
        self.mech = mech
        self.ns = mech.ns
        self.idx = mech.species_index()
        self.block = block
        self.reg_w = self.ns <= MAX_REG_SPECIES
        self.has_m = any(r.uses_m for r in mech.reactions)
        # EGp (FP64 kernel) or the log2 Gibbs terms (mixed) in tensor memory
        # instead of shared memory
        self.tmem = tmem
        self._eloc: Dict[str, str] = {}

    # ------------------------------------------------------------- helpers
    def ld(self, arr: str, idx: str) -> str:
        return f"__ldcs({arr} + {idx})" if self.stream_io else f"{arr}[{idx}]"

    def st(self, idx: str, val: str) -> str:
        return f"__stcs(wdot + {idx}, {val});" if self.stream_io else f"wdot[{idx}] = {val};"

    def C(self, sp: str) -> str:
        return f"sC[{self.idx[sp]}][t]"

    def E(self, sp: str) -> str:
        if self.tmem:
            return self._eloc[sp]
        return f"sE[{self.idx[sp]}][t]"

    def G(self, sp: str) -> str:
        if self.tmem:
            return self._eloc[sp]
        return f"sG[{self.idx[sp]}][t]"

    def tmem_cols(self) -> int:
        """Tensor-memory columns the FP64 kernel allocates (a power of two)."""
        need = -(-self.block // 128) * 2 * self.ns
        n = 32
        while n < need:
            n *= 2
        return n

    def _egp_species(self, r: Reaction) -> List[str]:
        return list(dict.fromkeys(list(r.reactants) + list(r.products)))

    def issue_egp(self, j: int, r: Reaction) -> List[str]:
        """Prefetch mode: start the loads of reaction j's values (function scope)."""
        sps = self._egp_species(r)
        L = [f"uint32_t tq{j}[{2 * len(sps)}];"]
        for n, sp in enumerate(sps):
            L.append(f"cgg::tm_issue(tw + {2 * self.idx[sp]}u, tq{j}[{2 * n}], tq{j}[{2 * n + 1}]);")
        return L

    def wait_egp(self, j: int, r: Reaction) -> List[str]:
        """Prefetch mode: complete reaction j's loads and name its values."""
        sps = self._egp_species(r)
        self._eloc = {sp: f"e{j}_{n}" for n, sp in enumerate(sps)}
        L = [f"cgg::tm_wait_{len(sps)}(tq{j});"]
        L.append("const double " + ", ".join(f"e{j}_{n} = __hiloint2double((int)tq{j}[{2 * n + 1}], (int)tq{j}[{2 * n}])"
                                             for n in range(len(sps))) + ";")
        return L

    def group_egp(self, p: int, rs: List[Reaction]) -> List[str]:
        """Grouped mode: issue the loads of the EGp values the reversible
        reactions in `rs` need, wait once, and name them for the reactions."""
        sps = list(dict.fromkeys(sp for r in rs if r.reversible for sp in self._egp_species(r)))
        self._egp_ready = True
        self._eloc = {sp: f"g{p}_{n}" for n, sp in enumerate(sps)}
        if not sps:
            return []
        L = [f"uint32_t gq{p}[{2 * len(sps)}];"]
        for n, sp in enumerate(sps):
            L.append(f"cgg::tm_issue(tw + {2 * self.idx[sp]}u, gq{p}[{2 * n}], gq{p}[{2 * n + 1}]);")
        ops = ", ".join(f'"+r"(gq{p}[{k}])' for k in range(2 * len(sps)))
        L.append(f'__syncwarp(); asm volatile("tcgen05.wait::ld.sync.aligned;" : {ops} :: "memory");')
        L.append("const double " + ", ".join(f"g{p}_{n} = __hiloint2double((int)gq{p}[{2 * n + 1}], (int)gq{p}[{2 * n}])"
                                             for n in range(len(sps))) + ";")
        return L

    def load_egp(self, r: Reaction) -> List[str]:
        """Tensor-memory mode: load the reaction's EGp (FP64 kernel) or log2
        Gibbs values (mixed) into locals, in batches of up to four loads that
        share one wait."""
        sps = list(dict.fromkeys(list(r.reactants) + list(r.products)))
        self._eloc = {sp: f"e{j}" for j, sp in enumerate(sps)}
        L = ["double " + ", ".join(self._eloc[sp] for sp in sps) + ";"]
        for b in range(0, len(sps), 4):
            grp = sps[b:b + 4]
            addrs = ", ".join(f"tw + {2 * self.idx[sp]}u" for sp in grp)
            outs = ", ".join(self._eloc[sp] for sp in grp)
            L.append(f"cgg::tm_ld({addrs}, {outs});")
        return L

    def W(self, sp: str) -> str:
        k = self.idx[sp]
        return f"w{k}" if self.reg_w else f"sW[{k}][t]"

    @staticmethod
    def _pow(x: str, nu: float) -> str:
        if nu == 1.0:
            return x
        if nu == 2.0:
            return f"({x}*{x})"
        if nu == 3.0:
            return f"({x}*{x}*{x})"
        return f"pow({x}, {_d(nu)})"

    def prod(self, side: Dict[str, float], fn) -> str:
        terms = [self._pow(fn(sp), nu) for sp, nu in side.items()]
        return "*".join(terms) if terms else "1.0"

    def scatter(self, r: Reaction, rr: str) -> List[str]:
        out = []
        for sp, nu in r.reactants.items():
            w = self.W(sp)
            out.append(f"{w} = fma({_d(-nu)}, {rr}, {w});" if nu != 1.0 else f"{w} -= {rr};")
        for sp, nu in r.products.items():
            w = self.W(sp)
            out.append(f"{w} = fma({_d(nu)}, {rr}, {w});" if nu != 1.0 else f"{w} += {rr};")
        return out

    @staticmethod
    def arr64(A: float, b: float, Ea: float) -> str:
        """A T^b exp(-Ea/(Rc T)) as one FP64 exp (reactions/standard.j2:4)."""
        A, Ea = r15(A), r15(Ea)
        if A == 0.0:
            return "0.0"
        lnA = math.log(abs(A))
        th = Ea / RC_CAL
        sgn = "-" if A < 0 else ""
        parts = [_d(lnA)]
        if b != 0.0:
            parts = [f"fma({_d(b)}, lnT, {_d(lnA)})"]
        if th != 0.0:
            parts.append(f"- {_d(th)}*invT")
        if b == 0.0 and th == 0.0:
            return _d(A)
        # the exponent over 100..10000 K decides whether clamping is needed
        Ts = [100.0 * 1.1 ** j for j in range(49)]
        args = [lnA + b * math.log(t) - th / t for t in Ts]
        fn = "cgm::cg_exp" if -700.0 < min(args) and max(args) < 700.0 else "cgm::cg_exp_clamped"
        return f"{sgn}{fn}({' '.join(parts)})"

    @staticmethod
    def arr2(A: float, b: float, Ea: float) -> Tuple[str, bool]:
        """log2 of |A T^b exp(-Ea/(Rc T))| as an FP64 expression, and the sign."""
        A, Ea = r15(A), r15(Ea)
        l2A = math.log2(abs(A)) if A != 0.0 else -2000.0
        th2 = Ea / RC_CAL * LOG2E
        e = _d(l2A)
        if b != 0.0:
            e = f"fma({_d(b)}, lnT2, {_d(l2A)})"    # b * log2 T
        if th2 != 0.0:
            e = f"fma({_d(-th2)}, invT, {e})"
        return e, A < 0

    # --------------------------------------------------------------- fp64
    @staticmethod
    def arg64(A: float, b: float, Ea: float) -> str:
        """ln|A| + b ln T - Ea/(Rc T) as an FP64 expression."""
        A, Ea = r15(A), r15(Ea)
        e = _d(math.log(abs(A)) if A != 0.0 else -745.0)
        if b != 0.0:
            e = f"fma({_d(b)}, lnT, {e})"
        th = Ea / RC_CAL
        if th != 0.0:
            e = f"fma({_d(-th)}, invT, {e})"
        return e

    def falloff64(self, r: Reaction) -> List[str]:
        """kinf * Pr/(1+Pr) * F (troe.j2:21-45) with Pr = exp(ln k0 - ln kinf) M
        and ln F folded into the exponent of kinf."""
        L = []
        if r15(r.arh[0]) <= 0.0 or r15(r.low[0]) <= 0.0:
            # zero or negative pre-exponential factors: direct form
            L.append(f"const double kinf = {self.arr64(*r.arh)};")
            L.append(f"const double k0 = {self.arr64(*r.low)};")
            L.append("const double Pr = k0 * M * rcp(kinf);")
            L.append("const double lkinf = 0.0;")
            direct = True
        else:
            L.append(f"const double lkinf = {self.arg64(*r.arh)};")
            L.append(f"const double lr = {self.arg64(*r.low)} - lkinf;")
            L.append("const double Pr = cgm::cg_exp_clamped(lr) * M;")
            direct = False
        if r.kind == "troe":
            a, T3, T1 = (r15(x) for x in r.troe[:3])
            fc = (f"fma({_d(r15(1.0 - a))}, cgm::cg_exp_clamped({_d(-1.0 / T3)}*Tv), "
                  f"{_d(a)}*cgm::cg_exp_clamped({_d(-1.0 / T1)}*Tv))")
            if len(r.troe) == 4 and r.troe[3] != 0.0:
                fc = f"({fc} + cgm::cg_exp_clamped({_d(-r15(r.troe[3]))}*invT))"
            L.append(f"const double Fc = {fc};")
            L.append("const double lFc = cgm::cg_log10(Fc);")
            if direct:
                L.append("const double lp = cgm::cg_log10(Pr) + fma(-0.67, lFc, -0.4);")
            else:
                L.append(f"const double lp = fma(lr, {_d(1.0 / LN10)}, cgm::cg_log10(M)) + fma(-0.67, lFc, -0.4);")
            L.append("const double f1 = lp * rcp(fma(-0.14, lp, fma(-1.27, lFc, 0.75)));")
            L.append(f"const double lnF = {_d(LN10)} * lFc * rcp(fma(f1, f1, 1.0));")
        elif r.kind == "sri":
            s_ = list(r.sri) + ([1.0, 0.0] if len(r.sri) == 3 else [])
            L.append("const double lp = cgm::cg_log10(Pr);")
            L.append("const double X = rcp(fma(lp, lp, 1.0));")
            L.append(f"const double base = fma({_d(s_[0])}, cgm::cg_exp_clamped({_d(-s_[1])}*invT), "
                     f"cgm::cg_exp_clamped({_d(-1.0 / s_[2])}*Tv));")
            L.append(f"const double lnF = {_d(math.log(s_[3]))} + fma(X, cgm::cg_log(base), {_d(s_[4])}*lnT);")
        else:
            L.append("const double lnF = 0.0;")
        if direct:
            L.append("const double kf = kinf * (Pr * rcp(1.0 + Pr)) * cgm::cg_exp_clamped(lnF);")
        else:
            L.append("const double kf = cgm::cg_exp_clamped(lkinf + lnF) * (Pr * rcp(1.0 + Pr));")
        return L

    def plog64(self, r: Reaction) -> List[str]:
        levels: Dict[float, List] = {}
        for (p, A, b, Ea) in r.plog:
            levels.setdefault(r15(p), []).append((A, b, Ea))
        ps = sorted(levels)

        def ksum(p):
            return " + ".join(f"({self.arr64(A, b, Ea)})" for (A, b, Ea) in levels[p])

        L = ["double kf;"]
        L.append(f"if (Pv < {_d(ps[0])}) {{ kf = {ksum(ps[0])}; }}")
        for lo, hi in zip(ps[:-1], ps[1:]):
            llo, lhi = r15(math.log(lo)), r15(math.log(hi))
            L.append(f"else if (Pv < {_d(hi)}) {{ const double kl = cgm::cg_log({ksum(lo)}); "
                     f"const double kh = cgm::cg_log({ksum(hi)}); "
                     f"kf = cgm::cg_exp_clamped(kl + (kh - kl) * (lnP - {_d(llo)}) * {_d(1.0 / (lhi - llo))}); }}")
        L.append(f"else {{ kf = {ksum(ps[-1])}; }}")
        return L

    def reaction64(self, r: Reaction) -> List[str]:
        L = [f"{{ // {r.equation}"]
        body = []
        if r.uses_m:
            m = "ctot"
            for sp, e in r.efficiencies.items():
                m = f"fma({_d(r15(e))}, {self.C(sp)}, {m})"
            body.append(f"const double M = {m};")
        if r.kind in ("standard", "third_body"):
            body.append(f"const double kf = {self.arr64(*r.arh)};")
        elif r.kind == "plog":
            body += self.plog64(r)
        else:
            body += self.falloff64(r)
        qf = f"kf*{self.prod(r.reactants, self.C)}"
        if r.reversible:
            if self.tmem and not self.tm_prefetch and not self._egp_ready:
                body += self.load_egp(r)
            num = self.prod(r.reactants, self.E)
            den = self.prod(r.products, self.E)
            body.append(f"const double rr = {qf} - kf*({num})*rcp({den})*{self.prod(r.products, self.C)};")
        else:
            body.append(f"const double rr = {qf};")
        rr = "(M*rr)" if r.kind == "third_body" else "rr"
        body += self.scatter(r, rr)
        L += ["  " + x for x in body] + ["}"]
        return L

    # -------------------------------------------------------------- mixed
    def cprod32(self, side: Dict[str, float]) -> Tuple[str, int]:
        """FP32 product of scaled concentrations and its total order."""
        terms, order = [], 0
        for sp, nu in side.items():
            x = f"sc[{self.idx[sp]}][t]"
            if nu in (1.0, 2.0, 3.0):
                terms += [x] * int(nu)
                order += int(nu)
            else:
                return "", -1
        return ("*".join(terms) if terms else "1.0f"), order

    def gsum(self, r: Reaction) -> str:
        """sum nu_r G_r - sum nu_p G_p with G = log2(EGp) (FP64, shared memory)."""
        terms = [(nu, sp) for sp, nu in r.reactants.items()] + [(-nu, sp) for sp, nu in r.products.items()]
        expr = None
        for coef, sp in terms:
            g = self.G(sp)
            if expr is None:
                expr = g if coef == 1.0 else f"{_d(coef)}*{g}"
            elif coef == 1.0:
                expr = f"({expr} + {g})"
            elif coef == -1.0:
                expr = f"({expr} - {g})"
            else:
                expr = f"fma({_d(coef)}, {g}, {expr})"
        return expr

    def falloff32(self, r: Reaction) -> List[str]:
        """log2 kf of a falloff reaction: FP64 exponents, FP32 blending."""
        L = []
        ainf, _ = self.arr2(*r.arh)
        a0, _ = self.arr2(*r.low)
        L.append(f"const double ainf = {ainf};")
        # Pr = 2^(a0 - ainf) * M ; M is carried as Ms = M * 2^32 in FP32
        L.append(f"int npr; float fpr; cgg::split2({a0} - ainf, npr, fpr);")
        L.append("float mpr = cgg::ex2f(fpr) * Ms;")
        L.append("int ex = ((__float_as_int(mpr) >> 23) & 0xff) - 126; npr += ex - 32;")
        L.append("mpr = __int_as_float((__float_as_int(mpr) & 0x807fffff) | (126 << 23));   // [0.5, 1)")
        # lg2 Pr/(1+Pr) = npr + lg2(mpr) - lg2(1+Pr) (Pr < 1) or -lg2(1+1/Pr), branch-free
        L.append("float l2r; int nfix; const float l2m = cgg::lg2f(mpr); const float l2pr = (float)npr + l2m;")
        L.append("cgg::falloff_blend(mpr, npr, l2m, l2r, nfix);")
        if r.kind == "troe":
            a, T3, T1 = (r15(x) for x in r.troe[:3])
            fc = (f"fmaf({_f(r15(1.0 - a))}, cgg::ex2f({_f(-LOG2E / T3)}*Tf), "
                  f"{_f(a)}*cgg::ex2f({_f(-LOG2E / T1)}*Tf))")
            if len(r.troe) == 4 and r.troe[3] != 0.0:
                fc = f"({fc} + cgg::ex2f({_f(-LOG2E * r15(r.troe[3]))}*invTf))"
            L.append(f"const float Fc = {fc};")
            L.append(f"const float lFc = {_f(LOG10_2)} * cgg::lg2f(Fc);")
            L.append(f"const float lp = {_f(LOG10_2)} * l2pr + fmaf(-0.67f, lFc, -0.4f);")
            L.append("const float f1 = __fdividef(lp, fmaf(-0.14f, lp, fmaf(-1.27f, lFc, 0.75f)));")
            L.append(f"const float l2F = {_f(1.0 / LOG10_2)} * __fdividef(lFc, fmaf(f1, f1, 1.0f));")
        elif r.kind == "sri":
            s = list(r.sri) + ([1.0, 0.0] if len(r.sri) == 3 else [])
            L.append(f"const float lp = {_f(LOG10_2)} * l2pr;")
            L.append("const float X = __fdividef(1.0f, fmaf(lp, lp, 1.0f));")
            L.append(f"const float base = fmaf({_f(s[0])}, cgg::ex2f({_f(-LOG2E * s[1])}*invTf), "
                     f"cgg::ex2f({_f(-LOG2E / s[2])}*Tf));")
            L.append(f"const float l2F = {_f(math.log2(s[3]) if s[3] > 0 else -200.0)} + X*cgg::lg2f(base) "
                     f"+ {_f(s[4])}*lnT2f;")
        else:
            L.append("const float l2F = 0.0f;")
        L.append("const double akf = ainf + ((double)nfix + (double)(l2r + l2F));")
        return L

    def reaction32(self, r: Reaction) -> List[str]:
        L = [f"{{ // {r.equation}"]
        body = []
        cf, of = self.cprod32(r.reactants)
        cb, ob = self.cprod32(r.products)
        if of < 0 or ob < 0 or r.kind == "plog":
            # fractional stoichiometry or PLOG: the FP64 formula of this reaction
            return self.reaction32_fallback(r)
        if r.uses_m:
            m = "ctot32"
            for sp, e in r.efficiencies.items():
                m = f"fmaf({_f(r15(e))}, sc[{self.idx[sp]}][t], {m})"
            body.append(f"const float Ms = {m};")
        if r.kind in ("standard", "third_body"):
            a, neg = self.arr2(*r.arh)
            body.append(f"const double akf = {a};")
            if r.kind == "third_body":
                cf, of = f"{cf}*Ms", of + 1
                cb, ob = f"{cb}*Ms", ob + 1
            sgn = "-" if neg else ""
        else:
            body += self.falloff32(r)
            sgn = ""
        body.append(f"double rr = {sgn}cgg::rate2(akf, {cf}, {-CSCALE_LOG2 * of});")
        if r.reversible:
            if self.tmem and not self._egp_ready:
                body += self.load_egp(r)
            body.append(f"rr -= {sgn}cgg::rate2(akf + {self.gsum(r)}, {cb}, {-CSCALE_LOG2 * ob});")
        body += self.scatter(r, "rr")
        L += ["  " + x for x in body] + ["}"]
        return L

    def reaction32_fallback(self, r: Reaction) -> List[str]:
        """FP64 evaluation inside the mixed kernel (fractional nu, PLOG)."""
        L = [f"{{ // {r.equation} (FP64)"]
        body = []
        C = lambda sp: f"((double)sc[{self.idx[sp]}][t] * {_d(2.0 ** -CSCALE_LOG2)})"
        E = lambda sp: f"exp2({self.G(sp)})"
        if r.uses_m:
            m = "((double)ctot32 * " + _d(2.0 ** -CSCALE_LOG2) + ")"
            for sp, e in r.efficiencies.items():
                m = f"fma({_d(r15(e))}, {C(sp)}, {m})"
            body.append(f"const double M = {m};")
        if r.kind in ("standard", "third_body"):
            body.append(f"const double kf = {self.arr64(*r.arh)};")
        elif r.kind == "plog":
            body += self.plog64(r)
        else:
            body += self.falloff64(r)
        qf = f"kf*{self.prod(r.reactants, C)}"
        if r.reversible:
            if self.tmem and not self._egp_ready:
                body += self.load_egp(r)
            body.append(f"const double rr = {qf} - kf*({self.prod(r.reactants, E)})*rcp({self.prod(r.products, E)})"
                        f"*{self.prod(r.products, C)};")
        else:
            body.append(f"const double rr = {qf};")
        rr = "(M*rr)" if r.kind == "third_body" else "rr"
        body += self.scatter(r, rr)
        L += ["  " + x for x in body] + ["}"]
        return L

    # ------------------------------------------------------------- kernels
    def prologue(self, mixed: bool) -> List[str]:
        """Load P, T, Y; C = Y/W * P/(R0 sum(Y/W) T) (ytoc.j2); Gibbs (exp_g.j2)."""
        ns, B = self.ns, self.block
        L = []
        L.append("const int t = threadIdx.x;")
        L.append(f"const int64_t i = (int64_t)blockIdx.x * {B} + t;")
        L.append("const bool act = i < ng;")
        L.append(f"const double Tv = act ? {self.ld('T', 'i')} : 1000.0;")
        L.append(f"const double Pv = act ? {self.ld('P', 'i')} : {_d(1013250.0)};")
        L.append("const double lnT = cgm::cg_log(Tv), invT = rcp(Tv);")
        if any(r.kind == "plog" for r in self.mech.reactions):
            L.append("const double lnP = cgm::cg_log(Pv);")
        mw = self.mech.mw()
        L.append("double csum = 0.0;")
        if mixed and self.tmem:
            # unscaled Y/W in registers (the accumulators are not live yet)
            for k in range(ns):
                L.append(f"const double y{k} = (act ? {self.ld('Y', f'(int64_t){k} * ng + i')} : 1.0) * {_d(1.0 / r15(mw[k]))}; "
                         f"csum += y{k};")
        else:
            tmp = "sC" if not mixed else "sG"      # unscaled Y/W, overwritten below
            for k in range(ns):
                L.append(f"{{ const double c = (act ? {self.ld('Y', f'(int64_t){k} * ng + i')} : 1.0) * {_d(1.0 / r15(mw[k]))}; "
                         f"{tmp}[{k}][t] = c; csum += c; }}")
        L.append(f"const double fac = Pv * rcp({_d(8.314510e+07)} * csum * Tv);")
        L.append("double ctot = 0.0;")
        if not mixed:
            for k in range(ns):
                L.append(f"{{ const double c = sC[{k}][t] * fac; sC[{k}][t] = c; ctot += c; }}")
            L.append(f"const double pfac = {_d(1013250.0 / 8.314510e+07)} * invT;")
        else:
            L.append(f"const double facs = fac * {_d(2.0 ** CSCALE_LOG2)};")
            for k in range(ns):
                src = f"y{k}" if self.tmem else f"sG[{k}][t]"
                L.append(f"{{ const double c = {src} * facs; sc[{k}][t] = (float)c; ctot += c; }}")
            L.append("const float ctot32 = (float)ctot;")
            L.append(f"const double lnT2 = lnT * {_d(LOG2E)};")
            L.append(f"const double lpfac2 = {_d(math.log2(1013250.0 / 8.314510e+07))} - lnT2;")
            L.append("const float Tf = (float)Tv, invTf = (float)invT, lnT2f = (float)lnT2;")
        for k, sp in enumerate(self.mech.species):
            lo, hi = smh_coefs(sp.nasa_low), smh_coefs(sp.nasa_high)
            if lo == hi:
                sel, pre = [_d(x) for x in lo], ""
            else:
                pre = f"const bool lo{k} = Tv < {_d(sp.t_ranges[1])}; "
                sel = [f"(lo{k} ? {_d(a)} : {_d(b)})" for a, b in zip(lo, hi)]
            poly = (f"fma(fma(fma(fma({sel[5]}, Tv, {sel[4]}), Tv, {sel[3]}), Tv, {sel[2]}), Tv, "
                    f"fma({sel[1]}, lnT, {sel[0]})) - {sel[6]} * invT")
            if not mixed:
                Ts = [200.0 + 50.0 * j for j in range(117)]
                vals = []
                for t in Ts:
                    c = lo if t < sp.t_ranges[1] else hi
                    vals.append(c[0] + c[1] * math.log(t) + c[2] * t + c[3] * t * t + c[4] * t ** 3
                                + c[5] * t ** 4 - c[6] / t)
                fn = "cgm::cg_exp" if max(abs(v) for v in vals) < 690.0 else "cgm::cg_exp_clamped"
                if self.tmem:
                    L.append(f"{{ {pre}cgg::tm_st(tw + {2 * k}u, {fn}({poly}) * pfac); }}")
                else:
                    L.append(f"{{ {pre}sE[{k}][t] = {fn}({poly}) * pfac; }}")
            else:
                if self.tmem:
                    L.append(f"{{ {pre}cgg::tm_st(tw + {2 * k}u, fma({poly}, {_d(LOG2E)}, lpfac2)); }}")
                else:
                    L.append(f"{{ {pre}sG[{k}][t] = fma({poly}, {_d(LOG2E)}, lpfac2); }}")
        if self.tmem:
            L.append("cgg::tm_wait_st();")
        if self.reg_w and self.live_order:
            pass                                   # declared at first touch (kernel())
        elif self.reg_w:
            L.append("double " + ", ".join(f"w{k} = 0.0" for k in range(ns)) + ";")
        else:
            for k in range(ns):
                L.append(f"sW[{k}][t] = 0.0;")
        return L

    def epilogue(self) -> List[str]:
        L = ["if (act) {"]
        for k in range(self.ns):
            w = f"w{k}" if self.reg_w else f"sW[{k}][t]"
            L.append(f"  {self.st(f'(int64_t){k} * ng + i', w)}")
        L.append("}")
        return L

    def smem_bytes(self, mixed: bool) -> int:
        return smem_per_species(mixed, self.tmem, self.reg_w) * self.ns * self.block

    def kernel(self, mixed: bool) -> str:
        ns, B = self.ns, self.block
        name = "cg_gen_mixed" if mixed else "cg_gen_fp64"
        L = [f"__global__ void __launch_bounds__({B}, 1) {name}(const double* __restrict__ P, "
             "const double* __restrict__ T, const double* __restrict__ Y, double* __restrict__ wdot, int64_t ng) {"]
        # dynamic shared memory: [array][species][thread]
        L.append("  extern __shared__ __align__(16) unsigned char dsm[];")
        if not mixed and self.tmem:
            L.append(f"  double (*sC)[{B}] = reinterpret_cast<double (*)[{B}]>(dsm);")
            L.append("  __shared__ uint32_t tm_slot;")
            L.append(f"  const uint32_t tbase = cgg::tm_alloc(&tm_slot, {self.tmem_cols()}u);")
            L.append(f"  const uint32_t tw = cgg::tm_thread_base(tbase, {2 * ns});")
            off = ns * B * 8
        elif not mixed:
            L.append(f"  double (*sC)[{B}] = reinterpret_cast<double (*)[{B}]>(dsm);")
            L.append(f"  double (*sE)[{B}] = reinterpret_cast<double (*)[{B}]>(dsm + {ns * B * 8});")
            off = 2 * ns * B * 8
        elif self.tmem:
            L.append(f"  float (*sc)[{B}] = reinterpret_cast<float (*)[{B}]>(dsm);")
            L.append("  __shared__ uint32_t tm_slot;")
            L.append(f"  const uint32_t tbase = cgg::tm_alloc(&tm_slot, {self.tmem_cols()}u);")
            L.append(f"  const uint32_t tw = cgg::tm_thread_base(tbase, {2 * ns});")
            off = ns * B * 4
        else:
            L.append(f"  double (*sG)[{B}] = reinterpret_cast<double (*)[{B}]>(dsm);")
            L.append(f"  float (*sc)[{B}] = reinterpret_cast<float (*)[{B}]>(dsm + {ns * B * 8});")
            off = ns * B * 12
        if not self.reg_w:
            L.append(f"  double (*sW)[{B}] = reinterpret_cast<double (*)[{B}]>(dsm + {off});")
        L += ["  " + x for x in self.prologue(mixed)]
        order = reaction_order(self.mech) if self.live_order else list(range(self.mech.nr))
        last = {}
        for p, j in enumerate(order):
            r = self.mech.reactions[j]
            for sp in list(r.reactants) + list(r.products):
                last[self.idx[sp]] = p
        declared = set()
        rev_pos = [p for p, j in enumerate(order) if self.mech.reactions[j].reversible] if (
            self.tm_prefetch and not mixed) else []
        if rev_pos:
            L += ["  " + x for x in self.issue_egp(order[rev_pos[0]], self.mech.reactions[order[rev_pos[0]]])]
        next_rev = {a: b for a, b in zip(rev_pos, rev_pos[1:])}
        for p, j in enumerate(order):
            r = self.mech.reactions[j]
            if p and self.sync_every and p % self.sync_every == 0:
                # keep the block's warps on the same stretch of code so they
                # share instruction fetches (the kernel is straight-line)
                L.append("  __syncthreads();")
            if self.live_order:
                new = [self.idx[sp] for sp in dict.fromkeys(list(r.reactants) + list(r.products))
                       if self.idx[sp] not in declared]
                if new:
                    L.append("  double " + ", ".join(f"w{k} = 0.0" for k in new) + ";")
                    declared.update(new)
            if self.egp_group > 1 and p % self.egp_group == 0:
                L += ["  " + x for x in self.group_egp(p, [self.mech.reactions[jj]
                                                            for jj in order[p:p + self.egp_group]])]
            if rev_pos and r.reversible:
                L += ["  " + x for x in self.wait_egp(j, r)]
                if p in next_rev:
                    jn = order[next_rev[p]]
                    L += ["  " + x for x in self.issue_egp(jn, self.mech.reactions[jn])]
            body = self.reaction32(r) if mixed else self.reaction64(r)
            if self.exp_noinline:
                body = [x.replace("cgm::cg_exp_clamped(", "cgm::cg_exp_clamped_ool(").replace(
                    "cgm::cg_exp(", "cgm::cg_exp_ool(") for x in body]
            L += ["  " + x for x in body]
            if self.live_order:
                done = [k for k in sorted(set(self.idx[sp] for sp in list(r.reactants) + list(r.products)))
                        if last[k] == p]
                if done:
                    L.append("  if (act) { " + " ".join(self.st(f"(int64_t){k} * ng + i", f"w{k}") for k in done)
                             + " }")
        if self.live_order:
            untouched = [k for k in range(ns) if k not in declared]
            if untouched:
                L.append("  if (act) { " + " ".join(self.st(f"(int64_t){k} * ng + i", "0.0") for k in untouched)
                         + " }")
        else:
            L += ["  " + x for x in self.epilogue()]
        if self.tmem:
            L.append(f"  cgg::tm_free(tbase, {self.tmem_cols()}u);")
        L.append("}")
        return "\n".join(L)


def smem_per_species(mixed: bool, tmem: bool, reg_w: bool) -> int:
    """Shared-memory bytes per species and point: C (FP64) and EGp, or, for
    the mixed kernel, C (FP32) and the log2 Gibbs terms (FP64); the second
    array leaves for tensor memory in tmem mode; wdot when not in registers."""
    per = (4 if tmem else 12) if mixed else (8 if tmem else 16)
    return per + (0 if reg_w else 8)


def choose_block(ns: int, mixed: bool, tmem: bool = False) -> int:
    """Threads per block; one block per SM, so this is also the SM's resident
    points.  The straight-line kernels are latency-bound: resident warps pay
    off until the per-point state (shared and tensor memory) or the registers
    run out.  Registers: two per FP64 accumulator plus temporaries (~64 when
    the Gibbs array is in shared memory, whose loads the compiler hoists;
    ~20 when batched tensor-memory loads replace them).  Measured on B200 at
    53/325: FP64 8 warps 394, 12 warps (tensor memory) 468, 16 warps 510
    Mpts/s; mixed 8 warps 624, 11 warps 775 Mpts/s; at 24/325 FP64 8 -> 16
    warps 450 -> 850 Mpts/s."""
    reg_w = ns <= MAX_REG_SPECIES
    per = smem_per_species(mixed, tmem, reg_w) * ns
    regs = (2 * ns if reg_w else 0) + (20 if tmem else 64)
    b = min(SMEM_BUDGET // per, REG_FILE // regs, MAX_BLOCK) // 32 * 32
    if tmem:
        while b > 32 and -(-b // 128) * 2 * ns > 512:     # 512 tensor-memory columns per SM
            b -= 32
    return max(b, 32)


def use_tmem(ns: int, mixed: bool = False) -> bool:
    """The per-point Gibbs array (EGp for the FP64 kernel, the log2 Gibbs
    terms for the mixed one) moves to tensor memory when that lets the block
    grow and the columns fit.  Measured on B200 at 53/325, 2^20 points, with
    the streaming input/output hints: mixed 16 warps (tensor memory) 1055
    against 11 warps (shared memory) 830 Mpts/s.  Before those hints the
    kernels were bound by instruction fetches from DRAM and the shared-memory
    form had won (795 against 761-770)."""
    if ns > MAX_REG_SPECIES:
        return False
    b = choose_block(ns, mixed, True)
    return b > choose_block(ns, mixed) and -(-b // 128) * 2 * ns <= 512


PRECISIONS = {"fp64": (True, False), "mixed": (False, True), "both": (True, True)}


def emit(mech: Mechanism, name: Optional[str] = None, block: Optional[int] = None,
         sync_every: Optional[int] = None, precision: str = "both", tmem: Optional[bool] = None,
         live_order: bool = True, exp_noinline: bool = False, live_order_mixed: Optional[bool] = False,
         tm_prefetch: bool = False, egp_group: Optional[int] = None, egp_group_mixed: int = 1,
         stream_io: bool = True) -> str:
    """CUDA source of the mechanism's kernels: `precision` selects the FP64
    kernel, the mixed one or both; a mode without a generated kernel runs on
    the table-driven kernels."""
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    want64, want32 = PRECISIONS[precision]
    blob = pack(mech).to_blob()
    fp = fingerprint(blob)
    tm64 = use_tmem(mech.ns, False) if tmem is None else tmem
    tm32 = use_tmem(mech.ns, True) if tmem is None else tmem
    em64 = _Emitter(mech, block or choose_block(mech.ns, False, tm64),
                    SYNC_EVERY if sync_every is None else sync_every, tmem=tm64, live_order=live_order,
                    exp_noinline=exp_noinline, tm_prefetch=tm_prefetch,
                    egp_group=EGP_GROUP if egp_group is None else egp_group, stream_io=stream_io)
    # the mixed kernel keeps file order unless asked: on B200 at 53/325 the live-range order made
    # the FP64 kernel 5 % faster (497 -> 522 Mpts/s) and the mixed one 2 % slower (794 -> 777)
    em32 = _Emitter(mech, block or choose_block(mech.ns, True, tm32),
                    SYNC_EVERY_MIXED if sync_every is None else sync_every, tmem=tm32,
                    live_order=live_order if live_order_mixed is None else live_order_mixed,
                    exp_noinline=exp_noinline, egp_group=egp_group_mixed, stream_io=stream_io)
    ident = "".join(ch if ch.isalnum() else "_" for ch in (name or mech.name))
    src = [
        f"// Generated by chemgen_b200 (generate_chemistry.py --language cuda --precision {precision}) for mechanism '{mech.name}':",
        f"// {mech.ns} species, {mech.nr} reactions {mech.counts()}.",
        f"// Blob fingerprint 0x{fp:016x}.  Target: sm_100a.",
        '#include "gen_common.cuh"',
        '#include "cg_math.cuh"',
        "using cgg::rcp;",
        "namespace {",
    ]
    attrs, dispatch = [], []
    for want, em, mixed, kname, mname in ((want64, em64, False, "cg_gen_fp64", "CHEMGEN_MODE_FP64"),
                                          (want32, em32, True, "cg_gen_mixed", "CHEMGEN_MODE_MIXED")):
        if not want:
            continue
        B = em.block
        src += [em.kernel(mixed), ""]
        attrs.append(f"cudaFuncSetAttribute({kname}, cudaFuncAttributeMaxDynamicSharedMemorySize, "
                     f"{em.smem_bytes(mixed)}) != cudaSuccess")
        dispatch.append(f"  if (mode == {mname}) {{ {kname}<<<(unsigned)((ng + {B - 1}) / {B}), {B}, "
                        f"{em.smem_bytes(mixed)}, st>>>"
                        "(P, T, Y, wdot, ng); return cudaGetLastError() == cudaSuccess ? CHEMGEN_OK : CHEMGEN_ERR_CUDA; }")
    modes = (1 if want64 else 0) | (2 if want32 else 0)
    src += [
        "int launch(int mode, const double* P, const double* T, int64_t ng, const double* Y, double* wdot, void* s) {",
        "  if (ng <= 0) return CHEMGEN_OK;",
        "  static bool attrs = false;",
        "  if (!attrs) {",
        "    if (" + " ||\n        ".join(attrs) + ")",
        "      return CHEMGEN_ERR_CUDA;",
        "    attrs = true;",
        "  }",
        "  cudaStream_t st = (cudaStream_t)s;",
    ] + dispatch + [
        "  return CHEMGEN_ERR_INVALID_ARGUMENT;",
        "}",
        "",
        "struct Register {",
        f"  Register() {{ chemgen_register_kernels(0x{fp:016x}ull, {mech.ns}, {mech.nr}, {modes}u, &launch); }}",
        "} register_once;",
        "}  // namespace",
        "",
        f'extern "C" unsigned long long chemgen_generated_fingerprint_{ident}(void) {{ return 0x{fp:016x}ull; }}',
        "// direct entry point of this module (the same call chemgen_getrates_ex dispatches to)",
        f'extern "C" int chemgen_generated_getrates_{ident}(int mode, const double* P, const double* T, int64_t ng,',
        "                                              const double* Y, double* wdot, void* stream) {",
        "  return launch(mode, P, T, ng, Y, wdot, stream);",
        "}",
    ]
    return "\n".join(src) + "\n"


HERE = os.path.dirname(os.path.abspath(__file__))
GEN_DIR = os.path.join(HERE, "_generated")


def codegen_version() -> str:
    """Short hash of this emitter and the headers generated code includes, so
    that a change to either gives built modules a new name (and a rebuild)."""
    h = hashlib.sha256()
    files = [os.path.abspath(__file__)] + [os.path.join(HERE, "csrc", f) for f in
                                           ("gen_common.cuh", "cg_math.cuh")]
    files.append(os.path.join(os.path.dirname(HERE), "include", "chemgen_b200.h"))
    for f in files:
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:8]


def module_path(mech: Mechanism) -> str:
    fp = fingerprint(pack(mech).to_blob())
    return os.path.join(GEN_DIR, f"libcg_{fp:016x}_{codegen_version()}.so")


def build_module(mech: Mechanism, out: Optional[str] = None, verbose: bool = False, keep_source: bool = True,
                 **emit_args) -> str:
    """Emit and compile the mechanism's kernels into a shared library that
    links libchemgen_b200.so and registers itself when loaded."""
    from .build import ARCH, FLAGS, OUT as LIBMAIN, nvcc
    os.makedirs(GEN_DIR, exist_ok=True)
    so = out or module_path(mech)
    src = so[:-3] + ".cu"
    text = emit(mech, **emit_args)
    with open(src, "w") as f:
        f.write(text)
    cmd = [nvcc()] + ARCH + FLAGS + ["-I", os.path.join(HERE, "csrc"), "-shared", "-o", so, src,
                                     "-L", os.path.dirname(LIBMAIN), "-lchemgen_b200",
                                     "-Xlinker", "-rpath=$ORIGIN/..", "-Xlinker", "-rpath=$ORIGIN",
                                     "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on generated {src}:\n{r.stdout}\n{r.stderr[-4000:]}")
    if verbose and r.stderr:
        print(r.stderr)
    return so
