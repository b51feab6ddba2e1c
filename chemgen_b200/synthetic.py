"""Seeded synthetic mechanisms and thermochemical states.

The workloads are described by size only (53 species / 325 reactions,
348 / 2163, a ~10-species H2/O2 set), so they are generated here from a seed
and are identical on every machine.  Rules:

* NASA-7 two-range thermo: cp/R = c0 + c1 (T/1000) + c2 (T/1000)^2 (+ tiny
  a4/a5 terms so every coefficient is exercised); the high range is a second
  draw made continuous in h and s at Tmid = 1000 K;
* Arrhenius A log-uniform in [1e6, 1e17] (cgs), b in [-2, 3], Ea in
  [0, 50] kcal/mol; falloff k0 = A * 10^U(2,7);
* every reaction is oriented exothermic in the forward direction, so the
  reverse rate kf/Kc carries an activation energy of Ea + |dH| (a random
  endothermic reaction with Ea = 0 would produce reverse rates no real
  mechanism has); reactions with max |d(g/RT)| > 300 over 300..2500 K (real
  mechanisms reach about 314) or with ln Kc < -20 anywhere in that range
  (a reverse rate above e^20 kf, which random entropy differences can
  produce) are redrawn;
* states: T ~ U(300, 2500) K, P = 1 atm * exp(U(0, ln 40)) in dyne/cm^2,
  Y ~ Dirichlet(0.5), float64, species-major (``Y[k, i]``).
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Tuple

import numpy as np

from .mechanism import PATM, Mechanism, Reaction, Species

_ELEMENTS = ("C", "H", "O", "N")


def _thermo(rng: np.random.Generator):
    tmid = 1000.0

    def poly(c0, c1, c2, a4, a5):
        return [c0, c1 / 1000.0, c2 / 1.0e6, a4, a5]

    lo = poly(rng.uniform(2.5, 4.0), rng.uniform(0.0, 6.0), rng.uniform(-1.5, 0.0),
              rng.uniform(-1, 1) * 1e-10, rng.uniform(-1, 1) * 1e-14)
    hi = poly(rng.uniform(3.0, 6.0), rng.uniform(0.0, 3.0), rng.uniform(-0.5, 0.0),
              rng.uniform(-1, 1) * 1e-12, rng.uniform(-1, 1) * 1e-16)
    a6 = float(np.clip(rng.normal(5000.0, 25000.0), -60000.0, 100000.0))
    a7 = rng.uniform(-5.0, 25.0)

    def h_poly(a, T):
        return a[0] * T + a[1] / 2 * T ** 2 + a[2] / 3 * T ** 3 + a[3] / 4 * T ** 4 + a[4] / 5 * T ** 5

    def s_poly(a, T):
        return a[0] * math.log(T) + a[1] * T + a[2] / 2 * T ** 2 + a[3] / 3 * T ** 3 + a[4] / 4 * T ** 4

    a6_hi = h_poly(lo, tmid) + a6 - h_poly(hi, tmid)
    a7_hi = s_poly(lo, tmid) + a7 - s_poly(hi, tmid)
    return (200.0, tmid, 5000.0), tuple(lo + [a6, a7]), tuple(hi + [a6_hi, a7_hi])


def _smh(sp: Species, T: np.ndarray) -> np.ndarray:
    out = np.empty_like(T)
    for sel, a in ((T < sp.t_ranges[1], sp.nasa_low), (T >= sp.t_ranges[1], sp.nasa_high)):
        t = T[sel]
        out[sel] = (a[6] - a[0] + a[0] * np.log(t) + a[1] / 2 * t + a[2] / 6 * t ** 2 + a[3] / 12 * t ** 3
                    + a[4] / 20 * t ** 4 - a[5] / t)
    return out


def _hrt(sp: Species, T: float) -> float:
    a = sp.nasa_low if T < sp.t_ranges[1] else sp.nasa_high
    return a[0] + a[1] / 2 * T + a[2] / 3 * T ** 2 + a[3] / 4 * T ** 3 + a[4] / 5 * T ** 4 + a[5] / T


def _arrhenius(rng: np.random.Generator) -> Tuple[float, float, float]:
    return (float(10.0 ** rng.uniform(6.0, 17.0)), float(rng.uniform(-2.0, 3.0)),
            float(rng.uniform(0.0, 50000.0)))


def synthetic_mechanism(ns: int, nr: int, n_third_body: int, n_troe: int, seed: int = 0,
                        frac_reversible: float = 0.7, n_lindemann: int = 0, n_sri: int = 0,
                        n_plog: int = 0, species_names: Optional[List[str]] = None,
                        name: Optional[str] = None) -> Mechanism:
    rng = np.random.default_rng(seed)
    names = species_names or [f"S{i}" for i in range(ns)]
    species = []
    for n in names:
        comp = {e: float(c) for e, c in zip(_ELEMENTS, rng.integers(0, 4, size=4)) if c}
        if not comp:
            comp = {"H": 1.0}
        tr, lo, hi = _thermo(rng)
        species.append(Species(name=n, composition=comp, t_ranges=tr, nasa_low=lo, nasa_high=hi))
    Tgrid = np.linspace(300.0, 2500.0, 45)
    smh = {s.name: _smh(s, Tgrid) for s in species}
    # a few "radical" hub species appear more often, as in real mechanisms
    weights = rng.gamma(0.7, size=ns)
    weights /= weights.sum()

    kinds = (["third_body"] * n_third_body + ["troe"] * n_troe + ["lindemann"] * n_lindemann
             + ["sri"] * n_sri + ["plog"] * n_plog)
    kinds += ["standard"] * (nr - len(kinds))
    order = rng.permutation(len(kinds))
    kinds = [kinds[i] for i in order]
    reactions: List[Reaction] = []
    for kind in kinds:
        while True:
            if kind in ("third_body", "troe", "lindemann", "sri"):
                nreac, nprod = (2, 1) if rng.random() < 0.5 else (1, 2)
            else:
                nreac = int(rng.choice([1, 2, 3], p=[0.1, 0.8, 0.1]))
                nprod = int(rng.choice([1, 2, 3], p=[0.15, 0.75, 0.1]))
            picks = rng.choice(ns, size=nreac + nprod, p=weights)
            reac: Dict[str, float] = {}
            prod: Dict[str, float] = {}
            for k in picks[:nreac]:
                reac[names[k]] = reac.get(names[k], 0.0) + 1.0
            for k in picks[nreac:]:
                prod[names[k]] = prod.get(names[k], 0.0) + 1.0
            if set(reac) == set(prod) and all(reac[s] == prod[s] for s in reac):
                continue
            d = sum(n * smh[s] for s, n in prod.items()) - sum(n * smh[s] for s, n in reac.items())
            if np.abs(d).max() > 300.0:
                continue
            dh = sum(n * _hrt(species[names.index(s)], 1000.0) for s, n in prod.items()) \
                - sum(n * _hrt(species[names.index(s)], 1000.0) for s, n in reac.items())
            if dh > 0.0:
                reac, prod = prod, reac
                d = -d
            # ln Kc (concentration units) = d(smh) + dnu ln(Patm/(R0 T))
            dnu = sum(prod.values()) - sum(reac.values())
            lnkc = d + dnu * np.log(PATM / (8.314510e07 * Tgrid))
            if lnkc.min() < -20.0:
                continue
            break
        rev = bool(rng.random() < frac_reversible)
        arh = _arrhenius(rng)
        eqn = " + ".join(reac) + (" <=> " if rev else " => ") + " + ".join(prod)
        r = Reaction(eqn, kind, reac, prod, rev, False, arh=arh)
        if kind in ("third_body", "troe", "lindemann", "sri"):
            nk = int(rng.integers(0, 7))
            ks = rng.choice(ns, size=nk, replace=False)
            r.efficiencies = {names[k]: float(np.round(rng.uniform(0.0, 6.0), 2)) - 1.0 for k in ks}
            r.efficiencies = {k: v for k, v in r.efficiencies.items() if v != 0.0}
        if kind in ("troe", "lindemann", "sri"):
            A, b, Ea = arh
            r.low = (A * 10.0 ** rng.uniform(2.0, 7.0), float(np.clip(b + rng.uniform(-2.0, 0.0), -2.0, 3.0)),
                     float(rng.uniform(0.0, 50000.0)))
        if kind == "troe":
            params = (float(rng.uniform(0.3, 0.9)), float(rng.uniform(50.0, 1000.0)),
                      float(rng.uniform(500.0, 10000.0)))
            if rng.random() < 0.5:
                params = params + (float(rng.uniform(1000.0, 10000.0)),)
            r.troe = params
        if kind == "sri":
            r.sri = (float(rng.uniform(0.5, 2.0)), float(rng.uniform(100.0, 1000.0)),
                     float(rng.uniform(500.0, 3000.0)), float(rng.uniform(0.5, 1.5)),
                     float(rng.uniform(-0.5, 0.5)))
        if kind == "plog":
            npts = int(rng.integers(2, 5))
            ps = np.sort(PATM * 10.0 ** rng.uniform(-2.0, 2.0, size=npts))
            r.plog = [(float(p),) + _arrhenius(rng) for p in ps]
        reactions.append(r)
    mech = Mechanism(name=name or f"synthetic_{ns}_{nr}_s{seed}", species=species, reactions=reactions)
    mech.validate()
    return mech


# Named workloads -------------------------------------------------------------

def h2o2_10sp(seed: int = 1) -> Mechanism:
    """~10-species H2/O2 set: 27 reversible reactions, 4 three-body, 2 Troe."""
    names = ["H2", "O2", "H2O", "H", "O", "OH", "HO2", "H2O2", "N2", "AR"]
    return synthetic_mechanism(10, 27, 4, 2, seed=seed, frac_reversible=1.0, species_names=names,
                               name="synthetic_h2o2_10_27")


def gri_shape(seed: int = 2) -> Mechanism:
    """53 species / 325 reactions: 28 three-body, 29 Troe, ~70% reversible."""
    return synthetic_mechanism(53, 325, 28, 29, seed=seed, name="synthetic_53_325")


def jetsurf_shape(seed: int = 3) -> Mechanism:
    """348 species / 2163 reactions: ~10% Troe falloff, ~8% three-body."""
    return synthetic_mechanism(348, 2163, 173, 216, seed=seed, name="synthetic_348_2163")


def all_kinds(seed: int = 4) -> Mechanism:
    """Small mechanism with every supported reaction kind (incl. Lindemann,
    SRI and PLOG) for parity tests."""
    return synthetic_mechanism(20, 60, 6, 6, seed=seed, n_lindemann=4, n_sri=4, n_plog=6,
                               name="synthetic_all_kinds")


def states(ns: int, ng: int, seed: int = 0) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(P[ng] dyne/cm^2, T[ng] K, Y[ns, ng]) with the distributions above."""
    rng = np.random.default_rng(seed)
    T = rng.uniform(300.0, 2500.0, size=ng)
    P = PATM * np.exp(rng.uniform(0.0, math.log(40.0), size=ng))
    Y = rng.dirichlet(np.full(ns, 0.5), size=ng).T.copy()
    Y /= Y.sum(axis=0, keepdims=True)
    return P, T, np.ascontiguousarray(Y)


def miniapp_states(ns: int, ng: int, seed: int = 0) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The reference mini-app's distribution (chemistry_mini_app.j2:37-44):
    T ~ U(300, 2000), P = 1 atm, Y_k ~ U(0, 1/(ns-1)) with the last species the
    remainder."""
    rng = np.random.default_rng(seed)
    T = rng.uniform(300.0, 2000.0, size=ng)
    P = np.full(ng, PATM)
    Y = np.empty((ns, ng))
    Y[:-1] = rng.uniform(0.0, 1.0 / (ns - 1), size=(ns - 1, ng))
    Y[-1] = 1.0 - Y[:-1].sum(axis=0)
    return P, T, Y
