"""Mechanism intermediate representation and the Cantera-free YAML front end.

The reference parses mechanisms through Cantera (``chemgen/parser.py:55-187``)
and converts every rate to cgs units with pint (``chemgen/parser.py:152-159``).
Neither library is part of this package, so this module reads the ck2yaml/
Cantera YAML format itself and applies the same conventions:

* reaction types ``standard`` / ``third_body`` / ``troe`` / ``plog``
  (``chemgen/parser.py:44-49``), plus ``lindemann`` and ``sri`` falloff, which
  the reference silently drops (``chemgen/parser.py:146-147``).  Passing
  ``reference_compat=True`` drops them too, so that a mechanism can be compared
  one-for-one against code the reference generates;
* third-body efficiencies stored as ``eff - 1`` for the species whose
  efficiency differs from one (``chemgen/parser.py:97,131``);
* a three-body reaction written with an explicit collider instead of ``M``
  becomes an elementary reaction with the collider on both sides
  (``chemgen/parser.py:107-130``);
* A in (cm^3/mol)^(order-1)/s, Ea in cal/mol, PLOG pressures in dyne/cm^2;
* species order = phase species order (``chemgen/chemistry.py:39-46``).

Gas constants are the CODATA-1986 values the reference hard-codes
(``chemgen/chemistry.py:204-206``).
"""
from __future__ import annotations

import dataclasses
import json
import math
import re
from typing import Dict, List, Optional, Sequence, Tuple

import yaml

# chemgen/chemistry.py:204-206
RC_CAL = 1.9872155832          # cal/(mol K)
R0_ERG = 8.314510e07           # erg/(mol K)
PATM = 1013250.0               # dyne/cm^2

# Standard atomic weights (IUPAC, abridged, g/mol).  Cantera's own table is not
# available here; molecular weights are therefore an input of every parity
# comparison rather than something checked against Cantera.
ATOMIC_WEIGHTS = {
    "H": 1.008, "D": 2.014101778, "T": 3.0160492779, "He": 4.002602, "Li": 6.94, "Be": 9.0121831,
    "B": 10.81, "C": 12.011, "N": 14.007, "O": 15.999, "F": 18.998403163,
    "Ne": 20.1797, "Na": 22.98976928, "Mg": 24.305, "Al": 26.9815385,
    "Si": 28.085, "P": 30.973761998, "S": 32.06, "Cl": 35.45, "Ar": 39.95,
    "K": 39.0983, "Ca": 40.078, "Ti": 47.867, "Cr": 51.9961, "Fe": 55.845,
    "Ni": 58.6934, "Cu": 63.546, "Zn": 65.38, "Br": 79.904, "Kr": 83.798,
    "I": 126.90447, "Xe": 131.293, "E": 5.48579909e-4,
}

REACTION_KINDS = ("standard", "third_body", "lindemann", "troe", "sri", "plog")


def _element_key(name: str) -> str:
    for key in ATOMIC_WEIGHTS:
        if key.lower() == name.lower():
            return key
    raise ValueError(f"unknown element {name!r}")


@dataclasses.dataclass
class Species:
    name: str
    composition: Dict[str, float]
    t_ranges: Tuple[float, float, float]          # (Tmin, Tmid, Tmax)
    nasa_low: Tuple[float, ...]                    # a1..a7 below Tmid
    nasa_high: Tuple[float, ...]                   # a1..a7 at/above Tmid
    mw: float = 0.0

    def __post_init__(self):
        if not self.mw:
            self.mw = sum(ATOMIC_WEIGHTS[_element_key(e)] * n for e, n in self.composition.items())


@dataclasses.dataclass
class Reaction:
    """One reaction in reference conventions (``chemgen/parser.py:70-145``)."""
    equation: str
    kind: str                                      # one of REACTION_KINDS
    reactants: Dict[str, float]
    products: Dict[str, float]
    reversible: bool = True
    duplicate: bool = False
    arh: Tuple[float, float, float] = (0.0, 0.0, 0.0)   # (A cgs, b, Ea cal/mol); kinf for falloff
    low: Optional[Tuple[float, float, float]] = None    # k0 for falloff
    troe: Optional[Tuple[float, ...]] = None             # (a, T3, T1[, T2])
    sri: Optional[Tuple[float, ...]] = None              # (a, b, c[, d, e])
    efficiencies: Dict[str, float] = dataclasses.field(default_factory=dict)  # eff - 1
    plog: Optional[List[Tuple[float, float, float, float]]] = None  # (P dyne/cm2, A, b, Ea)

    @property
    def uses_m(self) -> bool:
        return self.kind in ("third_body", "lindemann", "troe", "sri")

    @property
    def is_falloff(self) -> bool:
        return self.kind in ("lindemann", "troe", "sri")

    @property
    def dnu(self) -> float:
        """coeff_sum of ``chemgen/chemistry.py:276``: sum(nu_prod) - sum(nu_reac)."""
        return sum(self.products.values()) - sum(self.reactants.values())


@dataclasses.dataclass
class Mechanism:
    name: str
    species: List[Species]
    reactions: List[Reaction]
    dropped: List[str] = dataclasses.field(default_factory=list)

    @property
    def ns(self) -> int:
        return len(self.species)

    @property
    def nr(self) -> int:
        return len(self.reactions)

    @property
    def species_names(self) -> List[str]:
        return [s.name for s in self.species]

    def species_index(self) -> Dict[str, int]:
        return {s.name: i for i, s in enumerate(self.species)}

    def counts(self) -> Dict[str, int]:
        out = {k: 0 for k in REACTION_KINDS}
        for r in self.reactions:
            out[r.kind] += 1
        out["reversible"] = sum(r.reversible for r in self.reactions)
        return out

    def mw(self) -> List[float]:
        return [s.mw for s in self.species]

    # ------------------------------------------------------------------ json
    def to_json(self) -> str:
        return json.dumps(dataclasses.asdict(self))

    @staticmethod
    def from_json(text: str) -> "Mechanism":
        d = json.loads(text)
        species = [Species(name=s["name"], composition=s["composition"],
                           t_ranges=tuple(s["t_ranges"]), nasa_low=tuple(s["nasa_low"]),
                           nasa_high=tuple(s["nasa_high"]), mw=s["mw"]) for s in d["species"]]
        reactions = []
        for r in d["reactions"]:
            r = dict(r)
            for key in ("arh", "low", "troe", "sri"):
                if r.get(key) is not None:
                    r[key] = tuple(r[key])
            if r.get("plog") is not None:
                r["plog"] = [tuple(p) for p in r["plog"]]
            reactions.append(Reaction(**r))
        return Mechanism(name=d["name"], species=species, reactions=reactions,
                         dropped=d.get("dropped", []))

    def validate(self) -> None:
        idx = self.species_index()
        for r in self.reactions:
            if r.kind not in REACTION_KINDS:
                raise ValueError(f"bad reaction kind {r.kind!r} in {r.equation}")
            for side in (r.reactants, r.products):
                for sp, nu in side.items():
                    if sp not in idx:
                        raise ValueError(f"reaction {r.equation!r}: unknown species {sp!r}")
                    if not (nu > 0):
                        raise ValueError(f"reaction {r.equation!r}: bad coefficient {nu}")
            for sp in r.efficiencies:
                if sp not in idx:
                    raise ValueError(f"reaction {r.equation!r}: unknown collider {sp!r}")
            if r.is_falloff and r.low is None:
                raise ValueError(f"falloff reaction {r.equation!r} without low-pressure rate")
            if r.kind == "troe" and (r.troe is None or len(r.troe) not in (3, 4)):
                raise ValueError(f"Troe reaction {r.equation!r} needs 3 or 4 parameters")
            if r.kind == "sri" and (r.sri is None or len(r.sri) not in (3, 5)):
                raise ValueError(f"SRI reaction {r.equation!r} needs 3 or 5 parameters")
            if r.kind == "plog" and not r.plog:
                raise ValueError(f"PLOG reaction {r.equation!r} without rates")


# ---------------------------------------------------------------------- YAML
class _Yaml12Loader(yaml.SafeLoader):
    """SafeLoader with YAML-1.2 scalars: only true/false are booleans (so a
    species called ``NO`` stays a string) and ``1e5`` is a float."""


_Yaml12Loader.yaml_implicit_resolvers = {
    k: [(tag, rx) for tag, rx in v if tag not in ("tag:yaml.org,2002:bool", "tag:yaml.org,2002:float")]
    for k, v in yaml.SafeLoader.yaml_implicit_resolvers.items()
}
_Yaml12Loader.add_implicit_resolver(
    "tag:yaml.org,2002:bool", re.compile(r"^(?:true|True|TRUE|false|False|FALSE)$"), list("tTfF"))
_Yaml12Loader.add_implicit_resolver(
    "tag:yaml.org,2002:float",
    re.compile(r"""^(?:[-+]?(?:\.[0-9]+|[0-9]+(?:\.[0-9]*)?)(?:[eE][-+]?[0-9]+)?
                  |[-+]?\.(?:inf|Inf|INF)|\.(?:nan|NaN|NAN))$""", re.X),
    list("-+0123456789."))


def load_yaml_text(text: str):
    return yaml.load(text, Loader=_Yaml12Loader)


_LENGTH_CM = {"cm": 1.0, "m": 100.0, "mm": 0.1}
_QUANTITY_MOL = {"mol": 1.0, "kmol": 1000.0, "molec": 1.0 / 6.02214076e23, "molecule": 1.0 / 6.02214076e23}
_TIME_S = {"s": 1.0, "ms": 1e-3, "min": 60.0, "hr": 3600.0}
_ENERGY_CAL_PER_MOL = {
    "cal/mol": 1.0, "kcal/mol": 1000.0, "J/mol": 1.0 / 4.184, "kJ/mol": 1000.0 / 4.184,
    "J/kmol": 1.0 / 4184.0, "kJ/kmol": 1.0 / 4.184,
    # Ea given as Ea/R in kelvin, converted with Cantera's gas constant then to cal/mol
    "K": 8314.462618 / 4184.0,
    "eV": 96485.33212 / 4.184,
}
_PRESSURE_DYNE = {"Pa": 10.0, "kPa": 1e4, "MPa": 1e7, "bar": 1e6, "atm": 1013250.0,
                  "torr": 1013250.0 / 760.0, "dyn/cm^2": 1.0}


def _with_unit(value, table, default_factor, what):
    """Number or ``"<number> <unit>"`` string -> value scaled by the unit."""
    if isinstance(value, (int, float)):
        return float(value) * default_factor
    parts = str(value).split(None, 1)
    num = float(parts[0])
    if len(parts) == 1:
        return num * default_factor
    unit = parts[1].strip()
    if unit not in table:
        raise ValueError(f"unsupported {what} unit {unit!r}")
    return num * table[unit]


class _Units:
    def __init__(self, units: Optional[dict]):
        units = units or {}
        self.length = _LENGTH_CM[units.get("length", "m")]
        self.quantity = _QUANTITY_MOL[units.get("quantity", "kmol")]
        self.time = _TIME_S[units.get("time", "s")]
        self.energy = _ENERGY_CAL_PER_MOL[units.get("activation-energy", "J/kmol")]
        self.pressure = _PRESSURE_DYNE[units.get("pressure", "Pa")]
        # concentration unit of the file in mol/cm^3
        self.conc = self.quantity / self.length ** 3

    def rate(self, rc: dict, order: float) -> Tuple[float, float, float]:
        """(A, b, Ea) -> cgs; same rule as chemgen/parser.py:152-159."""
        if not isinstance(rc, dict):
            raise ValueError(f"unsupported rate-constant {rc!r}")
        raw = rc["A"]
        if isinstance(raw, str) and len(raw.split()) > 1:
            A = _parse_A_with_units(raw, order)
        else:
            A = float(raw) * self.conc ** (1.0 - order) / self.time
        b = float(rc.get("b", 0.0))
        Ea = _with_unit(rc.get("Ea", 0.0), _ENERGY_CAL_PER_MOL, self.energy, "activation-energy")
        return (A, b, Ea)


def _parse_A_with_units(text: str, order: float) -> float:
    # e.g. "1.0e+13 cm^3/mol/s": only cgs-mol strings are accepted
    num, unit = text.split(None, 1)
    unit = unit.replace(" ", "")
    expected = {1: "1/s", 2: "cm^3/mol/s", 3: "cm^6/mol^2/s"}
    if expected.get(round(order)) == unit:
        return float(num)
    raise ValueError(f"unsupported pre-exponential unit string {text!r}")


_TOKEN_RE = re.compile(r"^\s*([0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?)?\s*(.+?)\s*$")


def parse_equation(eqn: str):
    """Split a Cantera/Chemkin equation into (reactants, products, reversible,
    third_body) where third_body is None, "M", "(+M)" or "(+<species>)"."""
    if "<=>" in eqn:
        lhs, rhs = eqn.split("<=>"); rev = True
    elif "=>" in eqn:
        lhs, rhs = eqn.split("=>"); rev = False
    elif "=" in eqn:
        lhs, rhs = eqn.split("="); rev = True
    else:
        raise ValueError(f"no arrow in equation {eqn!r}")
    tb = None
    fall = re.compile(r"\(\s*\+\s*([^()\s]+)\s*\)")
    m_l, m_r = fall.search(lhs), fall.search(rhs)
    if m_l or m_r:
        if not (m_l and m_r) or m_l.group(1) != m_r.group(1):
            raise ValueError(f"unbalanced falloff collider in {eqn!r}")
        tb = "(+M)" if m_l.group(1) == "M" else f"(+{m_l.group(1)})"
        lhs, rhs = fall.sub(" ", lhs), fall.sub(" ", rhs)

    def side(s):
        out: Dict[str, float] = {}
        has_m = False
        # split on '+' that separates species; species names may contain '+'
        # only as a trailing charge, which ck2yaml surrounds by no spaces
        for tok in re.split(r"\s\+\s|^\+\s|\s\+$", " " + s.strip() + " "):
            tok = tok.strip()
            if not tok:
                continue
            if tok == "M":
                has_m = True
                continue
            m = re.match(r"^([0-9]*\.?[0-9]+)\s+(\S.*)$", tok)
            if m:
                nu, sp = float(m.group(1)), m.group(2).strip()
            else:
                nu, sp = 1.0, tok
            out[sp] = out.get(sp, 0.0) + nu
        return out, has_m

    reac, m1 = side(lhs)
    prod, m2 = side(rhs)
    if m1 or m2:
        if not (m1 and m2):
            raise ValueError(f"unbalanced third body in {eqn!r}")
        tb = tb or "M"
    return reac, prod, rev, tb


def _nasa(sp: dict) -> Tuple[Tuple[float, float, float], Tuple[float, ...], Tuple[float, ...]]:
    th = sp["thermo"]
    if th.get("model", "NASA7") != "NASA7":
        raise ValueError(f"species {sp['name']}: only NASA7 thermo is supported")
    tr = [float(t) for t in th["temperature-ranges"]]
    data = [tuple(float(c) for c in d) for d in th["data"]]
    if len(tr) == 2 and len(data) == 1:
        # single range: two identical ranges (the form Cantera reports back)
        return (tr[0], tr[1], tr[1]), data[0], data[0]
    if len(tr) == 3 and len(data) == 2:
        return (tr[0], tr[1], tr[2]), data[0], data[1]
    raise ValueError(f"species {sp['name']}: unsupported NASA7 layout with {len(tr)} ranges")


def mechanism_from_yaml(text: str, name: str = "mechanism", phase: Optional[str] = None,
                        reference_compat: bool = False) -> Mechanism:
    """Build a Mechanism from Cantera YAML text (ck2yaml output)."""
    d = load_yaml_text(text)
    units = _Units(d.get("units"))
    phases = d["phases"]
    ph = phases[0] if phase is None else next(p for p in phases if p["name"] == phase)
    sp_section = ph.get("species", "species")
    all_species = {s["name"]: s for s in d["species"]}
    if isinstance(sp_section, list) and sp_section and isinstance(sp_section[0], dict):
        names = [n for entry in sp_section for v in entry.values() for n in v]
    elif isinstance(sp_section, list):
        names = [str(n) for n in sp_section]
    elif sp_section in ("all", "species"):
        names = list(all_species)
    else:
        raise ValueError(f"unsupported species spec {sp_section!r}")
    species = []
    for n in names:
        s = all_species[n]
        t_ranges, lo, hi = _nasa(s)
        species.append(Species(name=n, composition={k: float(v) for k, v in s["composition"].items()},
                               t_ranges=t_ranges, nasa_low=lo, nasa_high=hi))
    rx_key = "reactions"
    kin = ph.get("reactions")
    if isinstance(kin, list) and kin and isinstance(kin[0], str) and kin[0] not in ("all", "declared-species"):
        rx_key = kin[0]
    reactions: List[Reaction] = []
    dropped: List[str] = []
    for rd in d.get(rx_key, []) or []:
        r = _reaction_from_yaml(rd, units, reference_compat)
        if r is None:
            dropped.append(rd["equation"])
        else:
            reactions.append(r)
    mech = Mechanism(name=name, species=species, reactions=reactions, dropped=dropped)
    mech.validate()
    return mech


def _effs(rd: dict) -> Dict[str, float]:
    # chemgen/parser.py:97,131 -- eff-1 for efficiencies different from 1;
    # the default efficiency is not used by the reference
    return {sp: float(e) - 1.0 for sp, e in (rd.get("efficiencies") or {}).items() if float(e) != 1.0}


def _reaction_from_yaml(rd: dict, units: _Units, reference_compat: bool) -> Optional[Reaction]:
    eqn = rd["equation"]
    rtype = rd.get("type", "elementary")
    reac, prod, rev, tb = parse_equation(eqn)
    if "reversible" in rd:
        rev = bool(rd["reversible"])
    dup = bool(rd.get("duplicate", False))
    order = sum(reac.values())
    if rtype in ("elementary", "reaction", "Arrhenius"):
        if tb is not None:
            rtype = "three-body"
        else:
            return Reaction(eqn, "standard", reac, prod, rev, dup, arh=units.rate(rd["rate-constant"], order))
    if rtype == "three-body":
        if tb == "M":
            return Reaction(eqn, "third_body", reac, prod, rev, dup,
                            arh=units.rate(rd["rate-constant"], order + 1), efficiencies=_effs(rd))
        # explicit collider: an elementary reaction that keeps the collider as
        # a species on both sides (chemgen/parser.py:107-130)
        if tb is not None and tb.startswith("(+"):
            raise ValueError(f"falloff collider in a three-body reaction {eqn!r}")
        return Reaction(eqn, "standard", reac, prod, rev, dup, arh=units.rate(rd["rate-constant"], order))
    if rtype == "falloff":
        hi = units.rate(rd["high-P-rate-constant"], order)
        lo = units.rate(rd["low-P-rate-constant"], order + 1)
        effs = _effs(rd)
        if "Troe" in rd:
            t = rd["Troe"]
            params = (float(t["A"]), float(t["T3"]), float(t["T1"]))
            if "T2" in t and float(t["T2"]) != 0.0:
                params = params + (float(t["T2"]),)
            kind, extra = "troe", {"troe": params}
        elif "SRI" in rd:
            if reference_compat:
                return None
            s = rd["SRI"]
            params = (float(s["A"]), float(s["B"]), float(s["C"]))
            if "D" in s or "E" in s:
                params = params + (float(s.get("D", 1.0)), float(s.get("E", 0.0)))
            kind, extra = "sri", {"sri": params}
        elif "Tsang" in rd:
            raise ValueError(f"Tsang falloff is not supported: {eqn!r}")
        else:
            if reference_compat:
                return None
            kind, extra = "lindemann", {}
        return Reaction(eqn, kind, reac, prod, rev, dup, arh=hi, low=lo, efficiencies=effs, **extra)
    if rtype == "pressure-dependent-Arrhenius":
        rates = []
        for rc in rd["rate-constants"]:
            p = _with_unit(rc["P"], _PRESSURE_DYNE, units.pressure, "pressure")
            A, b, Ea = units.rate(rc, order)
            rates.append((p, A, b, Ea))
        return Reaction(eqn, "plog", reac, prod, rev, dup, plog=rates)
    if rtype == "chemically-activated":
        if reference_compat:
            return None
        raise ValueError(f"chemically-activated reactions are not supported: {eqn!r}")
    raise ValueError(f"unsupported reaction type {rtype!r} in {eqn!r}")


def load_mechanism(path: str, name: Optional[str] = None, reference_compat: bool = False,
                   therm: Optional[str] = None) -> Mechanism:
    """Load a mechanism from a Cantera YAML file, a Chemkin ``.inp`` (+ thermo
    file) or this package's JSON form."""
    import os
    name = name or os.path.splitext(os.path.basename(path))[0]
    with open(path) as f:
        text = f.read()
    if path.endswith((".yaml", ".yml")):
        return mechanism_from_yaml(text, name=name, reference_compat=reference_compat)
    if path.endswith(".json"):
        return Mechanism.from_json(text)
    from .chemkin import mechanism_from_chemkin
    therm_text = None
    if therm is not None:
        with open(therm) as f:
            therm_text = f.read()
    return mechanism_from_chemkin(text, therm_text, name=name, reference_compat=reference_compat)
