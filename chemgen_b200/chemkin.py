"""Chemkin-II mechanism (``chem.inp``) and NASA-7 thermo (``therm.dat``) reader.

The reference hands Chemkin input to Cantera's ``ck2yaml`` and then reads the
YAML (``chemgen/parser.py:57-66``).  This reader produces the same
:class:`~chemgen_b200.mechanism.Mechanism` directly, following the Chemkin-II
input rules: ELEMENTS / SPECIES / THERMO / REACTIONS sections, units keywords
on the REACTIONS line, auxiliary lines LOW / TROE / SRI / PLOG / DUPLICATE and
third-body efficiencies ``SP/eff/``.  Fixed-column NASA-7 records follow the
Chemkin thermo format (4 lines per species, columns 1-80).
"""
from __future__ import annotations

import re
from typing import Dict, List, Optional, Tuple

from .mechanism import (ATOMIC_WEIGHTS, Mechanism, Reaction, Species, _element_key,
                        parse_equation)

_E_UNITS = {"CAL/MOLE": 1.0, "KCAL/MOLE": 1000.0, "JOULES/MOLE": 1.0 / 4.184,
            "KJOULES/MOLE": 1000.0 / 4.184, "KELVINS": 8314.462618 / 4184.0,
            "EVOLTS": 96485.33212 / 4.184}
_A_UNITS = {"MOLES": 1.0, "MOLECULES": 6.02214076e23}
_KEYWORDS = {"ELEMENTS", "ELEM", "SPECIES", "SPEC", "THERMO", "REACTIONS", "REAC", "TRANSPORT", "END"}


def _num(text: str) -> float:
    """A Chemkin number (Fortran D exponents allowed); a negative zero reads as
    +0.0, as ck2yaml writes it."""
    return float(text.replace("D", "E").replace("d", "e")) + 0.0


def _strip_comment(line: str) -> str:
    i = line.find("!")
    return (line if i < 0 else line[:i]).rstrip()


def _read_sections(text: str) -> Dict[str, List[str]]:
    sections: Dict[str, List[str]] = {}
    current = None
    for raw in text.splitlines():
        line = _strip_comment(raw)
        if not line.strip():
            continue
        head = line.split()[0].upper()
        if head in ("ELEMENTS", "ELEM", "SPECIES", "SPEC", "THERMO", "REACTIONS", "REAC", "TRANSPORT"):
            current = {"ELEM": "ELEMENTS", "SPEC": "SPECIES", "REAC": "REACTIONS"}.get(head, head)
            sections.setdefault(current, [])
            sections[current].append(line)          # keep header (units, ALL)
            continue
        if head == "END":
            current = None
            continue
        if current is not None:
            sections[current].append(line if current == "THERMO" else line)
    return sections


def parse_thermo(lines: List[str], wanted: Optional[List[str]] = None) -> Dict[str, Tuple]:
    """Fixed-column NASA-7 records -> {name: (composition, (Tlo, Tmid, Thi), low, high)}."""
    out: Dict[str, Tuple] = {}
    body = [l for l in lines if l.strip() and not l.split()[0].upper().startswith("THERMO")]
    default_mid = 1000.0
    i = 0
    # optional global temperature line
    if body and len(body[0].split()) == 3 and not body[0].rstrip().endswith("1"):
        try:
            default_mid = float(body[0].split()[1])
            i = 1
        except ValueError:
            pass
    while i + 3 < len(body) + 0 and i < len(body):
        l1 = body[i].ljust(80)
        if not l1[79:80] == "1":
            i += 1
            continue
        name = l1[0:18].split()[0]
        comp: Dict[str, float] = {}
        for j in range(4):
            el = l1[24 + 5 * j: 26 + 5 * j].strip()
            cnt = l1[26 + 5 * j: 29 + 5 * j].strip()
            if el and el != "0" and cnt:
                n = float(cnt)
                if n:
                    comp[_element_key(el)] = comp.get(_element_key(el), 0.0) + n
        el5 = l1[73:75].strip()
        if el5 and l1[75:78].strip():
            n = float(l1[75:78])
            if n:
                comp[_element_key(el5)] = comp.get(_element_key(el5), 0.0) + n
        tlo = float(l1[45:55]); thi = float(l1[55:65])
        tmid_s = l1[65:73].strip()
        tmid = float(tmid_s) if tmid_s else default_mid
        coefs = []
        for k in range(1, 4):
            lk = body[i + k].ljust(80)
            for j in range(5):
                field = lk[15 * j: 15 * (j + 1)].strip()
                if field:
                    coefs.append(_num(field))
        if len(coefs) < 14:
            raise ValueError(f"thermo record for {name} has {len(coefs)} coefficients")
        high, low = tuple(coefs[0:7]), tuple(coefs[7:14])
        if high == low:
            # identical ranges collapse to one, as ck2yaml writes them
            tmid = thi
        if name not in out:
            out[name] = (comp, (tlo, tmid, thi), low, high)
        i += 4
    return out


def _split_species(side: str, known: set) -> Dict[str, float]:
    toks = side.split("+")
    out: Dict[str, float] = {}
    k = 0
    while k < len(toks):
        tok = toks[k]
        # names ending in '+' (ions) produce empty tokens; merge greedily
        j = k + 1
        while j <= len(toks):
            cand = "+".join(toks[k:j])
            if cand in known:
                tok = cand
                k = j
                break
            j += 1
        else:
            k += 1
        tok = tok.strip()
        if not tok:
            continue
        if tok in known or tok == "M":
            sp, nu = tok, 1.0
        else:
            m = re.match(r"^([0-9]*\.?[0-9]+)(.+)$", tok)
            if not m or m.group(2) not in known:
                raise ValueError(f"unknown species token {tok!r}")
            nu, sp = float(m.group(1)), m.group(2)
        out[sp] = out.get(sp, 0.0) + nu
    return out


def _equation_to_canonical(eqn: str, known: set) -> str:
    """Chemkin equation without blanks -> the spaced form parse_equation reads."""
    for arrow in ("<=>", "=>", "="):
        if arrow in eqn:
            lhs, rhs = eqn.split(arrow, 1)
            break
    else:
        raise ValueError(f"no arrow in {eqn!r}")

    def side(s):
        fall = re.search(r"\(\+([^()]+)\)", s)
        coll = None
        if fall:
            coll = fall.group(1)
            s = s[:fall.start()] + s[fall.end():]
        parts = []
        for sp, nu in _split_species(s, known | {"M"}).items():
            parts.append(sp if nu == 1.0 else f"{nu:g} {sp}")
        txt = " + ".join(parts)
        if coll:
            txt += f" (+{coll})"
        return txt

    return f"{side(lhs)} {arrow} {side(rhs)}"


def mechanism_from_chemkin(text: str, therm_text: Optional[str] = None, name: str = "mechanism",
                           reference_compat: bool = False) -> Mechanism:
    secs = _read_sections(text)
    species_names: List[str] = []
    for line in secs.get("SPECIES", [])[0:]:
        toks = line.split()
        if toks and toks[0].upper() in ("SPECIES", "SPEC"):
            toks = toks[1:]
        species_names.extend(toks)
    known = set(species_names)
    thermo: Dict[str, Tuple] = {}
    if therm_text is not None:
        tsecs = _read_sections(therm_text)
        tl = tsecs.get("THERMO") or [l for l in therm_text.splitlines() if l.strip()]
        thermo.update(parse_thermo(tl))
    if "THERMO" in secs:
        thermo.update(parse_thermo(secs["THERMO"]))
    species = []
    for n in species_names:
        if n not in thermo:
            raise ValueError(f"no thermo data for species {n}")
        comp, tr, lo, hi = thermo[n]
        species.append(Species(name=n, composition=comp, t_ranges=tr, nasa_low=lo, nasa_high=hi))

    rlines = secs.get("REACTIONS", [])
    e_fac, a_fac = 1.0, 1.0
    if rlines:
        for tok in rlines[0].split()[1:]:
            t = tok.upper()
            if t in _E_UNITS:
                e_fac = _E_UNITS[t]
            elif t in _A_UNITS:
                a_fac = _A_UNITS[t]
        rlines = rlines[1:]
    if a_fac != 1.0:
        raise ValueError("MOLECULES units are not supported")

    raw: List[dict] = []
    num = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eEdD][-+]?\d+)?"
    rate_re = re.compile(rf"^(.*?)\s+({num})\s+({num})\s+({num})\s*$")
    for line in rlines:
        m = rate_re.match(line.strip())
        if m and ("=" in m.group(1)):
            raw.append({"eqn": m.group(1).replace(" ", ""),
                        "arh": tuple(_num(x) for x in m.groups()[1:]),
                        "aux": []})
        else:
            if not raw:
                raise ValueError(f"auxiliary line before any reaction: {line!r}")
            raw[-1]["aux"].append(line.strip())

    reactions: List[Reaction] = []
    dropped: List[str] = []
    for r in raw:
        eqn = _equation_to_canonical(r["eqn"], known)
        reac, prod, rev, tb = parse_equation(eqn)
        A, b, Ea = r["arh"]
        Ea *= e_fac
        effs: Dict[str, float] = {}
        low = troe = sri = None
        plog: List[Tuple[float, float, float, float]] = []
        dup = False
        for aux in r["aux"]:
            up = aux.upper()
            if up.startswith("DUP"):
                dup = True
                continue
            for key, vals in re.findall(r"([A-Za-z][^/\s]*)\s*/([^/]*)/", aux):
                K = key.upper()
                nums = [_num(v) for v in vals.split()]
                if K == "LOW":
                    low = (nums[0], nums[1], nums[2] * e_fac)
                elif K == "TROE":
                    troe = tuple(nums[:3]) + ((nums[3],) if len(nums) > 3 and nums[3] != 0.0 else ())
                elif K == "SRI":
                    sri = tuple(nums)
                elif K == "PLOG":
                    plog.append((nums[0] * 1013250.0, nums[1], nums[2], nums[3] * e_fac))
                elif K in ("DUP", "DUPLICATE"):
                    dup = True
                elif K in ("REV", "HIGH", "FORD", "RORD", "LT", "RLT", "TDEP", "XSMI", "EXCI", "JAN", "FIT1",
                           "MOME", "UNITS", "CHEB", "TCHEB", "PCHEB"):
                    raise ValueError(f"auxiliary keyword {K} is not supported ({eqn})")
                elif key in known:
                    if float(nums[0]) != 1.0:
                        effs[key] = float(nums[0]) - 1.0
                else:
                    raise ValueError(f"unknown auxiliary keyword {key!r} in {eqn}")
        order = sum(reac.values())
        del order  # A is already cgs in Chemkin input
        if plog:
            reactions.append(Reaction(eqn, "plog", reac, prod, rev, dup, plog=plog))
        elif tb in ("M",):
            reactions.append(Reaction(eqn, "third_body", reac, prod, rev, dup, arh=(A, b, Ea), efficiencies=effs))
        elif tb is not None:
            if low is None:
                raise ValueError(f"falloff reaction without LOW: {eqn}")
            if tb != "(+M)":
                # an explicit bath gas; like the reference, the collider
                # restriction is not applied (M = all species, eff from list)
                effs = {}
            if troe is not None:
                reactions.append(Reaction(eqn, "troe", reac, prod, rev, dup, arh=(A, b, Ea), low=low,
                                          troe=troe, efficiencies=effs))
            elif reference_compat:
                dropped.append(eqn)
            elif sri is not None:
                reactions.append(Reaction(eqn, "sri", reac, prod, rev, dup, arh=(A, b, Ea), low=low,
                                          sri=sri, efficiencies=effs))
            else:
                reactions.append(Reaction(eqn, "lindemann", reac, prod, rev, dup, arh=(A, b, Ea), low=low,
                                          efficiencies=effs))
        else:
            reactions.append(Reaction(eqn, "standard", reac, prod, rev, dup, arh=(A, b, Ea)))
    mech = Mechanism(name=name, species=species, reactions=reactions, dropped=dropped)
    mech.validate()
    return mech
