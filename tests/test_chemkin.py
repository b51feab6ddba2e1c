"""The Chemkin reader (chem.inp + therm.dat) against known answers, against
the Cantera-YAML reader on the same mechanism, and -- when a checkout of the
reference is named by CHEMGEN_REFERENCE -- against the reference's own
ck2yaml output (ck_files/*/chem.yaml beside chem.inp and therm.dat).

The reference reads Chemkin input only through ck2yaml + Cantera
(chemgen/parser.py:55-66); its reaction dicts keep A in cgs, Ea in cal/mol,
efficiencies as eff - 1 and the Troe tuple (a, T3, T1[, T2])
(chemgen/parser.py:70-159).  The same conventions are asserted here."""
import math
import os

import numpy as np
import pytest

from conftest import REFERENCE, reference_available
from chemgen_b200 import pack, synthetic
from chemgen_b200.chemkin import mechanism_from_chemkin
from chemgen_b200.mechanism import load_mechanism, mechanism_from_yaml
from oracle import oracle

NAMES = ["H2", "O2", "H2O", "H", "O", "OH", "HO2", "H2O2", "N2", "AR"]

REACTIONS = """\
REACTIONS   KCAL/MOLE
H+O2<=>O+OH            3.547E+15  -0.406  16.599
O+H2=H+OH              5.08D+04    2.67    6.290   ! a comment after the numbers
2OH=>O+H2O             3.57E+04    2.4    -2.110
H+H+M<=>H2+M           1.3E+18    -1.0     0.0
H2/2.5/ H2O/12.0/
AR/0.0/
H2O2(+M)<=>2OH(+M)     2.0E+12     0.9    48.749
LOW/2.49E+24 -2.3 48.749/
TROE/0.43 1.0E-30 1.0E+30/
H2O/7.5/ O2/1.2/
HO2+H<=>2OH            7.08E+13    0.0     0.295
DUPLICATE
HO2+H<=>2OH            1.0E+12     0.0     0.0
DUPLICATE
H+OH(+AR)<=>H2O(+AR)   1.0E+14     0.0     0.0
LOW/1.0E+20 -1.0 0.0/
H+O2(+M)<=>HO2(+M)     4.65E+12    0.44    0.0
LOW/6.366E+20 -1.72 0.525/
SRI/0.5 200.0 1000.0 1.2 0.3/
O+OH(+M)=HO2(+M)       1.0E+13     0.0     0.0
LOW/1.0E+18 -1.0 0.0/
TROE/0.7 100.0 2000.0 5000.0/
H2O2+H<=>H2O+OH        1.0E+13     0.0     3.6
PLOG/0.1  1.0E+12 0.5 1.0/
PLOG/1.0  2.0E+12 0.4 2.0/
PLOG/1.0  5.0E+11 0.1 -0.0/
PLOG/10.0 3.0E+12 0.3 3.0/
H2+O2=>H2O+O           1.0E+10     0.0    -0.0
END
"""

YAML_REACTIONS = """\
reactions:
- equation: H + O2 <=> O + OH
  rate-constant: {A: 3.547e+15, b: -0.406, Ea: 16.599 kcal/mol}
- equation: O + H2 <=> H + OH
  rate-constant: {A: 5.08e+04, b: 2.67, Ea: 6.290 kcal/mol}
- equation: 2 OH => O + H2O
  rate-constant: {A: 3.57e+04, b: 2.4, Ea: -2.110 kcal/mol}
- equation: H + H + M <=> H2 + M
  type: three-body
  rate-constant: {A: 1.3e+18, b: -1.0, Ea: 0.0 kcal/mol}
  efficiencies: {H2: 2.5, H2O: 12.0, AR: 0.0}
- equation: H2O2 (+M) <=> 2 OH (+M)
  type: falloff
  low-P-rate-constant: {A: 2.49e+24, b: -2.3, Ea: 48.749 kcal/mol}
  high-P-rate-constant: {A: 2.0e+12, b: 0.9, Ea: 48.749 kcal/mol}
  Troe: {A: 0.43, T3: 1.0e-30, T1: 1.0e+30}
  efficiencies: {H2O: 7.5, O2: 1.2}
- equation: HO2 + H <=> 2 OH
  rate-constant: {A: 7.08e+13, b: 0.0, Ea: 0.295 kcal/mol}
  duplicate: true
- equation: HO2 + H <=> 2 OH
  rate-constant: {A: 1.0e+12, b: 0.0, Ea: 0.0 kcal/mol}
  duplicate: true
- equation: H + OH (+AR) <=> H2O (+AR)
  type: falloff
  low-P-rate-constant: {A: 1.0e+20, b: -1.0, Ea: 0.0 kcal/mol}
  high-P-rate-constant: {A: 1.0e+14, b: 0.0, Ea: 0.0 kcal/mol}
- equation: H + O2 (+M) <=> HO2 (+M)
  type: falloff
  low-P-rate-constant: {A: 6.366e+20, b: -1.72, Ea: 0.525 kcal/mol}
  high-P-rate-constant: {A: 4.65e+12, b: 0.44, Ea: 0.0 kcal/mol}
  SRI: {A: 0.5, B: 200.0, C: 1000.0, D: 1.2, E: 0.3}
- equation: O + OH (+M) <=> HO2 (+M)
  type: falloff
  low-P-rate-constant: {A: 1.0e+18, b: -1.0, Ea: 0.0 kcal/mol}
  high-P-rate-constant: {A: 1.0e+13, b: 0.0, Ea: 0.0 kcal/mol}
  Troe: {A: 0.7, T3: 100.0, T1: 2000.0, T2: 5000.0}
- equation: H2O2 + H <=> H2O + OH
  type: pressure-dependent-Arrhenius
  rate-constants:
  - {P: 0.1 atm, A: 1.0e+12, b: 0.5, Ea: 1.0 kcal/mol}
  - {P: 1.0 atm, A: 2.0e+12, b: 0.4, Ea: 2.0 kcal/mol}
  - {P: 1.0 atm, A: 5.0e+11, b: 0.1, Ea: 0.0 kcal/mol}
  - {P: 10.0 atm, A: 3.0e+12, b: 0.3, Ea: 3.0 kcal/mol}
- equation: H2 + O2 => H2O + O
  rate-constant: {A: 1.0e+10, b: 0.0, Ea: 0.0 kcal/mol}
"""


def _e15(x: float) -> str:
    return f"{x:15.8E}"


def _species():
    """Ten species with NASA-7 coefficients rounded to the 8 digits the fixed
    columns of a thermo record hold (a seeded synthetic thermo set)."""
    out = []
    for s in synthetic.h2o2_10sp().species:
        lo = tuple(float(_e15(c)) for c in s.nasa_low)
        hi = tuple(float(_e15(c)) for c in s.nasa_high)
        comp = {e: float(int(n)) for e, n in s.composition.items()}
        out.append((s.name, comp, s.t_ranges, lo, hi))
    return out


def _therm_text(species) -> str:
    """Chemkin thermo records: columns 1-18 name, 25-44 four (element, count)
    pairs, 46-55 Tlow, 56-65 Thigh, 66-73 Tmid, column 80 the line number;
    then three lines of E15.8 coefficients (upper range first)."""
    lines = ["THERMO ALL", "   300.000  1000.000  5000.000"]
    for name, comp, (tlo, tmid, thi), lo, hi in species:
        els = "".join(f"{e.upper():<2s}{int(n):>3d}" for e, n in list(comp.items())[:4])
        l1 = f"{name:<18s}{'121286':<6s}{els:<20s}G{tlo:10.3f}{thi:10.3f}{tmid:8.2f}"
        lines.append(f"{l1:<79s}1")
        c = list(hi) + list(lo)
        lines.append(f"{''.join(_e15(x) for x in c[0:5]):<79s}2")
        lines.append(f"{''.join(_e15(x) for x in c[5:10]):<79s}3")
        lines.append(f"{''.join(_e15(x) for x in c[10:14]):<79s}4")
    lines.append("END")
    return "\n".join(lines) + "\n"


def _inp_text() -> str:
    return "ELEMENTS\nH O N C AR\nEND\nSPECIES\n" + " ".join(NAMES) + "\nEND\n" + REACTIONS


def _yaml_text(species) -> str:
    head = ("units: {length: cm, quantity: mol, activation-energy: cal/mol}\n"
            "phases:\n- name: gas\n  thermo: ideal-gas\n  elements: [H, O, N, C, Ar]\n"
            f"  species: [{', '.join(NAMES)}]\n  kinetics: gas\n  state: {{T: 300.0, P: 1 atm}}\n"
            "species:\n")
    body = []
    for name, comp, (tlo, tmid, thi), lo, hi in species:
        cs = ", ".join(f"{e}: {int(n)}" for e, n in comp.items())
        body.append(f"- name: {name}\n  composition: {{{cs}}}\n  thermo:\n    model: NASA7\n"
                    f"    temperature-ranges: [{tlo!r}, {tmid!r}, {thi!r}]\n    data:\n"
                    f"    - [{', '.join(repr(x) for x in lo)}]\n    - [{', '.join(repr(x) for x in hi)}]\n")
    return head + "".join(body) + YAML_REACTIONS


def test_chemkin_reader_known_answers():
    sp = _species()
    m = mechanism_from_chemkin(_inp_text(), _therm_text(sp), name="ck")
    assert m.species_names == NAMES
    for s, (name, comp, tr, lo, hi) in zip(m.species, sp):
        assert s.composition == comp and s.t_ranges == tr and s.nasa_low == lo and s.nasa_high == hi
    r = m.reactions
    assert [x.kind for x in r] == ["standard", "standard", "standard", "third_body", "troe", "standard", "standard",
                                   "lindemann", "sri", "troe", "plog", "standard"]
    # KCAL/MOLE on the REACTIONS line: Ea in cal/mol; Fortran D exponents
    assert r[0].arh == (3.547e15, -0.406, 16.599 * 1000.0)
    assert r[1].arh == (5.08e4, 2.67, 6.290 * 1000.0) and r[1].reversible
    # '=>' is irreversible; "2OH" is two OH molecules
    assert not r[2].reversible and r[2].reactants == {"OH": 2.0} and r[2].arh[2] == -2.110 * 1000.0
    # third body: H+H+M; efficiencies stored as eff - 1, over two lines
    assert r[3].reactants == {"H": 2.0} and r[3].products == {"H2": 1.0}
    assert r[3].efficiencies == {"H2": 1.5, "H2O": 11.0, "AR": -1.0}
    # Troe with three parameters, LOW in the file's energy units
    assert r[4].low == (2.49e24, -2.3, 48.749 * 1000.0) and r[4].troe == (0.43, 1e-30, 1e30)
    assert r[4].efficiencies == {"H2O": 6.5, "O2": pytest.approx(0.2)}
    assert r[4].products == {"OH": 2.0}
    assert r[5].duplicate and r[6].duplicate and not r[0].duplicate
    # explicit collider (+AR): M is the whole mixture, no efficiency list
    # (the reference ignores the collider restriction, chemgen/parser.py:97)
    assert r[7].efficiencies == {} and r[7].low == (1e20, -1.0, 0.0)
    assert r[8].sri == (0.5, 200.0, 1000.0, 1.2, 0.3) and r[8].low[2] == 525.0
    # Troe with T2
    assert r[9].troe == (0.7, 100.0, 2000.0, 5000.0)
    # PLOG: pressures in dyne/cm^2, two entries at one pressure kept
    assert [p for p, *_ in r[10].plog] == [0.1 * 1013250.0, 1013250.0, 1013250.0, 10.0 * 1013250.0]
    assert r[10].plog[1][1:] == (2e12, 0.4, 2000.0)
    # a negative zero reads as +0.0
    assert math.copysign(1.0, r[10].plog[2][3]) == 1.0 and math.copysign(1.0, r[11].arh[2]) == 1.0


def test_chemkin_reference_compat_drops_what_the_reference_drops():
    # chemgen/parser.py:146-147 keeps only Troe falloff
    m = mechanism_from_chemkin(_inp_text(), _therm_text(_species()), reference_compat=True)
    assert m.nr == 10
    assert len(m.dropped) == 2 and all("(+" in e for e in m.dropped)


@pytest.mark.parametrize("units,factor", [("", 1.0), ("CAL/MOLE", 1.0), ("KCAL/MOLE", 1000.0),
                                          ("JOULES/MOLE", 1.0 / 4.184), ("KJOULES/MOLE", 1000.0 / 4.184),
                                          ("MOLES KELVINS", 8314.462618 / 4184.0)])
def test_chemkin_energy_units(units, factor):
    text = ("ELEMENTS\nH O N C AR\nEND\nSPECIES\n" + " ".join(NAMES) + "\nEND\n"
            f"REACTIONS {units}\nH+O2<=>O+OH  1.0E+14  0.0  1000.0\nEND\n")
    m = mechanism_from_chemkin(text, _therm_text(_species()))
    assert m.reactions[0].arh[2] == pytest.approx(1000.0 * factor, rel=1e-15)


def test_chemkin_and_yaml_readers_agree():
    sp = _species()
    a = mechanism_from_chemkin(_inp_text(), _therm_text(sp), name="m")
    b = mechanism_from_yaml(_yaml_text(sp), name="m")
    assert a.species_names == b.species_names
    assert pack.pack(a).to_blob() == pack.pack(b).to_blob()
    blob = pack.pack(a).to_blob()
    assert oracle.check_blob(blob) == 0
    P, T, Y = synthetic.states(a.ns, 64, seed=5)
    w = oracle.getrates(blob, P, T, Y)
    assert np.all(np.isfinite(w))


CK_DIRS = ["GRI30", "H2_burke", "methane_NUI"]


def _fields(r):
    return (r.kind, r.reactants, r.products, r.reversible, r.duplicate, r.efficiencies, r.troe, r.sri)


def _close(x, y, rel=1e-12):
    if x is None or y is None:
        return x is None and y is None
    return len(x) == len(y) and all(a == b or abs(a - b) <= rel * max(abs(a), abs(b)) for a, b in zip(x, y))


@pytest.mark.skipif(not reference_available(), reason="set CHEMGEN_REFERENCE to a checkout of the reference")
@pytest.mark.parametrize("compat", [False, True])
@pytest.mark.parametrize("name", CK_DIRS)
def test_chemkin_matches_reference_ck2yaml_output(name, compat):
    d = os.path.join(REFERENCE, "ck_files", name)
    a = load_mechanism(os.path.join(d, "chem.inp"), therm=os.path.join(d, "therm.dat"), reference_compat=compat)
    b = load_mechanism(os.path.join(d, "chem.yaml"), reference_compat=compat)
    assert a.species_names == b.species_names
    for s, t in zip(a.species, b.species):
        assert s.composition == t.composition and _close(s.t_ranges, t.t_ranges)
        assert _close(s.nasa_low, t.nasa_low) and _close(s.nasa_high, t.nasa_high)
    assert a.nr == b.nr and len(a.dropped) == len(b.dropped)
    for r, q in zip(a.reactions, b.reactions):
        assert _fields(r) == _fields(q), (r.equation, q.equation)
        assert _close(r.arh, q.arh) and _close(r.low, q.low), r.equation
        assert (r.plog is None) == (q.plog is None)
        if r.plog:
            assert len(r.plog) == len(q.plog) and all(_close(x, y) for x, y in zip(r.plog, q.plog))
    ba, bb = pack.pack(a).to_blob(), pack.pack(b).to_blob()
    assert ba == bb
    P, T, Y = synthetic.states(a.ns, 256, seed=11)
    np.testing.assert_array_equal(oracle.getrates(ba, P, T, Y), oracle.getrates(bb, P, T, Y))
