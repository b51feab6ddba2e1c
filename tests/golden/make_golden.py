"""Generate the golden fixtures from the reference's OWN generated getrates.

Runs only where the reference sources are present (this script is the one
committed recipe that reads them).  For each mechanism it:

1. registers stand-in ``cantera`` / ``pint`` modules (imported at module top by
   ``chemgen/parser.py:6,9`` and ``chemgen/chemistry.py:2`` but not used by the
   emitter);
2. hands the reference's emitter, ``chemgen.chemistry.chemistry_expressions``
   (``chemgen/chemistry.py:185-369``), a duck-typed mechanism object built from
   this package's Mechanism IR with the reference's dict conventions
   (``chemgen/parser.py:70-145``);
3. renders the reference's Python getrates, scalar and vectorised
   (``language='python'``), imports them and runs them on seeded states;
4. saves ``<name>.npz``: the mechanism (JSON), P, T, Y[ns, ng], and wdot from
   the scalar and the vectorised generated code.

Usage:  python tests/golden/make_golden.py <reference_root>   (or CHEMGEN_REFERENCE=<reference_root>)
"""
from __future__ import annotations

import importlib.util
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from chemgen_b200 import synthetic  # noqa: E402
from chemgen_b200.mechanism import Mechanism, load_mechanism  # noqa: E402


def _stub_modules():
    ct = types.ModuleType("cantera")
    pint = types.ModuleType("pint")

    class UnitRegistry:  # never called by the emitter
        def __init__(self, *a, **k):
            raise RuntimeError("pint is not available")

    pint.UnitRegistry = UnitRegistry
    sys.modules.setdefault("cantera", ct)
    sys.modules.setdefault("pint", pint)


class _Sp:
    def __init__(self, s):
        self.molecular_weight = s.mw
        self.input_data = {"thermo": {"model": "NASA7", "temperature-ranges": list(s.t_ranges),
                                      "data": [list(s.nasa_low), list(s.nasa_high)]}}


class _Chem:
    """The attributes chemistry_expressions reads (chemgen/chemistry.py:186-321)."""

    def __init__(self, mech: Mechanism):
        self.species = mech.species_names
        self.reduced_species = list(self.species)
        self.stoi = {s: i for i, s in enumerate(self.species)}
        self.stoi_red = dict(self.stoi)
        self.n_species_sk = self.n_species_red = len(self.species)
        self.species_dict = {s.name: _Sp(s) for s in mech.species}
        self.reaction_types = ["standard", "troe", "third_body", "plog"]
        self.reactions = {}
        for i, r in enumerate(mech.reactions):
            if r.kind not in ("standard", "third_body", "troe", "plog"):
                raise ValueError(f"the reference cannot express {r.kind} ({r.equation})")
            d = {"eqn": r.equation, "reacts": dict(r.reactants), "prods": dict(r.products), "type": r.kind,
                 "reversible": r.reversible, "dup": r.duplicate, "ct": None}
            if r.kind != "plog":
                d["arh"] = tuple(r.arh)
            if r.kind == "troe":
                d["troe"] = {"low": tuple(r.low), "troe": tuple(r.troe)}
            if r.kind in ("troe", "third_body"):
                d["third_body"] = dict(r.efficiencies)
            if r.kind == "plog":
                d["plog"] = [tuple(p) for p in r.plog]
            self.reactions[i] = d


def _render(ref_root: str, mech: Mechanism, vec: bool, outdir: str):
    _stub_modules()
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    from chemgen.chemistry import chemistry_expressions
    fname = os.path.join(outdir, f"ref_{mech.name}_{'vec' if vec else 'scalar'}.py")
    ce = chemistry_expressions(_Chem(mech), vec=vec, omp=False, mod=False, language="python")
    ce.write_expressions_to_file(fname, write_rtypes_together=False, input_MW=False)
    spec = importlib.util.spec_from_file_location(os.path.basename(fname)[:-3], fname)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def edge_states(ns: int, seed: int):
    """Edge cases: exact zeros in Y, T at 300/1000/2500 K (1000 K is every
    species' range switch), pressures at both ends, a pure species."""
    rng = np.random.default_rng(seed + 99)
    T = np.array([300.0, 1000.0, 2500.0, 999.999999, 1000.000001, 1500.0, 700.0, 2000.0])
    P = np.array([1013250.0, 1013250.0 * 40, 1013250.0, 1013250.0 * 3, 1013250.0 * 7, 1013250.0 * 20,
                  1013250.0, 1013250.0 * 39.9])
    Y = rng.dirichlet(np.full(ns, 0.5), size=len(T)).T.copy()
    Y[: ns // 2, 0] = 0.0
    Y[ns // 3:, 5] = 0.0
    Y[:, 6] = 0.0
    Y[ns - 1, 6] = 1.0
    Y /= Y.sum(axis=0, keepdims=True)
    return P, T, Y


def make(ref_root: str, mech: Mechanism, ng: int, seed: int, outdir: str, tmp: str):
    P, T, Y = synthetic.states(mech.ns, ng, seed=seed)
    Pe, Te, Ye = edge_states(mech.ns, seed)
    P = np.concatenate([P, Pe]); T = np.concatenate([T, Te]); Y = np.concatenate([Y, Ye], axis=1)
    ngt = T.size
    scal = _render(ref_root, mech, False, tmp)
    w_s = np.zeros((mech.ns, ngt))
    for i in range(ngt):
        w = np.zeros(mech.ns)
        scal.getrates(np.float64(T[i]), Y[:, i].copy(), np.float64(P[i]), w)
        w_s[:, i] = w
    vec = _render(ref_root, mech, True, tmp)
    w_v = np.zeros((ngt, mech.ns))
    vec.getrates_i(ngt, T.copy(), np.ascontiguousarray(Y.T), P.copy(), w_v)
    path = os.path.join(outdir, f"{mech.name}.npz")
    np.savez_compressed(path, mech=np.array(mech.to_json()), P=P, T=T, Y=Y, wdot_scalar=w_s,
                        wdot_vec=np.ascontiguousarray(w_v.T), seed=seed)
    print(f"{path}: ns={mech.ns} nr={mech.nr} ng={ngt}")


def plog_mechanism() -> Mechanism:
    """A small synthetic mechanism with PLOG reactions (kinds the reference expresses)."""
    return synthetic.synthetic_mechanism(15, 40, 4, 4, seed=7, n_plog=8, name="synthetic_plog_15_40")


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CHEMGEN_REFERENCE", "")
    if not ref or not os.path.isdir(os.path.join(ref, "ck_files")):
        sys.exit("usage: make_golden.py <reference checkout> (or set CHEMGEN_REFERENCE)")
    ck = os.path.join(ref, "ck_files")
    jobs = [
        (load_mechanism(os.path.join(ck, "H2_burke/chem.yaml"), name="h2_burke", reference_compat=True), 504, 1),
        (load_mechanism(os.path.join(ck, "Hydrogen_H2/Burke_et_al_2012/chem.yaml"), name="burke2012",
                        reference_compat=True), 504, 2),
        (load_mechanism(os.path.join(ck, "GRI30/chem.yaml"), name="gri30", reference_compat=True), 248, 3),
        (synthetic.h2o2_10sp(), 504, 4),
        (synthetic.gri_shape(), 248, 5),
        (plog_mechanism(), 248, 6),
        (load_mechanism(os.path.join(ck, "JetSurf/2.0/chem.yaml"), name="jetsurf2", reference_compat=True), 24, 7),
        (synthetic.jetsurf_shape(), 24, 8),
    ]
    with tempfile.TemporaryDirectory() as tmp:
        for mech, ng, seed in jobs:
            make(ref, mech, ng, seed, HERE, tmp)


if __name__ == "__main__":
    main()
