"""The tensor-core mixed kernel (table-driven; q scaled per point and split
into three BF16 parts, nu . q accumulated by tcgen05.mma in tensor memory)
against the FP64 oracle.  The bar is the mixed-precision gate, 1e-6
normwise (max over points of max_k |dwdot_k| / max_k |wdot_k|), for every
mechanism, the 348-species ones included; the per-species maxima are
printed."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from chemgen_b200 import pack, synthetic
from chemgen_b200.runtime import GpuMechanism
from oracle import oracle

pytestmark = pytest.mark.gpu


def _run(gm, P, T, Y, mode):
    import torch
    Pt, Tt, Yt = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (P, T, Y))
    w = gm.getrates(Pt, Tt, Yt, mode=mode)
    torch.cuda.synchronize()
    return w.cpu().numpy()


@pytest.mark.parametrize("name", golden_names())
def test_tc_mixed_matches_reference_golden(name):
    mech, d = load_golden(name)
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(blob)
    gm.use_generated(False)
    assert gm.kernel_kind("mixed") == "table"
    S = oracle.rates(blob, d["P"], d["T"], d["Y"], mech.nr)["S"]
    w = _run(gm, d["P"], d["T"], d["Y"], "mixed")
    e = oracle.errors(w, d["wdot_scalar"], S)
    print(name, e)
    assert np.all(np.isfinite(w))
    assert e["norm_max"] <= 1e-6, e


@pytest.mark.parametrize("factory,ng", [(synthetic.all_kinds, 1000), (synthetic.gri_shape, 1 << 16),
                                        (synthetic.h2o2_10sp, 129), (synthetic.gri_shape, 1)])
def test_tc_mixed_matches_oracle_sizes(factory, ng):
    mech = factory()
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, ng, seed=ng + 7)
    gm = GpuMechanism(blob)
    gm.use_generated(False)
    w = _run(gm, P, T, Y, "mixed")
    idx = np.arange(0, ng, max(1, ng // 4096))
    r = oracle.rates(blob, P[idx], T[idx], np.ascontiguousarray(Y[:, idx]), mech.nr)
    e = oracle.errors(w[:, idx], r["wdot"], r["S"])
    print(mech.name, ng, e)
    assert e["norm_max"] <= 1e-6, e


def _per_species(w, ref):
    """Per species: max over points of |dwdot_k| / max_k |wdot_k| (the
    normwise measure split by species) and of |dwdot_k| / max |wdot_k| over
    the batch (relative to the species' own scale)."""
    d = np.abs(w - ref)
    den = np.abs(ref).max(axis=0)
    by_point = (d / np.where(den > 0, den, 1.0)).max(axis=1)
    own = np.abs(ref).max(axis=1)
    return by_point, d.max(axis=1) / np.where(own > 0, own, 1.0)


@pytest.mark.parametrize("golden,ng,stride", [("synthetic_348_2163", 4096, 1), ("jetsurf2", 1 << 18, 16)])
def test_tc_mixed_348_species_per_species_error(golden, ng, stride):
    """348 species / 2163 reactions (C3), including the real JetSurf 2.0 at
    2^18 points (every 16th point checked against the oracle)."""
    mech, _ = load_golden(golden)
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, ng, seed=31)
    gm = GpuMechanism(blob)
    w = _run(gm, P, T, Y, "mixed")
    idx = np.arange(0, ng, stride)
    r = oracle.rates(blob, P[idx], T[idx], np.ascontiguousarray(Y[:, idx]), mech.nr)
    ws = np.ascontiguousarray(w[:, idx])
    by_point, own = _per_species(ws, r["wdot"])
    e = oracle.errors(ws, r["wdot"], r["S"])
    worst = np.argsort(-by_point)[:5]
    print(golden, ng, e, "worst species", [(mech.species[k].name, float(by_point[k])) for k in worst],
          "max relative to own scale", float(own.max()))
    assert np.all(np.isfinite(w))
    assert e["norm_max"] <= 1e-6, e
    assert by_point.max() <= 1e-6


@pytest.mark.parametrize("factory", [synthetic.jetsurf_shape, synthetic.gri_shape])
def test_tc_mixed_low_temperature_states(factory):
    """At 300-400 K every rate of progress of a point can lie below FP32's
    range (2^-126 mol/cm^3/s); the per-point scale keeps them representable."""
    mech = factory()
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, 2048, seed=41)
    T = np.linspace(300.0, 400.0, T.size)
    gm = GpuMechanism(blob)
    gm.use_generated(False)
    w = _run(gm, P, T, Y, "mixed")
    r = oracle.rates(blob, P, T, Y, mech.nr)
    e = oracle.errors(w, r["wdot"], r["S"])
    print(mech.name, "300-400 K", e, "smallest max|wdot|", float(np.abs(r["wdot"]).max(axis=0).min()))
    assert e["norm_max"] <= 1e-6, e
