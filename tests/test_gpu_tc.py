"""The tensor-core mixed kernel (table-driven; q split into three BF16 parts,
nu . q accumulated by tcgen05.mma in tensor memory) against the FP64 oracle.
Bars: 1e-6 normwise for mechanisms up to 72 species (the mixed-precision
gate); for 348-species mechanisms the FP32 accumulation over hundreds of
reactions per species is reported per species and bounded at 1e-4."""
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
    assert e["norm_max"] <= (1e-6 if mech.ns <= 72 else 1e-4), e


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


def test_tc_mixed_large_mechanism_per_species_error():
    mech = synthetic.jetsurf_shape()
    blob = pack.pack(mech).to_blob()
    ng = 4096
    P, T, Y = synthetic.states(mech.ns, ng, seed=31)
    gm = GpuMechanism(blob)
    w = _run(gm, P, T, Y, "mixed")
    r = oracle.rates(blob, P, T, Y, mech.nr)
    d = np.abs(w - r["wdot"])
    per_species_gross = (d / np.where(r["S"] > 0, r["S"], 1.0)).max(axis=1)
    e = oracle.errors(w, r["wdot"], r["S"])
    print("348/2163", e, "worst species (gross)", per_species_gross.max())
    assert np.all(np.isfinite(w))
    assert e["gross_max"] <= 1e-5 and e["norm_max"] <= 1e-4, e
