"""The oracle against the reference's own generated getrates (golden fixtures
made by tests/golden/make_golden.py) and against the data-free invariants."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from chemgen_b200 import pack, synthetic
from oracle import oracle


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_generated_code(name):
    mech, d = load_golden(name)
    blob = pack.pack(mech).to_blob()
    w = oracle.getrates(blob, d["P"], d["T"], d["Y"], nthreads=2)
    r = oracle.rates(blob, d["P"], d["T"], d["Y"], mech.nr, nthreads=2)
    assert np.array_equal(w, r["wdot"])
    for ref in ("wdot_scalar", "wdot_vec"):
        e = oracle.errors(w, d[ref], r["S"])
        # FP64 restatement of the same expressions: only libm rounding differs
        assert e["norm_max"] < 1e-13, (ref, e)
        assert e["gross_max"] < 1e-13, (ref, e)
    # most outputs are bit-identical to the generated Python
    assert np.mean(w == d["wdot_scalar"]) > 0.5


@pytest.mark.parametrize("name", ["h2_burke", "burke2012", "gri30"])
def test_real_mechanisms_conserve_mass(name):
    mech, d = load_golden(name)
    blob = pack.pack(mech).to_blob()
    r = oracle.rates(blob, d["P"], d["T"], d["Y"], mech.nr, nthreads=2)
    mw = np.array(mech.mw())[:, None]
    resid = np.abs((mw * r["wdot"]).sum(axis=0))
    scale = (mw * r["S"]).sum(axis=0)
    assert np.all(resid <= 1e-13 * scale + 1e-300)


def test_oracle_rejects_corrupt_blob():
    blob = bytearray(pack.pack(synthetic.h2o2_10sp()).to_blob())
    assert oracle.check_blob(bytes(blob)) == 0
    bad = bytes(blob[:100])
    assert oracle.check_blob(bad) != 0
    blob2 = bytearray(blob)
    blob2[0:8] = b"NOTMAGIC"
    assert oracle.check_blob(bytes(blob2)) == -2
