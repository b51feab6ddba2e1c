"""The torch FP64 restatement (autograd checker) agrees with the C oracle."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from chemgen_b200 import pack
from oracle import oracle


@pytest.mark.parametrize("name", ["h2_burke", "burke2012", "synthetic_plog_15_40", "synthetic_h2o2_10_27"])
def test_torch_reference_matches_oracle(name):
    import torch
    from oracle import torch_ref
    mech, d = load_golden(name)
    w = torch_ref.getrates(mech, torch.from_numpy(d["P"]), torch.from_numpy(d["T"]), torch.from_numpy(d["Y"]))
    e = oracle.errors(w.numpy(), d["wdot_scalar"])
    assert e["norm_max"] < 1e-12, e
