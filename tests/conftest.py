import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")
# a checkout of the reference repository, for the tests that read its
# mechanism files; those tests are skipped when it is not named
REFERENCE = os.environ.get("CHEMGEN_REFERENCE", "")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    import numpy as np
    from chemgen_b200.mechanism import Mechanism
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return Mechanism.from_json(str(d["mech"])), d


def reference_available():
    return bool(REFERENCE) and os.path.isdir(os.path.join(REFERENCE, "ck_files"))
