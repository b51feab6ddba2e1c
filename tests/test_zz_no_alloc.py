"""chemgen_getrates_noalloc -- the entry point for callers that cannot
allocate device memory while they run -- against chemgen_getrates, the
allocating entry point, through the C ABI.  Two calls in a row on different
states share the library's fixed scratch array; each must match the FP64
tolerance of the other GPU tests (1e-10 normwise).  Collected last so that a
run stopping at the first failure has run every other test first."""
import numpy as np
import pytest

from conftest import load_golden
from chemgen_b200 import pack, synthetic
from chemgen_b200.runtime import GpuMechanism, lib
from oracle import oracle

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-10


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("which", ["jetsurf2", "h2o2"])
def test_noalloc_matches_allocating_entry_point_twice(which):
    import torch
    if which == "jetsurf2":
        mech, _ = load_golden("jetsurf2")      # 348 species: the no-alloc entry point keeps state in scratch
    else:
        mech = synthetic.h2o2_10sp()           # small: the allocating entry point keeps it in shared memory
    gm = GpuMechanism(pack.pack(mech).to_blob())
    for seed in (11, 12):                      # two calls in a row on different states
        P, T, Y = synthetic.states(mech.ns, 3001, seed=seed)
        Pt, Tt, Yt = _dev(P), _dev(T), _dev(Y)
        w_ref = torch.empty_like(Yt)
        w_na = torch.full_like(Yt, float("nan"))
        s = torch.cuda.current_stream().cuda_stream
        assert lib().chemgen_getrates(gm.handle, Pt.data_ptr(), Tt.data_ptr(), 3001, Yt.data_ptr(),
                                      w_ref.data_ptr(), s) == 0
        assert lib().chemgen_getrates_noalloc(gm.handle, Pt.data_ptr(), Tt.data_ptr(), 3001, Yt.data_ptr(),
                                              w_na.data_ptr(), s) == 0
        torch.cuda.synchronize()
        e = oracle.errors(w_na.cpu().numpy(), w_ref.cpu().numpy())
        assert e["norm_max"] <= TOL_FP64, (seed, e)


def test_noalloc_rejects_bad_arguments():
    import torch
    gm = GpuMechanism(pack.pack(synthetic.h2o2_10sp()).to_blob())
    x = torch.ones(64, dtype=torch.float64, device="cuda")
    assert lib().chemgen_getrates_noalloc(None, x.data_ptr(), x.data_ptr(), 1, x.data_ptr(), x.data_ptr(), None) == 1
    assert lib().chemgen_getrates_noalloc(gm.handle, x.data_ptr() + 4, x.data_ptr(), 1, x.data_ptr(),
                                          x.data_ptr(), None) == 5
    assert lib().chemgen_getrates_noalloc(gm.handle, x.data_ptr(), x.data_ptr(), 0, x.data_ptr(),
                                          x.data_ptr(), None) == 0
