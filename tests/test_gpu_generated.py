"""Mechanism-specialised kernels (generate_chemistry.py --language cuda)
against the oracle and the reference's generated code, through the C ABI.
FP64 bar: 1e-10 normwise and gross-scaled.  Mixed bar: 1e-6 normwise
(max over points of max_k |dw_k| / max_k |w_k|)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from chemgen_b200 import pack, synthetic
from chemgen_b200.runtime import GpuMechanism
from oracle import oracle

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-10
TOL_MIXED = 1e-6


def _run(gm, P, T, Y, mode):
    import torch
    dev = torch.device("cuda", gm.device)
    Pt, Tt, Yt = (torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (P, T, Y))
    w = gm.getrates(Pt, Tt, Yt, mode=mode)
    torch.cuda.synchronize()
    return w.cpu().numpy()


SMALL = [n for n in golden_names() if load_golden(n)[0].ns <= 72]


@pytest.mark.parametrize("name", SMALL)
def test_generated_fp64_and_mixed_match_reference_golden(name):
    mech, d = load_golden(name)
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(mech, generated=True)
    assert gm.kernel_kind("fp64") == "generated" and gm.kernel_kind("mixed") == "generated"
    S = oracle.rates(blob, d["P"], d["T"], d["Y"], mech.nr)["S"]
    e = oracle.errors(_run(gm, d["P"], d["T"], d["Y"], "fp64"), d["wdot_scalar"], S)
    assert e["norm_max"] <= TOL_FP64 and e["gross_max"] <= TOL_FP64, e
    e = oracle.errors(_run(gm, d["P"], d["T"], d["Y"], "mixed"), d["wdot_scalar"], S)
    assert e["norm_max"] <= TOL_MIXED, e


@pytest.mark.parametrize("factory", [synthetic.all_kinds, synthetic.h2o2_10sp, synthetic.gri_shape])
@pytest.mark.parametrize("ng", [1, 63, 65, 4099])
def test_generated_ragged_sizes(factory, ng):
    mech = factory()
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, ng, seed=ng + 1)
    r = oracle.rates(blob, P, T, Y, mech.nr)
    gm = GpuMechanism(mech, generated=True)
    e = oracle.errors(_run(gm, P, T, Y, "fp64"), r["wdot"], r["S"])
    assert e["norm_max"] <= TOL_FP64 and e["gross_max"] <= TOL_FP64, e
    e = oracle.errors(_run(gm, P, T, Y, "mixed"), r["wdot"], r["S"])
    assert e["norm_max"] <= TOL_MIXED, e


def test_generated_and_table_kernels_agree_at_full_size():
    mech = synthetic.gri_shape()
    ng = 1 << 20
    P, T, Y = synthetic.states(mech.ns, ng, seed=21)
    gm = GpuMechanism(mech, generated=True)
    w_gen = _run(gm, P, T, Y, "fp64")
    w_mix = _run(gm, P, T, Y, "mixed")
    gm.use_generated(False)
    assert gm.kernel_kind("fp64") == "table"
    w_tab = _run(gm, P, T, Y, "fp64")
    e = oracle.errors(w_gen, w_tab)
    assert e["norm_max"] <= TOL_FP64, e
    e = oracle.errors(w_mix, w_tab)
    assert e["norm_max"] <= TOL_MIXED, e
    assert np.all(np.isfinite(w_mix))


def test_generated_mixed_edge_states():
    mech = synthetic.all_kinds()
    blob = pack.pack(mech).to_blob()
    ng = 300
    P, T, Y = synthetic.states(mech.ns, ng, seed=9)
    Y[:, ::3] = 0.0
    Y[0, ::3] = 1.0
    Y[::2, 1::3] = 0.0
    Y /= Y.sum(axis=0, keepdims=True)
    T[::5] = 1000.0
    T[1::7] = 300.0
    T[2::7] = 2500.0
    r = oracle.rates(blob, P, T, Y, mech.nr)
    gm = GpuMechanism(mech, generated=True)
    for mode, tol in (("fp64", TOL_FP64), ("mixed", TOL_MIXED)):
        w = _run(gm, P, T, Y, mode)
        assert np.all(np.isfinite(w))
        e = oracle.errors(w, r["wdot"], r["S"])
        assert e["norm_max"] <= tol, (mode, e)


def test_fp64_only_module_leaves_mixed_on_the_table_kernels(tmp_path):
    """A module generated with precision="fp64" registers the FP64 mode only:
    mixed runs on the table-driven (tensor-core) kernel, both stay in parity.
    (A mechanism no other test loads: kernel registration is process-wide.)"""
    import ctypes
    import torch
    from chemgen_b200 import emit_cuda
    from chemgen_b200.runtime import lib
    mech = synthetic.synthetic_mechanism(12, 30, 3, 2, seed=77, name="synthetic_12_30_s77")
    so = emit_cuda.build_module(mech, out=str(tmp_path / "fp64only.so"), precision="fp64")
    lib()
    ctypes.CDLL(so, mode=ctypes.RTLD_GLOBAL)
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(blob)
    assert gm.kernel_kind("fp64") == "generated" and gm.kernel_kind("mixed") == "table"
    P, T, Y = synthetic.states(mech.ns, 3000, seed=5)
    S = oracle.rates(blob, P, T, Y, mech.nr)["S"]
    w_ref = oracle.getrates(blob, P, T, Y)
    Pd, Td, Yd = (torch.from_numpy(x).cuda() for x in (P, T, Y))
    e64 = oracle.errors(gm.getrates(Pd, Td, Yd, mode="fp64").cpu().numpy(), w_ref, S)
    emx = oracle.errors(gm.getrates(Pd, Td, Yd, mode="mixed").cpu().numpy(), w_ref, S)
    assert e64["norm_max"] <= 1e-10 and emx["norm_max"] <= 1e-6, (e64, emx)


def test_tensor_memory_gibbs_terms_in_both_kernels(tmp_path):
    """emit(tmem=True) keeps the Gibbs array in tensor memory in both kernels
    (the default for the FP64 kernel when it lets the block grow; an option
    for the mixed kernel, where it measured slower): both stay in parity with
    the oracle on a ragged point count.  (A mechanism no other test loads:
    kernel registration is process-wide.)"""
    import ctypes
    import torch
    from chemgen_b200 import emit_cuda
    from chemgen_b200.runtime import lib
    mech = synthetic.synthetic_mechanism(20, 60, 4, 4, seed=91, name="synthetic_20_60_s91")
    assert emit_cuda.emit(mech, tmem=True).count("cgg::tm_alloc") == 2
    so = emit_cuda.build_module(mech, out=str(tmp_path / "tmem.so"), tmem=True)
    lib()
    ctypes.CDLL(so, mode=ctypes.RTLD_GLOBAL)
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(blob)
    assert gm.kernel_kind("fp64") == "generated" and gm.kernel_kind("mixed") == "generated"
    P, T, Y = synthetic.states(mech.ns, 3017, seed=6)
    S = oracle.rates(blob, P, T, Y, mech.nr)["S"]
    w_ref = oracle.getrates(blob, P, T, Y)
    Pd, Td, Yd = (torch.from_numpy(x).cuda() for x in (P, T, Y))
    e64 = oracle.errors(gm.getrates(Pd, Td, Yd, mode="fp64").cpu().numpy(), w_ref, S)
    emx = oracle.errors(gm.getrates(Pd, Td, Yd, mode="mixed").cpu().numpy(), w_ref, S)
    assert e64["norm_max"] <= 1e-10 and emx["norm_max"] <= 1e-6, (e64, emx)
