"""CUDA getrates against the oracle and the reference's generated code, all
through the C ABI.  FP64 bar: normwise error <= 1e-10 (max over points of
max_k |dw_k| / max_k |w_k|) and gross-scaled error <= 1e-10."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from chemgen_b200 import pack, synthetic
from chemgen_b200.runtime import GpuMechanism
from oracle import oracle

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-10


def _run(gm, P, T, Y, mode="fp64"):
    import torch
    dev = torch.device("cuda", gm.device)
    Pt = torch.from_numpy(np.ascontiguousarray(P)).to(dev)
    Tt = torch.from_numpy(np.ascontiguousarray(T)).to(dev)
    Yt = torch.from_numpy(np.ascontiguousarray(Y)).to(dev)
    w = gm.getrates(Pt, Tt, Yt, mode=mode)
    torch.cuda.synchronize()
    return w.cpu().numpy()


@pytest.mark.parametrize("name", golden_names())
def test_fp64_matches_reference_golden(name):
    mech, d = load_golden(name)
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(blob)
    w = _run(gm, d["P"], d["T"], d["Y"])
    S = oracle.rates(blob, d["P"], d["T"], d["Y"], mech.nr)["S"]
    for ref in ("wdot_scalar", "wdot_vec"):
        e = oracle.errors(w, d[ref], S)
        assert e["norm_max"] <= TOL_FP64 and e["gross_max"] <= TOL_FP64, (ref, e)


@pytest.mark.parametrize("factory", [synthetic.all_kinds, synthetic.h2o2_10sp, synthetic.gri_shape])
@pytest.mark.parametrize("ng", [1, 31, 33, 1000])
def test_fp64_matches_oracle_ragged_sizes(factory, ng):
    mech = factory()
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, ng, seed=ng)
    w = _run(GpuMechanism(blob), P, T, Y)
    r = oracle.rates(blob, P, T, Y, mech.nr)
    e = oracle.errors(w, r["wdot"], r["S"])
    assert e["norm_max"] <= TOL_FP64 and e["gross_max"] <= TOL_FP64, e


def test_fp64_exact_zeros_and_range_switch():
    mech = synthetic.all_kinds()
    blob = pack.pack(mech).to_blob()
    ng = 257
    P, T, Y = synthetic.states(mech.ns, ng, seed=5)
    Y[:, ::3] = 0.0
    Y[0, ::3] = 1.0                      # pure species
    Y[::2, 1::3] = 0.0
    Y /= Y.sum(axis=0, keepdims=True)
    T[::7] = 1000.0                       # every species switches range here
    w = _run(GpuMechanism(blob), P, T, Y)
    r = oracle.rates(blob, P, T, Y, mech.nr)
    e = oracle.errors(w, r["wdot"], r["S"])
    assert np.all(np.isfinite(w))
    assert e["norm_max"] <= TOL_FP64 and e["gross_max"] <= TOL_FP64, e


def test_fp64_empty_input_is_a_no_op():
    import torch
    gm = GpuMechanism(synthetic.h2o2_10sp())
    z = torch.empty(0, dtype=torch.float64, device="cuda")
    w = gm.getrates(z, z, torch.empty(gm.ns, 0, dtype=torch.float64, device="cuda"))
    assert w.shape == (gm.ns, 0)


def test_fp64_full_size_53_325_subsample_and_mass():
    """2^20 points of the 53/325 workload; the oracle checks a seeded subsample."""
    mech = synthetic.gri_shape()
    blob = pack.pack(mech).to_blob()
    ng = 1 << 20
    P, T, Y = synthetic.states(mech.ns, ng, seed=11)
    w = _run(GpuMechanism(blob), P, T, Y)
    assert np.all(np.isfinite(w))
    idx = np.sort(np.random.default_rng(0).choice(ng, 2048, replace=False))
    r = oracle.rates(blob, P[idx], T[idx], np.ascontiguousarray(Y[:, idx]), mech.nr)
    e = oracle.errors(w[:, idx], r["wdot"], r["S"])
    assert e["norm_max"] <= TOL_FP64 and e["gross_max"] <= TOL_FP64, e


def test_fp64_real_gri30_conserves_mass_at_size():
    mech, d = load_golden("gri30")
    blob = pack.pack(mech).to_blob()
    ng = 1 << 18
    P, T, Y = synthetic.states(mech.ns, ng, seed=3)
    w = _run(GpuMechanism(blob), P, T, Y)
    mw = np.array(mech.mw())[:, None]
    idx = np.arange(0, ng, 97)
    S = oracle.rates(blob, P[idx], T[idx], np.ascontiguousarray(Y[:, idx]), mech.nr)["S"]
    resid = np.abs((mw * w[:, idx]).sum(axis=0))
    assert np.all(resid <= 1e-12 * (mw * S).sum(axis=0))


def test_host_pointer_path_matches_device_path():
    mech = synthetic.gri_shape()
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(blob)
    ng = 300001
    P, T, Y = synthetic.states(mech.ns, ng, seed=2)
    w_dev = _run(gm, P, T, Y)
    w_host = gm.getrates_host(P, T, Y)
    assert np.array_equal(w_dev, w_host)


def test_workspace_variant_large_mechanism():
    """348 species: the FP64 staged kernel keeps its state on chip (no
    workspace); the mixed tensor-core kernel keeps its Gibbs terms in the
    caller's workspace."""
    mech, d = load_golden("jetsurf2")
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(blob)
    import torch
    ng = d["T"].size
    assert gm.workspace_bytes(ng, "fp64") == 0
    assert gm.workspace_bytes(ng, "mixed") > 0
    S = oracle.rates(blob, d["P"], d["T"], d["Y"], mech.nr)["S"]
    Pt, Tt, Yt = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (d["P"], d["T"], d["Y"]))
    for mode, tol in (("fp64", TOL_FP64), ("mixed", 1e-6)):
        wb = gm.workspace_bytes(ng, mode)
        ws = torch.empty(wb // 8 + 64, dtype=torch.float64, device="cuda") if wb else None
        out = torch.empty_like(Yt)
        gm.getrates_ws(Pt, Tt, Yt, out, ws, mode=mode)
        torch.cuda.synchronize()
        e = oracle.errors(out.cpu().numpy(), d["wdot_scalar"], S)
        assert e["norm_max"] <= tol, (mode, e)


@pytest.mark.parametrize("name,ng", [("jetsurf2", 1), ("jetsurf2", 33), ("jetsurf2", 1000),
                                     ("synthetic_348_2163", 777)])
def test_staged_fp64_kernel_large_mechanisms(name, ng):
    """The staged FP64 kernel (32-point tiles, C and EGp in shared memory,
    reactions in chunks, species-owned register accumulators) at ragged
    sizes, against the oracle and against the global-scratch FP64 kernel that
    the no-allocation entry point runs."""
    import torch
    from chemgen_b200.runtime import lib
    mech, _ = load_golden(name)
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(blob)
    assert gm.workspace_bytes(ng, "fp64") == 0
    P, T, Y = synthetic.states(mech.ns, ng, seed=ng)
    w = _run(gm, P, T, Y)
    r = oracle.rates(blob, P, T, Y, mech.nr)
    e = oracle.errors(w, r["wdot"], r["S"])
    assert e["norm_max"] <= TOL_FP64 and e["gross_max"] <= TOL_FP64, e
    Pt, Tt, Yt = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (P, T, Y))
    w2 = torch.empty_like(Yt)
    assert lib().chemgen_getrates_noalloc(gm.handle, Pt.data_ptr(), Tt.data_ptr(), ng, Yt.data_ptr(),
                                          w2.data_ptr(), torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert oracle.errors(w, w2.cpu().numpy())["norm_max"] <= TOL_FP64


def test_reference_wrapper_drop_in():
    """getrates_hip_wrapper_v1 with the reference's signature and scratch."""
    import ctypes
    import torch
    from chemgen_b200.runtime import lib
    for name in ("gri30", "jetsurf2"):
        mech, d = load_golden(name)
        blob = pack.pack(mech).to_blob()
        buf = ctypes.create_string_buffer(blob, len(blob))
        assert lib().chemgen_init_constants(buf, len(blob)) == 0
        ng = d["T"].size
        Pt, Tt, Yt = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (d["P"], d["T"], d["Y"]))
        w = torch.zeros_like(Yt)
        eg = torch.empty_like(Yt)
        c = torch.empty_like(Yt)
        lib().getrates_hip_wrapper_v1(Pt.data_ptr(), Tt.data_ptr(), ng, Yt.data_ptr(), w.data_ptr(),
                                      eg.data_ptr(), c.data_ptr())
        assert lib().chemgen_last_wrapper_status() == 0
        S = oracle.rates(blob, d["P"], d["T"], d["Y"], mech.nr)["S"]
        e = oracle.errors(w.cpu().numpy(), d["wdot_scalar"], S)
        assert e["norm_max"] <= TOL_FP64, e
    assert lib().chemgen_free_constants() == 0
    lib().getrates_hip_wrapper_v1(0, 0, 1, 0, 0, 0, 0)
    assert lib().chemgen_last_wrapper_status() == 8


@pytest.mark.parametrize("version", [1, 2, 3, 4])
def test_fortran_module_call_sequence(tmp_path, monkeypatch, version):
    """What chemgen_m (include/chemgen_m.F90) does, through the same symbols:
    init_chemgen loads the blob file named by CHEMGEN_BLOB, sizes EG and C from
    chemgen_global_num_species, reserves scratch for v4, and getrates_gpu calls
    getrates_hip_wrapper_v<version> (chemgen_mod.j2:108-166)."""
    import torch
    from chemgen_b200.runtime import lib
    L = lib()
    for name in ("h2_burke", "jetsurf2"):
        mech, d = load_golden(name)
        blob = pack.pack(mech).to_blob()
        path = tmp_path / f"{name}.blob"
        path.write_bytes(blob)
        monkeypatch.setenv("CHEMGEN_BLOB", str(path))
        assert L.chemgen_init_constants_file(None) == 0
        ns = L.chemgen_global_num_species()
        assert ns == mech.ns
        ng = d["T"].size
        if version == 4:
            L.allocate_intermediate_DeviceMemory(ng)
            assert L.chemgen_last_wrapper_status() == 0
        Pt, Tt, Yt = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (d["P"], d["T"], d["Y"]))
        w = torch.zeros_like(Yt)
        eg = torch.empty((ns, ng), dtype=torch.float64, device="cuda")
        c = torch.empty((ns, ng), dtype=torch.float64, device="cuda")
        getattr(L, f"getrates_hip_wrapper_v{version}")(Pt.data_ptr(), Tt.data_ptr(), ng, Yt.data_ptr(),
                                                        w.data_ptr(), eg.data_ptr(), c.data_ptr())
        assert L.chemgen_last_wrapper_status() == 0
        S = oracle.rates(blob, d["P"], d["T"], d["Y"], mech.nr)["S"]
        e = oracle.errors(w.cpu().numpy(), d["wdot_scalar"], S)
        assert e["norm_max"] <= TOL_FP64, (name, e)
    assert L.chemgen_free_constants() == 0
    assert L.chemgen_global_num_species() == -1


def test_bad_arguments_return_status():
    import torch
    from chemgen_b200.runtime import ChemgenError
    gm = GpuMechanism(synthetic.h2o2_10sp())
    x = torch.ones(9, dtype=torch.float64, device="cuda")
    with pytest.raises(ChemgenError):
        gm.getrates_ptr(x.data_ptr() + 4, x.data_ptr(), 1, x.data_ptr(), x.data_ptr())
    with pytest.raises(ChemgenError):
        gm.getrates_ptr(x.data_ptr(), x.data_ptr(), -1, x.data_ptr(), x.data_ptr())


def test_kernel_exp_log_against_cuda_libm():
    import torch
    from chemgen_b200.runtime import lib
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-740, 705, 200000), rng.uniform(-1, 1, 100000),
                        np.exp(rng.uniform(-700, 700, 100000)), [0.0, -0.0, 1.0, 2.0, 700.0, -708.0]])
    xt = torch.from_numpy(x).cuda()
    outs = [torch.empty_like(xt) for _ in range(4)]
    assert lib().chemgen_probe_math(ctypes_ptr(xt), x.size, *(ctypes_ptr(o) for o in outs)) == 0
    e, l, er, lr = (o.cpu().numpy() for o in outs)
    ok = (er > 1e-300) & np.isfinite(er)
    assert np.max(np.abs(e[ok] - er[ok]) / er[ok]) < 1e-15
    assert np.all(np.isinf(e[np.isinf(er)]))
    # the documented ends of cg_exp: +inf from x >= 1023.5 ln 2, zero at and
    # below -1022.5 ln 2 (flushed, where CUDA's exp is subnormal)
    hi = np.linspace(1023.5 * np.log(2) + 1e-12, 709.78, 64)
    lo = np.linspace(-745.0, -1022.5 * np.log(2) - 1e-12, 64)
    xe = torch.from_numpy(np.concatenate([hi, lo])).cuda()
    oe = [torch.empty_like(xe) for _ in range(4)]
    assert lib().chemgen_probe_math(ctypes_ptr(xe), xe.numel(), *(ctypes_ptr(o) for o in oe)) == 0
    ee, _, eer, _ = (o.cpu().numpy() for o in oe)
    assert np.all(np.isinf(ee[:64])) and np.all(np.isfinite(eer[:64]))
    assert np.all(ee[64:] == 0.0) and np.all(eer[64:] < 2.0 ** -1022)
    ok = np.abs(lr) > 1e-3
    assert np.max(np.abs(l[ok] - lr[ok]) / np.abs(lr[ok])) < 1e-15
    assert np.max(np.abs(l - lr)) < 1e-15 * 800


def ctypes_ptr(t):
    return t.data_ptr()


def test_point_major_layout_matches_species_major():
    """Y given per point ([ng, ns], the reference's getrates_i layout): same
    wdot, returned in that layout, and the same gradients through autograd."""
    import torch
    from chemgen_b200 import getrates
    mech = synthetic.h2o2_10sp()
    gm = GpuMechanism(mech)
    P, T, Y = (torch.from_numpy(x).cuda() for x in synthetic.states(mech.ns, 777, seed=11))
    w_sm = gm.getrates(P, T, Y)
    w_pm = gm.getrates(P, T, Y.t().contiguous(), layout="point_major")
    assert w_pm.shape == (777, mech.ns) and torch.equal(w_pm, w_sm.t())
    Ys = Y.clone().requires_grad_(True)
    Yp = Y.t().contiguous().requires_grad_(True)
    G = torch.randn(mech.ns, 777, dtype=torch.float64, device="cuda")
    (getrates(gm, P, T, Ys) * G).sum().backward()
    (getrates(gm, P, T, Yp, layout="point_major") * G.t()).sum().backward()
    assert torch.equal(Yp.grad.t(), Ys.grad)
    with pytest.raises(ValueError):
        gm.getrates(P, T, Y, layout="rows")


@pytest.mark.parametrize("factory,counts", [(synthetic.h2o2_10sp, [0, 1, 777, 4096, 10 ** 9]),
                                            (synthetic.gri_shape, [0, 33, 4095, 4096])])
def test_counted_getrates_computes_only_the_counted_points(factory, counts):
    """chemgen_getrates_counted: with the count on the device, the first
    min(count, ng) points equal the staged FP64 kernel's (and the oracle's
    within the FP64 bar), and the rest of the output is left as it was; a
    count past ng covers every point."""
    import torch
    from chemgen_b200.runtime import lib
    mech = factory()
    blob = pack.pack(mech).to_blob()
    ng = 4096
    P, T, Y = synthetic.states(mech.ns, ng, seed=17)
    gm = GpuMechanism(blob)
    dev = torch.device("cuda", 0)
    Pt, Tt, Yt = (torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (P, T, Y))
    r = oracle.rates(blob, P, T, Y, mech.nr)
    s = torch.cuda.current_stream().cuda_stream
    for c in counts:
        count = torch.tensor([c], dtype=torch.int64, device=dev)
        W = torch.full((mech.ns, ng), -3.0, dtype=torch.float64, device=dev)
        assert lib().chemgen_getrates_counted(gm._h, Pt.data_ptr(), Tt.data_ptr(), ng, Yt.data_ptr(), W.data_ptr(),
                                              count.data_ptr(), s) == 0
        torch.cuda.synchronize()
        n = min(c, ng)
        w = W.cpu().numpy()
        assert (w[:, n:] == -3.0).all()
        if n:
            e = oracle.errors(w[:, :n], r["wdot"][:, :n], r["S"][:, :n])
            assert e["norm_max"] <= TOL_FP64, e
    assert lib().chemgen_getrates_counted(gm._h, Pt.data_ptr(), Tt.data_ptr(), ng, Yt.data_ptr(), W.data_ptr(),
                                          0, s) == 1
