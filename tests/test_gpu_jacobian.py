"""Analytic Jacobian and adjoint kernels against central finite differences
(h = 1e-6 * max(|x|, floor)) of the FP64 oracle and against torch autograd
through the FP64 torch restatement of the reference's getrates."""
import numpy as np
import pytest

from conftest import load_golden
from chemgen_b200 import pack, synthetic
from chemgen_b200.runtime import GpuMechanism
from oracle import oracle

pytestmark = pytest.mark.gpu


def _t(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def fd_jacobian(blob, P, T, Y, floor_y=1e-8, rel=1e-6):
    """Central differences of the oracle: [ns, ns+1, ng]."""
    ns, ng = Y.shape
    J = np.empty((ns, ns + 1, ng))
    h = rel * np.maximum(T, 1.0)
    wp = oracle.getrates(blob, P, T + h, Y)
    wm = oracle.getrates(blob, P, T - h, Y)
    J[:, 0, :] = (wp - wm) / (2 * h)
    for j in range(ns):
        h = rel * np.maximum(np.abs(Y[j]), floor_y)
        Yp, Ym = Y.copy(), Y.copy()
        Yp[j] += h
        Ym[j] -= h
        J[:, 1 + j, :] = (oracle.getrates(blob, P, T, Yp) - oracle.getrates(blob, P, T, Ym)) / (2 * h)
    return J


def _rel(a, b):
    """max over points of ||a - b|| / ||b|| (Frobenius per point)."""
    num = np.sqrt(((a - b) ** 2).sum(axis=(0, 1)))
    den = np.sqrt((b ** 2).sum(axis=(0, 1)))
    return float((num / den).max())


def _wide_90():
    """90 species, 150 reactions: a wider mechanism, whose per-point state
    (4 x 90 doubles) and J (90 x 91) stress the scratch and J strides."""
    return synthetic.synthetic_mechanism(90, 150, 12, 12, seed=11, name="synthetic_90_150")


@pytest.mark.parametrize("factory", [synthetic.h2o2_10sp, synthetic.all_kinds, synthetic.gri_shape, _wide_90])
def test_jacobian_matches_central_differences(factory):
    mech = factory()
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, 40, seed=3)
    Y = np.maximum(Y, 1e-6)
    Y /= Y.sum(axis=0, keepdims=True)
    gm = GpuMechanism(blob)
    J = gm.jacobian(_t(P), _t(T), _t(Y)).cpu().numpy()
    Jfd = fd_jacobian(blob, P, T, Y)
    assert _rel(J, Jfd) < 1e-5


def test_jacobian_large_mechanism_scratch_path():
    """348 species: beyond the row-owner kernel's shared memory, J is
    accumulated in place with library scratch; central differences agree."""
    mech, d = load_golden("jetsurf2")
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, 8, seed=13)
    Y = np.maximum(Y, 1e-6)
    Y /= Y.sum(axis=0, keepdims=True)
    J = GpuMechanism(blob).jacobian(_t(P), _t(T), _t(Y)).cpu().numpy()
    Jfd = fd_jacobian(blob, P, T, Y)
    assert _rel(J, Jfd) < 1e-4


@pytest.mark.parametrize("name", ["h2_burke", "synthetic_plog_15_40"])
def test_jacobian_matches_autograd_through_fp64_reference(name):
    import torch
    from oracle import torch_ref
    mech, d = load_golden(name)
    blob = pack.pack(mech).to_blob()
    ng = 24
    P, T, Y = d["P"][:ng], d["T"][:ng], np.ascontiguousarray(d["Y"][:, :ng])
    gm = GpuMechanism(blob)
    J = gm.jacobian(_t(P), _t(T), _t(Y)).cpu().numpy()
    Pt = torch.from_numpy(P)
    Ja = np.empty_like(J)
    for i in range(ng):
        def f(x):
            return torch_ref.getrates(mech, Pt[i:i + 1], x[:1], x[1:, None])[:, 0]
        x = torch.cat([torch.from_numpy(T[i:i + 1]), torch.from_numpy(Y[:, i])])
        Ja[:, :, i] = torch.autograd.functional.jacobian(f, x).numpy()
    assert _rel(J, Ja) < 1e-9


def autograd_jacobian(mech, P, T, Y):
    """J [ns, ns+1, ng] of the FP64 torch restatement by reverse-mode autograd:
    points are independent, so one backward pass per species (a one-hot
    output weight at every point) gives that species' row at all points."""
    import torch
    from oracle import torch_ref
    Tt = torch.from_numpy(np.ascontiguousarray(T)).requires_grad_(True)
    Yt = torch.from_numpy(np.ascontiguousarray(Y)).requires_grad_(True)
    w = torch_ref.getrates(mech, torch.from_numpy(np.ascontiguousarray(P)), Tt, Yt)
    ns, ng = Y.shape
    J = np.empty((ns, ns + 1, ng))
    for k in range(ns):
        gT, gY = torch.autograd.grad(w[k].sum(), (Tt, Yt), retain_graph=k + 1 < ns)
        J[k, 0, :] = gT.numpy()
        J[k, 1:, :] = gY.numpy()
    return J


@pytest.mark.parametrize("name", ["gri30", "synthetic_53_325"])
def test_jacobian_53_species_matches_autograd_through_fp64_reference(name):
    """The C4 configuration's mechanisms (53 species): the FP64 analytic
    Jacobian within 1e-9 and the FP32 one within 1e-5 of autograd through the
    FP64 torch restatement, per point (Frobenius norm)."""
    mech, d = load_golden(name)
    blob = pack.pack(mech).to_blob()
    ng = 96
    P, T, Y = d["P"][:ng], d["T"][:ng], np.ascontiguousarray(d["Y"][:, :ng])
    gm = GpuMechanism(blob)
    Ja = autograd_jacobian(mech, P, T, Y)
    J64 = gm.jacobian(_t(P), _t(T), _t(Y), "fp64").cpu().numpy()
    J32 = gm.jacobian(_t(P), _t(T), _t(Y), "fp32").cpu().numpy().astype(np.float64)
    e64, e32 = _rel(J64, Ja), _rel(J32, Ja)
    print(name, "fp64", e64, "fp32", e32)
    assert e64 < 1e-9
    assert e32 < 1e-5


def test_fp32_jacobian_close_to_fp64():
    mech = synthetic.gri_shape()
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, 65536, seed=4)
    gm = GpuMechanism(blob)
    J64 = gm.jacobian(_t(P), _t(T), _t(Y), "fp64").cpu().numpy()
    J32 = gm.jacobian(_t(P), _t(T), _t(Y), "fp32").cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(J64))
    assert _rel(J32, J64) < 1e-5


def test_vjp_equals_jacobian_transpose_and_autograd_function():
    import torch
    from chemgen_b200.autograd import getrates
    mech = synthetic.all_kinds()
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, 500, seed=8)
    gm = GpuMechanism(blob)
    Pt, Tt, Yt = _t(P), _t(T), _t(Y)
    G = torch.randn(mech.ns, 500, dtype=torch.float64, device="cuda")
    J = gm.jacobian(Pt, Tt, Yt)
    gT, gY, gP = gm.vjp(Pt, Tt, Yt, G)
    ref_T = (J[:, 0, :] * G).sum(0)
    ref_Y = torch.einsum("kjn,kn->jn", J[:, 1:, :], G)
    assert torch.allclose(gT, ref_T, rtol=1e-9, atol=1e-9 * ref_T.abs().max().item())
    assert torch.allclose(gY, ref_Y, rtol=1e-9, atol=1e-9 * ref_Y.abs().max().item())
    # dL/dP against central differences of the forward kernel
    h = 1e-6 * Pt
    wp = gm.getrates(Pt + h, Tt, Yt)
    wm = gm.getrates(Pt - h, Tt, Yt)
    fdP = ((wp - wm) * G).sum(0) / (2 * h)
    assert torch.allclose(gP, fdP, rtol=1e-5, atol=1e-6 * fdP.abs().max().item())
    # autograd.Function: backward is the adjoint kernel
    Tr, Yr = Tt.clone().requires_grad_(True), Yt.clone().requires_grad_(True)
    w = getrates(gm, Pt, Tr, Yr)
    (w * G).sum().backward()
    assert torch.allclose(Tr.grad, gT) and torch.allclose(Yr.grad, gY)


@pytest.mark.parametrize("name,ng", [("gri30", 32 * 70 + 5), ("synthetic_53_325", 65536)])
def test_vjp_53_species_matches_jacobian_transpose(name, ng):
    """The C4 mechanisms on the tile adjoint kernel (shared-memory state,
    per-warp accumulators added in a fixed order), ragged last tile included:
    the VJP equals J^T G from the row-owner Jacobian, and two calls agree bit
    for bit."""
    import torch
    mech, d = load_golden(name)
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, ng, seed=21)
    gm = GpuMechanism(blob)
    Pt, Tt, Yt = _t(P), _t(T), _t(Y)
    G = torch.randn(mech.ns, ng, dtype=torch.float64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(5))
    J = gm.jacobian(Pt, Tt, Yt)
    gT, gY, gP = gm.vjp(Pt, Tt, Yt, G)
    gT2, gY2, gP2 = gm.vjp(Pt, Tt, Yt, G)
    assert torch.equal(gT, gT2) and torch.equal(gY, gY2) and torch.equal(gP, gP2)
    ref_T = (J[:, 0, :] * G).sum(0)
    ref_Y = torch.einsum("kjn,kn->jn", J[:, 1:, :], G)
    # per point, relative to that point's largest term
    eT = ((gT - ref_T).abs() / (J[:, 0, :].abs() * G.abs()).sum(0).clamp_min(1e-300)).max().item()
    eY = ((gY - ref_Y).abs().max(0).values /
          torch.einsum("kjn,kn->jn", J[:, 1:, :].abs(), G.abs()).max(0).values.clamp_min(1e-300)).max().item()
    assert eT < 1e-10 and eY < 1e-10, (eT, eY)


def test_jacobian_with_zero_species_is_exact():
    """Y_j = 0 exactly: the analytic derivative must not vanish where FD says it doesn't."""
    import torch
    from oracle import torch_ref
    mech = synthetic.h2o2_10sp()
    blob = pack.pack(mech).to_blob()
    P, T, Y = synthetic.states(mech.ns, 8, seed=2)
    Y[3, :] = 0.0
    Y /= Y.sum(axis=0, keepdims=True)
    J = GpuMechanism(blob).jacobian(_t(P), _t(T), _t(Y)).cpu().numpy()
    for i in range(8):
        def f(x):
            return torch_ref.getrates(mech, torch.from_numpy(P[i:i + 1]), x[:1], x[1:, None])[:, 0]
        x = torch.cat([torch.from_numpy(T[i:i + 1]), torch.from_numpy(Y[:, i])])
        Ja = torch.autograd.functional.jacobian(f, x).numpy()
        assert np.abs(J[:, :, i] - Ja).max() <= 1e-9 * np.abs(Ja).max()
        assert np.abs(J[:, 4, i]).max() > 0      # column of the absent species
