"""CPU checks of the surrogate's host logic: the MLP oracle's gradients
against torch autograd of the same network, the Adam schedule, and the
per-point fallback of SurrogateGetrates (with a fake network and a fake
exact kernel, so no GPU is needed)."""
import math

import pytest
import torch

from chemgen_b200 import surrogate as S
from oracle import mlp_ref


def test_oracle_gradients_equal_autograd():
    g = torch.Generator().manual_seed(0)
    dims = [16, 32, 32, 32, 8]
    W = [torch.randn(dims[l + 1], dims[l], generator=g) / math.sqrt(dims[l]) for l in range(4)]
    b = [torch.randn(dims[l + 1], generator=g) * 0.1 for l in range(4)]
    X = torch.randn(40, 16, generator=g)
    tgt = torch.randn(40, 8, generator=g)
    colw = torch.rand(8, generator=g)
    out, loss, gW, gb = mlp_ref.forward_backward(W, b, X, tgt, colw, round_bf16=False)
    Wv = [w.clone().requires_grad_(True) for w in W]
    bv = [x.clone().requires_grad_(True) for x in b]
    H = X
    for l in range(4):
        Z = H @ Wv[l].T + bv[l]
        H = mlp_ref.gelu(Z) if l < 3 else Z
    L = (colw * (H - tgt) ** 2).sum() / X.shape[0]
    L.backward()
    assert torch.allclose(L, loss, rtol=1e-6)
    for got, ref in zip(gW + gb, [w.grad for w in Wv] + [x.grad for x in bv]):
        assert torch.allclose(got, ref, rtol=1e-4, atol=1e-6)


def test_dgelu_matches_central_difference():
    z = torch.linspace(-6, 6, 241, dtype=torch.float64)
    h = 1e-6
    fd = (mlp_ref.gelu(z + h) - mlp_ref.gelu(z - h)) / (2 * h)
    assert torch.allclose(mlp_ref.dgelu(z), fd, atol=1e-8)


def test_adam_schedule_rows():
    s = S.adam_schedule(101, 1e-3, 1e-5)
    assert s.shape == (101, 3)
    assert abs(float(s[0, 0]) - 1e-3) < 1e-9 and abs(float(s[-1, 0]) - 1e-5) < 1e-9
    assert abs(float(s[0, 1]) - 10.0) < 1e-4            # 1 / (1 - 0.9)
    assert abs(float(s[0, 2]) - 1000.0) < 1e-1          # 1 / (1 - 0.999)
    assert (s[1:, 0] <= s[:-1, 0]).all()


class _FakeGM:
    def __init__(self):
        self.calls = []

    def getrates(self, P, T, Y, mode="fp64"):
        self.calls.append((T.clone(), mode))
        return torch.stack([T * (k + 1) for k in range(Y.shape[0])])


class _FakeSur:
    """Predicts -wdot_exact (wrong on purpose) with a chosen error estimate."""

    def __init__(self, est):
        self.gm = _FakeGM()
        self.est = est

    def predict(self, P, T, Y, check_range=False):
        est = self.est.clone()
        if check_range:                 # as the real one: +inf outside the training support
            est.masked_fill_(~self.in_range(P, T, Y), float("inf"))
        return -torch.stack([T * (k + 1) for k in range(Y.shape[0])]), est

    def in_range(self, P, T, Y):
        return (T >= 300) & (T <= 2500)


def test_fallback_replaces_untrusted_and_out_of_range_points():
    T = torch.tensor([400.0, 800.0, 3000.0, 1200.0, 1600.0], dtype=torch.float64)
    P = torch.full_like(T, 1013250.0)
    Y = torch.full((3, 5), 1.0 / 3, dtype=torch.float64)
    est = torch.tensor([-4.0, -1.0, -4.0, -2.5, -3.5])
    sur = _FakeSur(est)
    run = S.SurrogateGetrates(sur, tol=1e-3, exact_mode="mixed")
    W = run(P, T, Y)
    exact = torch.stack([T * (k + 1) for k in range(3)])
    # trusted and in range: points 0 and 4 keep the (negated) prediction
    assert torch.equal(W[:, [0, 4]], -exact[:, [0, 4]])
    # estimate above tolerance (1, 3) or T out of range (2): exact kernel
    assert torch.equal(W[:, [1, 2, 3]], exact[:, [1, 2, 3]])
    assert run.last_fallback == pytest.approx(3 / 5)
    (Tcalled, mode), = sur.gm.calls
    assert mode == "mixed" and torch.equal(Tcalled, T[[1, 2, 3]])


def test_no_fallback_call_when_all_trusted():
    T = torch.tensor([500.0, 900.0], dtype=torch.float64)
    sur = _FakeSur(torch.tensor([-5.0, -6.0]))
    run = S.SurrogateGetrates(sur, tol=1e-3)
    run(torch.full_like(T, 1013250.0), T, torch.full((2, 2), 0.5, dtype=torch.float64))
    assert sur.gm.calls == [] and run.last_fallback == 0.0


def test_gate_batch_growth_rule():
    """After an overflow the fixed batch grows to a quarter more than the
    failing points, in whole multiples of one wave (65536), never past ng."""
    g = S.SurrogateGetrates.grown_cap
    m = S.SurrogateGetrates.MIN_CAP
    assert m == 65536
    assert g(70000, 1 << 22) == 2 * m            # 87500 -> two waves
    assert g(4 * m, 1 << 22) == 5 * m            # 327680 exactly
    assert g(4 * m + 4, 1 << 22) == 6 * m
    assert g(200000, 150000) == 150000           # capped at ng
    assert g(1, 1 << 22) == m
