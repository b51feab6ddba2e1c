"""ORACLE -- test infrastructure only.  CPU restatement of the surrogate
MLP's forward and backward (chemgen_b200/surrogate.py, csrc/mlp.cu) in torch
FP32, with the same BF16 roundings of weights, activations and gradients the
GPU kernels apply, so that their parameter gradients can be checked; with
`round_bf16=False` it is the plain FP32 network (what the BF16 kernels
approximate).  The GPU kernels take tanh inside GELU from the hardware
approximation (relative error about 2^-11); this oracle uses exact tanh, and
the tests' tolerances allow for the difference.  The surrogate has no
counterpart in the reference (its
chemgen/chemistry_nn.py:15-85 prototype never ran), so this oracle is
pinned by the CPU tests of its own algebra (central differences of the FP32
network), not by reference vectors.
"""
from __future__ import annotations

import math

import torch


def _r(x, on):
    return x.to(torch.bfloat16).to(torch.float32) if on else x


def gelu(z):
    k0, k1 = math.sqrt(2.0 / math.pi), 0.044715
    return 0.5 * z * (1.0 + torch.tanh(k0 * (z + k1 * z ** 3)))


def dgelu(z):
    k0, k1 = math.sqrt(2.0 / math.pi), 0.044715
    t = torch.tanh(k0 * (z + k1 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * k0 * (1.0 + 3.0 * k1 * z * z)


def forward(W, b, X, round_bf16=True):
    """Output [B, dout] and the kept (acts, zs) of the network."""
    Wr = [_r(w, round_bf16) for w in W]
    acts, zs = [X], []
    H = X
    for l in range(4):
        Z = H @ Wr[l].T + b[l]
        zs.append(Z)
        if l < 3:
            H = _r(gelu(Z), round_bf16)
            acts.append(H)
    return zs[-1], acts, zs, Wr


def forward_backward(W, b, X, target, colw, round_bf16=True):
    """W[l]: [n, k] FP32 master weights, b[l]: [n]; X: [B, din] (values the
    kernels see, already BF16 or a sum of BF16 parts); returns (out, loss,
    gW list, gb list) of loss = mean_rows sum_j colw_j (out - target)^2."""
    B = X.shape[0]
    out, acts, zs, Wr = forward(W, b, X, round_bf16)
    d = out - target
    loss = (colw * d * d).sum() / B
    dZf = 2.0 * colw * d / B
    dZb = _r(dZf, round_bf16)
    gW, gb = [None] * 4, [None] * 4
    for l in range(3, -1, -1):
        gW[l] = dZb.T @ acts[l]
        gb[l] = dZf.sum(dim=0)
        if l == 0:
            break
        dH = dZb @ Wr[l]
        dZf = dH * dgelu(zs[l - 1])
        dZb = _r(dZf, round_bf16)
    return out, loss, gW, gb
