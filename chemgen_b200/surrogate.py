"""Learned surrogate of getrates with per-point fallback to the exact kernel.

Network: inputs (1000/T, ln T, ln P and the ln mole fraction of each of the
ns species, centred and scaled) padded to `din`, each held as a BF16 pair
(hi + lo) that the first layer multiplies by the same weights; three hidden
layers of width 256 with GELU; `dout` outputs: the direction
u_k = w_k / |w|_2 of the rate vector (columns 0..ns-1), its centred log
length (ln |w|_2 - c) / s (column ns) and an estimate of log10 of the
network's own normwise error at that point (column ns + 1).  Because the
normwise error of a decoded prediction is, to first order,
max_k |du_k| / max_k |u_k| + |d ln |w|_2|, the regression loss weighs the
outputs the way the error gate measures them.  BF16 weights (FP32 master
copies) and FP32 accumulation.

Training runs entirely on this package's CUDA kernels (chemgen_mlp_* in
libchemgen_b200.so): the forward products, the input and weight gradients,
GELU and its derivative, the loss gradient, bias sums and Adam; one training
step is captured as a CUDA graph and replayed.  The training data are
(P, T, Y) -> wdot samples produced by the exact kernel.

Inference (`SurrogateGetrates`): the network predicts wdot and its error
estimate; a point falls back to the exact kernel when its inputs leave the
training ranges or the estimate exceeds the tolerance.  The exact kernel is
also the reference used to report the surrogate's accuracy.

The reference has no surrogate; its chemgen/chemistry_nn.py:15-85 torch
prototype (log-space Arrhenius layers) never ran.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass
from typing import Dict, List

from .runtime import GpuMechanism, check, lib

HIDDEN = 256
DIN = 64
DOUT = 64


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


@dataclass
class TrainConfig:
    samples: int = 10_000_000
    batch: int = 1024
    epochs: int = 16
    lr: float = 1e-3
    lr_final: float = 5e-5
    weight_decay: float = 0.0
    error_head_epochs: int = 1
    # the error head's target: 0 -> the mean of log10 normwise error (least
    # squares); q in (0, 1) -> its q-quantile (pinball loss), a conservative
    # estimate for the gate
    error_quantile: float = 0.0
    seed: int = 0


# epilogues of chemgen_mlp_gemm_tc
EPI_STORE, EPI_STORE_T, EPI_BIAS_GELU, EPI_BIAS, EPI_GELU_BACK = 0, 1, 2, 3, 4


def _p(t) -> int:
    if t is None:
        return 0
    return t if isinstance(t, int) else t.data_ptr()


def _gemm_tc(A, lda, B, ldb, M, N, K, epi, bias=None, zprev=None, ldz=0, C=None, ldc=0, H=None, ldh=0, HT=None,
             ldt=0, accumulate=0):
    check(lib().chemgen_mlp_gemm_tc(_p(A), lda, _p(B), ldb, M, N, K, epi, _p(bias), _p(zprev), ldz, _p(C), ldc, _p(H),
                                    ldh, _p(HT), ldt, accumulate, _stream()), "mlp_gemm_tc")


def _transpose(src, rows, cols, dst, lds=None, ldd=None):
    check(lib().chemgen_mlp_transpose_bf16(_p(src), cols if lds is None else lds, rows, cols, _p(dst),
                                           rows if ldd is None else ldd, _stream()), "mlp_transpose_bf16")


class MLP:
    """The network's parameters and the kernel calls of one forward/backward.

    With `tc` (the default) the products run on the tensor cores through
    chemgen_mlp_gemm_tc, each fused with its epilogue: bias + GELU in the
    forward, GELU' in the input gradients; the weight gradients take the
    transposed activations (written by the forward's epilogues) as K-major
    operands.  A batch that is not a multiple of 128 rows, or tc=False, runs
    on the warp-level chemgen_mlp_gemm with the separate elementwise kernels."""

    def __init__(self, din: int = DIN, hidden: int = HIDDEN, dout: int = DOUT, seed: int = 0, device: int = 0,
                 tc: bool = True):
        import torch
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.dims = [din, hidden, hidden, hidden, dout]
        self.tc = tc
        self.dev = torch.device("cuda", device)
        self.W: List = []       # FP32 master [N x K]
        self.Wb: List = []      # BF16 copy
        self.b: List = []
        for l in range(4):
            k, n = self.dims[l], self.dims[l + 1]
            w = torch.randn(n, k, generator=g) * math.sqrt(2.0 / k)
            self.W.append(w.to(self.dev).contiguous())
            self.Wb.append(self.W[-1].to(torch.bfloat16).contiguous())
            self.b.append(torch.zeros(n, device=self.dev))
        self.params = self.W + self.b
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self._ws: Dict = {}
        # operands of the tensor-core products: the first layer's weights twice
        # side by side (its input is a hi + lo pair of BF16 parts), and the
        # transposed weights [k x n] of the input-gradient products
        self.Wd0 = torch.empty(hidden, 2 * din, dtype=torch.bfloat16, device=self.dev)
        self.WT = [torch.empty(self.dims[l], self.dims[l + 1], dtype=torch.bfloat16, device=self.dev)
                   for l in range(4)]
        self.refresh_operands()

    def refresh_operands(self):
        """Rebuild Wd0 and the transposed weights from the BF16 weights (at
        construction and after weights are loaded or changed outside the
        training step, whose Adam launch writes them itself)."""
        for l in range(4):
            k, n = self.dims[l], self.dims[l + 1]
            _transpose(self.Wb[l], n, k, self.WT[l])
        din, hid = self.dims[0], self.dims[1]
        _transpose(self.WT[0], din, hid, self.Wd0, ldd=2 * din)
        _transpose(self.WT[0], din, hid, self.Wd0.data_ptr() + 2 * din, ldd=2 * din)

    def _side_stream(self):
        import torch
        if getattr(self, "_side", None) is None:
            self._side = torch.cuda.Stream(device=self.dev)
        return self._side

    def _use_tc(self, B: int) -> bool:
        return self.tc and B % 128 == 0

    def _buf(self, key, shape, dtype):
        import torch
        t = self._ws.get(key)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=self.dev)
            self._ws[key] = t
        return t

    def _input_parts(self, X):
        """(pointer, row stride) of each BF16 part of the input: one part for
        X [B, din], two (hi, lo) for X [B, 2 din], whose sum is the input."""
        din = self.dims[0]
        if X.shape[1] == din:
            return [(X.data_ptr(), din)]
        if X.shape[1] == 2 * din:
            return [(X.data_ptr(), 2 * din), (X.data_ptr() + 2 * din, 2 * din)]
        raise ValueError(f"input width {X.shape[1]} is neither {din} nor {2 * din}")

    def _forward_tc(self, X, keep: bool):
        import torch
        B = X.shape[0]
        din, hid, dout = self.dims[0], self.dims[1], self.dims[4]
        if X.shape[1] == 2 * din:
            W0, K0 = self.Wd0, 2 * din
        elif X.shape[1] == din:
            W0, K0 = self.Wb[0], din
        else:
            raise ValueError(f"input width {X.shape[1]} is neither {din} nor {2 * din}")
        self.acts, self.zs, self.actsT = [X], [], []
        if keep:
            # training: one fused kernel for the four layers; Z_l (FP32) and
            # H_l (BF16) leave transposed, [feature][row], for the backward
            ZT = [self._buf(("ZT", l), (hid, B), torch.float32) for l in range(3)]
            HT = [self._buf(("HT", l), (hid, B), torch.bfloat16) for l in range(3)]
            out = self._buf(("Z", 3, keep), (B, dout), torch.float32)
            P = ctypes.c_void_p
            Ws = (P * 4)(W0.data_ptr(), *[self.Wb[l].data_ptr() for l in (1, 2, 3)])
            bs = (P * 4)(*[self.b[l].data_ptr() for l in range(4)])
            check(lib().chemgen_mlp_forward_tc(X.data_ptr(), X.shape[1], K0, Ws, bs, B,
                                               (P * 3)(*[z.data_ptr() for z in ZT]),
                                               (P * 3)(*[h.data_ptr() for h in HT]), out.data_ptr(), _stream()),
                  "mlp_forward_tc")
            self.zs, self.actsT = ZT, HT
            self.zs_transposed = True
            return out
        self.zs_transposed = False
        A, lda, Bw, K = X, X.shape[1], W0, K0
        for l in range(3):
            Z = self._buf(("Z", l, keep), (B, hid), torch.float32) if keep else None
            H = self._buf(("H", l, keep), (B, hid), torch.bfloat16)
            HT = self._buf(("HT", l), (hid, B), torch.bfloat16) if keep else None
            _gemm_tc(A, lda, Bw, K, B, hid, K, EPI_BIAS_GELU, bias=self.b[l], C=Z, ldc=hid, H=H, ldh=hid, HT=HT,
                     ldt=B)
            self.zs.append(Z)
            self.acts.append(H)
            self.actsT.append(HT)
            A, lda, Bw, K = H, hid, self.Wb[l + 1], hid
        out = self._buf(("Z", 3, keep), (B, dout), torch.float32)
        _gemm_tc(A, lda, Bw, K, B, dout, K, EPI_BIAS, bias=self.b[3], C=out, ldc=dout)
        self.zs.append(out)
        return out

    def _backward_tc(self, dout_b, dout_f):
        """One fused kernel takes the input gradients dZ_2, dZ_1, dZ_0 down the
        network (with the bias gradients and the transposed operands); the
        weight-gradient products then run on two streams side by side (each
        fills only 8-32 of the SMs), while a side stream has transposed the
        input and summed the output gradient meanwhile.  The current stream
        joins the side stream at the end (CUDA-graph capture keeps the fork
        and join)."""
        import torch
        B = dout_b.shape[0]
        main = torch.cuda.current_stream()
        side = self._side_stream()
        din, hid, dout = self.dims[0], self.dims[1], self.dims[4]
        gW = [self._buf(("gW", l), (self.dims[l + 1], self.dims[l]), torch.float32) for l in range(4)]
        gb = [self._buf(("gb", l), (self.dims[l + 1],), torch.float32) for l in range(4)]
        doutT = self._buf(("doutT",), (dout, B), torch.bfloat16)
        dZT = [self._buf(("dZT", l), (hid, B), torch.bfloat16) for l in range(3)]
        X = self.acts[0]
        w = X.shape[1]
        XT = self._buf(("XT",), (w, B), torch.bfloat16)

        def fork():
            ev = torch.cuda.Event()
            ev.record(main)
            side.wait_event(ev)

        fork()
        with torch.cuda.stream(side):
            check(lib().chemgen_mlp_colsum(dout_f.data_ptr(), gb[3].data_ptr(), B, dout, _stream()), "mlp_colsum")
            _transpose(X, B, w, XT)
        P = ctypes.c_void_p
        nwork = -(-int(lib().chemgen_mlp_backward_tc_work_bytes(B)) // 4)
        work = self._ws.get(("bwork", B))
        if work is None:
            work = self._ws[("bwork", B)] = torch.zeros(nwork, dtype=torch.float32, device=self.dev)
        check(lib().chemgen_mlp_backward_tc(dout_b.data_ptr(), (P * 4)(None, *[self.WT[l].data_ptr() for l in (1, 2, 3)]),
                                            (P * 3)(*[z.data_ptr() for z in self.zs]), B,
                                            (P * 3)(*[d.data_ptr() for d in dZT]),
                                            (P * 3)(*[g.data_ptr() for g in gb[:3]]), doutT.data_ptr(),
                                            work.data_ptr(), _stream()),
              "mlp_backward_tc")
        fork()
        with torch.cuda.stream(side):
            # dW3[n][k] = sum_m dout[m][n] H2[m][k], as (H2^T)(dout^T)^T stored transposed
            _gemm_tc(self.actsT[2], B, doutT, B, hid, dout, B, EPI_STORE_T, C=gW[3], ldc=hid)
            # layer 0: the input's transposed parts (hi, lo, transposed above on
            # this stream) as operands, summed
            for j in range(w // din):
                _gemm_tc(dZT[0], B, XT.data_ptr() + 2 * j * din * B, B, hid, din, B, EPI_STORE, C=gW[0],
                         ldc=din, accumulate=1 if j else 0)
        # dW_l[n][k] = sum_m dZ_l[m][n] H_{l-1}[m][k]
        _gemm_tc(dZT[2], B, self.actsT[1], B, hid, hid, B, EPI_STORE, C=gW[2], ldc=hid)
        _gemm_tc(dZT[1], B, self.actsT[0], B, hid, hid, B, EPI_STORE, C=gW[1], ldc=hid)
        main.wait_stream(side)
        return gW + gb

    def forward(self, X, keep: bool = True):
        """X: BF16 [B, din], or [B, 2 din] holding hi and lo parts.  Returns
        the FP32 output [B, dout]; keeps Z_l and H_l for the backward when
        `keep`."""
        import torch
        B = X.shape[0]
        self._tc_last = self._use_tc(B)
        if self._tc_last:
            return self._forward_tc(X, keep)
        s = _stream()
        H = X
        self.acts = [X]
        self.zs = []
        for l in range(4):
            k, n = self.dims[l], self.dims[l + 1]
            Z = self._buf(("Z", l, keep), (B, n), torch.float32)
            parts = self._input_parts(X) if l == 0 else [(H.data_ptr(), k)]
            for j, (ptr, ld) in enumerate(parts):
                check(lib().chemgen_mlp_gemm(ptr, ld, 1, self.Wb[l].data_ptr(), k, 1, Z.data_ptr(), n, B, n, k,
                                             1 if j else 0, s), "mlp_gemm")
            Hn = self._buf(("H", l, keep), (B, n), torch.bfloat16) if l < 3 else None
            check(lib().chemgen_mlp_bias_gelu(Z.data_ptr(), self.b[l].data_ptr(), 0 if Hn is None else Hn.data_ptr(),
                                              B, n, 1 if l < 3 else 0, s), "mlp_bias_gelu")
            self.zs.append(Z)
            if Hn is not None:
                self.acts.append(Hn)
                H = Hn
        return self.zs[-1]

    def backward(self, dout_b, dout_f):
        """dout: gradient of the loss wrt the output (BF16 and FP32 [B, dout]).
        Returns the parameter gradients (same order as self.params)."""
        import torch
        B = dout_b.shape[0]
        if getattr(self, "_tc_last", False):
            return self._backward_tc(dout_b, dout_f)
        s = _stream()
        gW = [None] * 4
        gb = [None] * 4
        dZb, dZf = dout_b, dout_f
        for l in range(3, -1, -1):
            k, n = self.dims[l], self.dims[l + 1]
            H = self.acts[l]
            gw = self._buf(("gW", l), (n, k), torch.float32)
            # gW[n][k] = sum_m dZ[m][n] H[m][k]
            parts = self._input_parts(H) if l == 0 else [(H.data_ptr(), k)]
            for j, (ptr, ld) in enumerate(parts):
                check(lib().chemgen_mlp_gemm(dZb.data_ptr(), 1, n, ptr, 1, ld, gw.data_ptr(), k, n, k, B, 1 if j else 0,
                                             s), "mlp_gemm dW")
            g_b = self._buf(("gb", l), (n,), torch.float32)
            check(lib().chemgen_mlp_colsum(dZf.data_ptr(), g_b.data_ptr(), B, n, s), "mlp_colsum")
            gW[l], gb[l] = gw, g_b
            if l == 0:
                break
            # dH[m][k] = sum_n dZ[m][n] W[n][k]
            dH = self._buf(("dH", l), (B, k), torch.float32)
            check(lib().chemgen_mlp_gemm(dZb.data_ptr(), n, 1, self.Wb[l].data_ptr(), 1, k, dH.data_ptr(), k, B, k, n,
                                         0, s), "mlp_gemm dH")
            nb = self._buf(("dZb", l - 1), (B, k), torch.bfloat16)
            nf = self._buf(("dZf", l - 1), (B, k), torch.float32)
            check(lib().chemgen_mlp_gelu_backward(dH.data_ptr(), self.zs[l - 1].data_ptr(), nb.data_ptr(),
                                                  nf.data_ptr(), B * k, s), "mlp_gelu_backward")
            dZb, dZf = nb, nf
        return gW + gb

    def _adam_tables(self, grads, wd: float):
        """Host pointer tables of chemgen_mlp_adam_multi for these gradient
        buffers (cached: the buffers do not move between steps)."""
        import ctypes
        key = (tuple(g.data_ptr() for g in grads), wd)
        if getattr(self, "_adam_key", None) != key:
            n = len(self.params)
            P = ctypes.c_void_p * n
            rows = [p.shape[0] for p in self.params]
            cols = [p.shape[1] if p.dim() == 2 else 1 for p in self.params]
            self._adam_tab = (
                P(*[p.data_ptr() for p in self.params]), P(*[g.data_ptr() for g in grads]),
                P(*[m.data_ptr() for m in self.m]), P(*[v.data_ptr() for v in self.v]),
                P(*[self.Wb[j].data_ptr() if j < 4 else None for j in range(n)]),
                P(*[self.WT[j].data_ptr() if j < 4 else None for j in range(n)]),
                P(*[self.Wd0.data_ptr() if j == 0 else None for j in range(n)]),
                (ctypes.c_int * n)(*rows), (ctypes.c_int * n)(*cols),
                (ctypes.c_float * n)(*[wd if j < 4 else 0.0 for j in range(n)]))
            self._adam_key = key
        return self._adam_tab

    def adam(self, grads, hyper, wd: float = 0.0, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        """One Adam step; `hyper` is a device FP32 tensor {lr, 1/(1-b1^t), 1/(1-b2^t)}.
        With the tensor-core products, one launch updates every tensor and
        writes the BF16, transposed and doubled operands."""
        s = _stream()
        if self.tc:
            t = self._adam_tables(grads, wd)
            check(lib().chemgen_mlp_adam_multi(len(self.params), *t, hyper.data_ptr(), b1, b2, eps, s),
                  "mlp_adam_multi")
            return
        for j, (p, g) in enumerate(zip(self.params, grads)):
            wb = self.Wb[j].data_ptr() if j < 4 else 0
            check(lib().chemgen_mlp_adam(p.data_ptr(), g.data_ptr(), self.m[j].data_ptr(), self.v[j].data_ptr(), wb,
                                         p.numel(), hyper.data_ptr(), b1, b2, eps, wd if j < 4 else 0.0, s),
                  "mlp_adam")


def adam_schedule(total: int, lr: float, lr_final: float, b1: float = 0.9, b2: float = 0.999, device=None):
    """[total, 3] FP32 rows {lr_t, 1/(1-b1^t), 1/(1-b2^t)} for t = 1..total,
    lr_t on a cosine from lr to lr_final."""
    import torch
    t = torch.arange(1, total + 1, dtype=torch.float64)
    frac = (t - 1) / max(total - 1, 1)
    lrs = lr_final + 0.5 * (lr - lr_final) * (1.0 + torch.cos(math.pi * frac))
    return torch.stack([lrs, 1.0 / (1.0 - b1 ** t), 1.0 / (1.0 - b2 ** t)], dim=1).float().to(device)


class Surrogate:
    """MLP surrogate for one mechanism, trained from the exact kernel."""

    def __init__(self, gm: GpuMechanism, seed: int = 0, device: int = 0):
        import torch
        if gm.ns + 2 > DOUT or gm.ns + 3 > DIN:
            raise ValueError(f"the surrogate supports up to {DOUT - 2} species")
        if gm.mech is None:
            raise ValueError("the surrogate needs the mechanism's molecular weights (construct GpuMechanism from a "
                             "Mechanism)")
        self.gm = gm
        self.ns = gm.ns
        self.net = MLP(seed=seed, device=device)
        self.dev = self.net.dev
        self.inv_mw = 1.0 / torch.tensor(gm.mech.mw(), dtype=torch.float64, device=self.dev)
        # centring and scaling of 1000/T, ln T and ln(P/1 atm) over the
        # training ranges (T 300..2500 K, P 1..40 atm); those of ln X_k are
        # set from the training data in fit()
        self.norm = torch.tensor([1.3, 1.0 / 0.9, 6.9, 1.0 / 0.55, math.log(40.0) / 2,
                                  1.0 / (math.log(40.0) / math.sqrt(12.0)), 0.0, 1.0], device=self.dev)
        self.lnorm = torch.tensor([0.0, 1.0], device=self.dev)
        self.colw = torch.zeros(DOUT, device=self.dev)
        self.T_range = (300.0, 2500.0)
        self.P_range = (1013250.0, 1013250.0 * 40.0)
        self.history: List[float] = []
        self._img = None

    # ------------------------------------------------------------ transforms
    def features(self, P, T, Y):
        """BF16 [ng, 2 din]: the hi and lo parts of the network inputs."""
        import torch
        ng = T.numel()
        X = torch.empty((ng, 2 * DIN), dtype=torch.bfloat16, device=self.dev)
        check(lib().chemgen_surrogate_features(P.data_ptr(), T.data_ptr(), Y.data_ptr(), ng, self.ns, DIN,
                                               self.norm.data_ptr(), self.inv_mw.data_ptr(), X.data_ptr(), 0,
                                               _stream()), "features")
        return X

    def targets(self, W):
        import torch
        ng = W.shape[1]
        Tg = torch.empty((ng, DOUT), dtype=torch.float32, device=self.dev)
        check(lib().chemgen_surrogate_targets(W.data_ptr(), ng, self.ns, DOUT, self.lnorm.data_ptr(), Tg.data_ptr(),
                                              _stream()), "targets")
        return Tg

    def decode(self, out):
        import torch
        ng = out.shape[0]
        W = torch.empty((self.ns, ng), dtype=torch.float64, device=self.dev)
        est = torch.empty(ng, dtype=torch.float32, device=self.dev)
        check(lib().chemgen_surrogate_decode(out.data_ptr(), ng, self.ns, DOUT, self.lnorm.data_ptr(), W.data_ptr(),
                                             est.data_ptr(), _stream()), "decode")
        return W, est

    def _set_species_norm(self, Y):
        """Centre and spread of ln X_k over a sample of states."""
        import torch
        n = Y.clamp_min(1e-30) * self.inv_mw[:, None]
        lx = torch.log(n) - torch.log(n.sum(dim=0, keepdim=True))
        self.norm[6] = float(lx.mean())
        self.norm[7] = 1.0 / float(lx.std())

    # --------------------------------------------------------------- data
    def sample_states(self, n: int, gen):
        """States with the workload's distributions (T ~ U(300, 2500) K, P
        log-uniform over 1..40 atm, Y ~ Dirichlet(0.5)), drawn on the GPU."""
        import torch
        T = torch.rand(n, generator=gen, device=self.dev, dtype=torch.float64) * 2200.0 + 300.0
        P = 1013250.0 * torch.exp(torch.rand(n, generator=gen, device=self.dev, dtype=torch.float64) * math.log(40.0))
        G = torch._standard_gamma(torch.full((self.ns, n), 0.5, device=self.dev, dtype=torch.float64), generator=gen)
        Y = (G / G.sum(dim=0, keepdim=True)).contiguous()
        return P.contiguous(), T.contiguous(), Y

    def make_dataset(self, n: int, seed: int, chunk: int = 1 << 20, mode: str = "fp64"):
        """(features BF16 [n, 2 din] chunks, wdot FP64 [ns, n] chunks) from the exact kernel."""
        import torch
        gen = torch.Generator(device=self.dev).manual_seed(seed)
        Xs, Ws = [], []
        for i0 in range(0, n, chunk):
            m = min(chunk, n - i0)
            P, T, Y = self.sample_states(m, gen)
            if i0 == 0:
                self._set_species_norm(Y)
            W = self.gm.getrates(P, T, Y, mode=mode)
            Xs.append(self.features(P, T, Y))
            Ws.append(W)
        return Xs, Ws

    # ------------------------------------------------------------- training
    def fit(self, cfg: TrainConfig = TrainConfig(), log=None, graph: bool = True) -> Dict:
        """Train on cfg.samples exact-kernel samples.  The training step (batch
        gather, forward, loss gradient, backward, Adam) is captured as a CUDA
        graph of eight consecutive steps and replayed; per replay only the
        eight steps' batch indices and schedule rows are copied in."""
        import torch
        t0 = time.perf_counter()
        Xs, Ws = self.make_dataset(cfg.samples, cfg.seed)
        # centre and spread of ln |w|_2 over the first chunk; the log-length
        # column is weighted by spread^2 so that its loss is in units of ln |w|_2
        ln_n = torch.log(Ws[0].norm(dim=0).clamp_min(1e-300))
        self.lnorm[0] = float(ln_n.mean())
        self.lnorm[1] = float(ln_n.std().clamp_min(1e-3))
        self.colw.zero_()
        self.colw[: self.ns] = 1.0
        self.colw[self.ns] = float(self.lnorm[1]) ** 2
        X = torch.cat(Xs)
        Tg = torch.cat([self.targets(W) for W in Ws])
        del Xs, Ws
        n = X.shape[0]
        torch.cuda.synchronize(self.dev)
        t_data = time.perf_counter() - t0
        B = cfg.batch
        steps_per_epoch = n // B
        total = steps_per_epoch * cfg.epochs
        sched = adam_schedule(total, cfg.lr, cfg.lr_final, device=self.dev)
        # one CUDA graph holds `chunk` consecutive training steps, each with its
        # own row of batch indices and of the schedule; per replay the host
        # copies in `chunk` rows of each, so its per-step cost stays small
        chunk = 8 if graph else 1
        hyper = torch.empty((chunk, 3), device=self.dev)
        idx = torch.zeros((chunk, B), dtype=torch.int64, device=self.dev)
        xb = torch.empty((B, X.shape[1]), dtype=X.dtype, device=self.dev)
        tb = torch.empty((B, DOUT), dtype=torch.float32, device=self.dev)
        loss = torch.zeros(1, device=self.dev)
        dout_b = torch.empty((B, DOUT), dtype=torch.bfloat16, device=self.dev)
        dout_f = torch.empty((B, DOUT), dtype=torch.float32, device=self.dev)
        gen = torch.Generator(device=self.dev).manual_seed(cfg.seed + 1)

        def body(k):
            torch.index_select(X, 0, idx[k], out=xb)
            torch.index_select(Tg, 0, idx[k], out=tb)
            out = self.net.forward(xb)
            check(lib().chemgen_mlp_mse_grad(out.data_ptr(), tb.data_ptr(), self.colw.data_ptr(), dout_b.data_ptr(),
                                             dout_f.data_ptr(), loss.data_ptr(), B, DOUT, _stream()), "mse_grad")
            grads = self.net.backward(dout_b, dout_f)
            self.net.adam(grads, hyper[k], cfg.weight_decay)

        g = None
        step = 0
        t1 = time.perf_counter()
        for ep in range(cfg.epochs):
            perm = torch.randperm(n, device=self.dev, generator=gen)
            loss.zero_()
            b = 0
            while b < steps_per_epoch:
                if g is not None and b + chunk <= steps_per_epoch:
                    idx.copy_(perm[b * B:(b + chunk) * B].view(chunk, B))
                    hyper.copy_(sched[step:step + chunk])
                    g.replay()
                    step += chunk
                    b += chunk
                    continue
                # single eager steps: the first few (every buffer comes to
                # exist) and an epoch's last steps short of a whole replay
                idx[0].copy_(perm[b * B:(b + 1) * B])
                hyper[0].copy_(sched[step])
                body(0)
                step += 1
                b += 1
                if graph and g is None and step == 3:
                    torch.cuda.synchronize(self.dev)
                    side = torch.cuda.Stream(device=self.dev)
                    side.wait_stream(torch.cuda.current_stream())
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.stream(side):
                        with torch.cuda.graph(g, stream=side):
                            for k in range(chunk):
                                body(k)
                    torch.cuda.current_stream().wait_stream(side)
            self.history.append(loss.item() / max(steps_per_epoch, 1))
            if log:
                log(f"epoch {ep}: loss {self.history[-1]:.4e}")
        torch.cuda.synchronize(self.dev)
        t_train = time.perf_counter() - t1
        del g
        # error head: regress log10 of the per-point normwise error of the
        # decoded prediction, on the same data, with the same kernels
        t2 = time.perf_counter()
        self.fit_error_head(X, Tg, cfg, gen, log)
        torch.cuda.synchronize(self.dev)
        t_head = time.perf_counter() - t2
        self._img = None
        return {"samples": n, "t_data_s": t_data, "t_train_s": t_train, "t_error_head_s": t_head,
                "steps": step, "final_loss": self.history[-1] if self.history else None}

    def _normwise_error(self, out, tgt):
        """log10 of max_k |w_hat - w| / max_k |w| per row, from network-space
        tensors (both vectors divided by the true |w|_2)."""
        import torch
        ns = self.ns
        r = torch.exp(((out[:, ns] - tgt[:, ns]) * self.lnorm[1]).clamp(-30.0, 30.0))
        e = (out[:, :ns] * r[:, None] - tgt[:, :ns]).abs().max(dim=1).values
        e = e / tgt[:, :ns].abs().max(dim=1).values.clamp_min(1e-30)
        return torch.log10(e.clamp_min(1e-12))

    def fit_error_head(self, X, Tg, cfg: TrainConfig, gen, log=None):
        import torch
        n = X.shape[0]
        colw = torch.zeros(DOUT, device=self.dev)
        colw[self.ns + 1] = 1.0
        loss = torch.zeros(1, device=self.dev)
        dout_b = torch.empty((cfg.batch, DOUT), dtype=torch.bfloat16, device=self.dev)
        dout_f = torch.empty((cfg.batch, DOUT), dtype=torch.float32, device=self.dev)
        s = _stream()
        per_epoch = max(n // cfg.batch, 1)
        steps = per_epoch * cfg.error_head_epochs
        perm = torch.randperm(n, device=self.dev, generator=gen)
        hm = [torch.zeros_like(self.net.W[3]), torch.zeros_like(self.net.b[3])]
        hv = [torch.zeros_like(self.net.W[3]), torch.zeros_like(self.net.b[3])]
        keep = torch.zeros(DOUT, device=self.dev)
        keep[self.ns + 1] = 1.0
        sched = adam_schedule(max(steps, 1), 1e-3, 1e-3, device=self.dev)
        for b in range(steps):
            j = b % per_epoch
            idx = perm[j * cfg.batch:(j + 1) * cfg.batch]
            xb = X.index_select(0, idx)
            tb = Tg.index_select(0, idx)
            out = self.net.forward(xb)
            tb[:, self.ns + 1] = self._normwise_error(out, tb)
            if cfg.error_quantile > 0.0:
                # pinball loss: slope -q above the estimate, 1 - q below it
                y, o = tb[:, self.ns + 1], out[:, self.ns + 1].float()
                g = torch.where(y > o, -cfg.error_quantile, 1.0 - cfg.error_quantile) / xb.shape[0]
                dout_f.zero_()
                dout_f[: xb.shape[0], self.ns + 1] = g
                dout_b.copy_(dout_f)
                loss += (torch.maximum(cfg.error_quantile * (y - o), (cfg.error_quantile - 1.0) * (y - o))).mean()
            else:
                check(lib().chemgen_mlp_mse_grad(out.data_ptr(), tb.data_ptr(), colw.data_ptr(), dout_b.data_ptr(),
                                                 dout_f.data_ptr(), loss.data_ptr(), xb.shape[0], DOUT, s),
                      "mse_grad")
            grads = self.net.backward(dout_b[: xb.shape[0]], dout_f[: xb.shape[0]])
            # only the error-estimate output (row ns + 1 of the last layer and
            # its bias) moves, with its own Adam state
            gW4, gb4 = grads[3], grads[7]
            gW4.mul_(keep[:, None])
            gb4.mul_(keep)
            hyper = sched[b]
            for p, g, m, v, wb in ((self.net.W[3], gW4, hm[0], hv[0], self.net.Wb[3]),
                                   (self.net.b[3], gb4, hm[1], hv[1], None)):
                check(lib().chemgen_mlp_adam(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(),
                                             0 if wb is None else wb.data_ptr(), p.numel(), hyper.data_ptr(), 0.9,
                                             0.999, 1e-8, 0.0, s), "mlp_adam")
        self.net.refresh_operands()
        if log:
            log(f"error head: loss {loss.item() / max(steps, 1):.4e}")

    # ------------------------------------------------------------ checkpoint
    def _mech_hash(self) -> str:
        import hashlib
        return hashlib.sha256(bytes(self.gm.blob)).hexdigest()

    def state_dict(self) -> Dict:
        """Weights (FP32 masters), biases and the input/output normalisation."""
        return {"W": [w.cpu() for w in self.net.W], "b": [b.cpu() for b in self.net.b], "norm": self.norm.cpu(),
                "lnorm": self.lnorm.cpu(), "ns": self.ns, "mechanism_sha256": self._mech_hash()}

    def load_state_dict(self, st: Dict) -> None:
        import torch
        if st["ns"] != self.ns or st.get("mechanism_sha256") != self._mech_hash():
            raise ValueError("the checkpoint was trained on a different mechanism")
        for l in range(4):
            self.net.W[l].copy_(st["W"][l].to(self.dev))
            self.net.Wb[l].copy_(self.net.W[l].to(torch.bfloat16))
            self.net.b[l].copy_(st["b"][l].to(self.dev))
        self.net.refresh_operands()
        self.norm.copy_(st["norm"].to(self.dev))
        self.lnorm.copy_(st["lnorm"].to(self.dev))
        self._img = None

    def save(self, path: str) -> None:
        import torch
        torch.save(self.state_dict(), path)

    def load(self, path: str) -> None:
        import torch
        self.load_state_dict(torch.load(path, map_location="cpu"))

    # ------------------------------------------------------------- inference
    def packed(self):
        """(weight image, biases) of the fused inference kernel, built from
        the current BF16 weights."""
        import torch
        if self._img is None:
            img = torch.empty(lib().chemgen_surrogate_image_elems(), dtype=torch.bfloat16, device=self.dev)
            Wb = self.net.Wb
            check(lib().chemgen_surrogate_pack(Wb[0].data_ptr(), Wb[1].data_ptr(), Wb[2].data_ptr(), Wb[3].data_ptr(),
                                               img.data_ptr(), _stream()), "surrogate_pack")
            self._img = (img, torch.cat(self.net.b).contiguous())
        return self._img

    def range_bounds(self):
        """Device copy of the training support {T_lo, T_hi, P_lo, P_hi} (P
        widened by 0.1 %) that the fused kernel checks."""
        import torch
        key = (self.T_range, self.P_range)
        if getattr(self, "_range_key", None) != key:
            self._range_dev = torch.tensor([self.T_range[0], self.T_range[1], self.P_range[0] * 0.999,
                                            self.P_range[1] * 1.001], dtype=torch.float64, device=self.dev)
            self._range_key = key
        return self._range_dev

    def predict_fused(self, P, T, Y, out=None, est=None, check_range: bool = False):
        """(wdot [ns, ng] FP64, log10 error estimate [ng]) from the fused
        tensor-core kernel (one launch); with `check_range` the kernel sets
        the estimate of points outside the training support to +inf."""
        import torch
        ng = T.numel()
        img, bias = self.packed()
        W = out if out is not None else torch.empty((self.ns, ng), dtype=torch.float64, device=self.dev)
        e = est if est is not None else torch.empty(ng, dtype=torch.float32, device=self.dev)
        rng = self.range_bounds().data_ptr() if check_range else None
        check(lib().chemgen_surrogate_infer(img.data_ptr(), bias.data_ptr(), self.norm.data_ptr(),
                                            self.lnorm.data_ptr(), self.inv_mw.data_ptr(), self.ns, P.data_ptr(),
                                            T.data_ptr(), ng, Y.data_ptr(), W.data_ptr(), e.data_ptr(), rng,
                                            _stream()),
              "surrogate_infer")
        return W, e

    def predict(self, P, T, Y, chunk: int = 1 << 20, fused: bool = True, check_range: bool = False):
        """(wdot [ns, ng] FP64, log10 error estimate [ng]); `fused` selects
        the one-kernel tensor-core path, otherwise the layer-by-layer kernels
        used in training.  With `check_range`, points outside the training
        support (`in_range`) get an error estimate of +inf."""
        import torch
        if fused:
            return self.predict_fused(P.contiguous(), T.contiguous(), Y.contiguous(), check_range=check_range)
        ng = T.numel()
        W = torch.empty((self.ns, ng), dtype=torch.float64, device=self.dev)
        est = torch.empty(ng, dtype=torch.float32, device=self.dev)
        for i0 in range(0, ng, chunk):
            i1 = min(ng, i0 + chunk)
            X = self.features(P[i0:i1].contiguous(), T[i0:i1].contiguous(), Y[:, i0:i1].contiguous())
            out = self.net.forward(X, keep=False)
            w, e = self.decode(out)
            W[:, i0:i1] = w
            est[i0:i1] = e
        if check_range:
            est.masked_fill_(~self.in_range(P, T, Y), math.inf)
        return W, est

    def in_range(self, P, T, Y):
        """Points inside the training distribution's support."""
        ok = (T >= self.T_range[0]) & (T <= self.T_range[1]) & (P >= self.P_range[0] * 0.999) & \
             (P <= self.P_range[1] * 1.001)
        ok &= (Y >= 0).all(dim=0) & ((Y.sum(dim=0) - 1.0).abs() < 1e-6)
        return ok


class SurrogateGetrates:
    """wdot from the surrogate where it is trusted, from the exact kernel elsewhere.

    A point is trusted when its log10 error estimate is at most log10(tol) -
    margin.  The estimate is a regression on the network's own features and
    under-estimates some states at the edges of the training distribution;
    a margin of 0.5 (a factor 3.2 on the estimate) trades more fallback for
    a bounded worst case (on B200 at 53/325 with the default training:
    fallback 0.15 % -> 6-29 %, max normwise error after fallback 15 -> ~1).

    On CUDA tensors the gate runs on the device behind the fused inference
    kernel, with no host round trip in between: chemgen_gate_select lists the
    failing points, chemgen_gate_gather packs their states into a batch, the
    exact kernel runs on that batch and chemgen_gate_scatter writes its
    results over the surrogate's.  Two ways to run the batch:

    * exact_mode="fp64" (when the mechanism's handle has the staged FP64
      kernel): the batch holds every point and chemgen_getrates_counted
      computes only the points counted on the device, so nothing waits for
      the host; the fallback rate is read when `last_fallback` is asked for.
      The staged kernel costs ~5x the generated mixed kernel per point, so
      this suits the few-tenths-of-a-percent fallback of a gate at its
      tolerance.  The batch buffers hold 2 ns + 3 values per point (a copy
      of the states and rates of every point, on the device).
    * otherwise (exact_mode="mixed", or no staged kernel): a batch of `cap`
      points on the exact kernel of that mode, and one read of the count at
      the end of the call; if more points failed than the batch holds, all
      failing points go through the host path (`_host_gate`) and the batch
      grows for the next call.  The batch starts at one wave of the exact
      kernel (65536 points) because an exact launch over fewer points takes
      about as long: a point's latency, not the batch size, sets its time."""

    MIN_CAP = 1 << 16

    def __init__(self, sur: Surrogate, tol: float, exact_mode: str = "fp64", margin: float = 0.0,
                 cap: int = 0):
        self.sur = sur
        self.tol = tol
        self.exact_mode = exact_mode
        self.margin = margin
        self._last = 0.0
        self._pending = None          # (buffers, ng) of a call whose count is still on the device
        self._cap = cap
        self._bufs = None
        self._counted = exact_mode == "fp64"   # cleared when the handle has no staged kernel

    @property
    def threshold(self) -> float:
        return math.log10(self.tol) - self.margin

    @classmethod
    def grown_cap(cls, n: int, ng: int) -> int:
        """Batch capacity after a call in which n of ng points failed and
        overflowed the batch: a quarter more than n, in whole multiples of
        MIN_CAP, at most ng."""
        return min(ng, -(-(n + n // 4) // cls.MIN_CAP) * cls.MIN_CAP)

    @property
    def last_fallback(self) -> float:
        """Fraction of the last call's points sent to the exact kernel."""
        if self._pending is not None:
            b, ng = self._pending
            b["done"].synchronize()
            self._last = int(b["count_host"][0]) / ng
            self._pending = None
        return self._last

    def _host_gate(self, P, T, Y, W, est):
        """Host-side gate: every failing point through the exact kernel."""
        import torch
        ok = est <= self.threshold
        bad = torch.nonzero(~ok).flatten()
        if bad.numel():
            Pb, Tb = P.index_select(0, bad).contiguous(), T.index_select(0, bad).contiguous()
            Yb = Y.index_select(1, bad).contiguous()
            W[:, bad] = self.sur.gm.getrates(Pb, Tb, Yb, mode=self.exact_mode)
        return bad.numel()

    def _buffers(self, ng: int, cap: int):
        """Batch buffers of the device gate (cap points) and the estimate
        buffer (ng points); device pointers are kept so that a call does
        little host work between its launches.  On the batch path the unused
        slots always hold a valid state (1 atm, 1000 K, equal mass fractions,
        or a state of an earlier call), so the exact kernel's work on them is
        harmless."""
        import torch
        b = self._bufs
        if b is None or b["cap"] != cap:
            dev, ns = self.sur.dev, self.sur.ns
            f64 = dict(dtype=torch.float64, device=dev)
            b = {"cap": cap,
                 "P": torch.full((cap,), 1013250.0, **f64), "T": torch.full((cap,), 1000.0, **f64),
                 "Y": torch.full((ns, cap), 1.0 / ns, **f64), "W": torch.empty((ns, cap), **f64),
                 "idx": torch.empty(cap, dtype=torch.int64, device=dev),
                 "count": torch.zeros(1, dtype=torch.int64, device=dev),
                 "count_host": torch.zeros(1, dtype=torch.int64, pin_memory=True),
                 "done": torch.cuda.Event(), "est": None}
            for k in ("P", "T", "Y", "W", "idx", "count"):
                b["p_" + k] = b[k].data_ptr()
            self._bufs = b
        if b["est"] is None or b["est"].numel() != ng:
            b["est"] = torch.empty(ng, dtype=torch.float32, device=self.sur.dev)
        return b

    def __call__(self, P, T, Y, out=None):
        """wdot [ns, ng] (FP64, species-major) for P[ng], T[ng], Y[ns, ng];
        written into `out` when given."""
        import torch
        P, T, Y = P.contiguous(), T.contiguous(), Y.contiguous()
        ng = T.numel()
        if not (T.is_cuda and ng):
            # the fused kernel folds the training-support check into the estimate
            W, est = self.sur.predict(P, T, Y, check_range=True)
            self._pending = None
            self._last = self._host_gate(P, T, Y, W, est) / max(ng, 1)
            if out is not None:
                out.copy_(W)
                return out
            return W
        cap = ng if self._counted else min(ng, max(self._cap, self.MIN_CAP))
        if out is not None and not (out.is_cuda and out.dtype == torch.float64 and out.is_contiguous()
                                    and tuple(out.shape) == (self.sur.ns, ng)):
            raise ValueError(f"out must be a contiguous float64 CUDA tensor of shape ({self.sur.ns}, {ng})")
        b = self._buffers(ng, cap)
        est = b["est"]
        W = out if out is not None else torch.empty((self.sur.ns, ng), dtype=torch.float64, device=self.sur.dev)
        self.sur.predict_fused(P, T, Y, W, est, check_range=True)
        ns, s, L = self.sur.ns, _stream(), lib()
        check(L.chemgen_gate_select(est.data_ptr(), self.threshold, ng, b["p_idx"], cap, b["p_count"], s),
              "gate_select")
        check(L.chemgen_gate_gather(P.data_ptr(), T.data_ptr(), Y.data_ptr(), ns, ng, b["p_idx"], b["p_count"], cap,
                                    b["p_P"], b["p_T"], b["p_Y"], s), "gate_gather")
        if self._counted:
            st = L.chemgen_getrates_counted(self.sur.gm._h, b["p_P"], b["p_T"], cap, b["p_Y"], b["p_W"],
                                            b["p_count"], s)
            if st == 6:                             # no staged kernel for this mechanism: batch path
                self._counted = False
                self._bufs = None
                return self(P, T, Y, out=W)
            check(st, "chemgen_getrates_counted")
        else:
            self.sur.gm.getrates_ptr(b["p_P"], b["p_T"], cap, b["p_Y"], b["p_W"], self.exact_mode, s)
        check(L.chemgen_gate_scatter(b["p_W"], ns, cap, b["p_idx"], b["p_count"], W.data_ptr(), ng, s),
              "gate_scatter")
        b["count_host"].copy_(b["count"], non_blocking=True)
        b["done"].record()
        if self._counted:
            # the batch holds every point: nothing can overflow, so the host
            # reads the count only when the fallback rate is asked for
            self._pending = (b, ng)
            return W
        b["done"].synchronize()
        n = int(b["count_host"][0])
        if n > cap:
            # more failing points than the batch holds: all of them through
            # the host path, and a larger batch next time
            self._host_gate(P, T, Y, W, est)
            self._cap = self.grown_cap(n, ng)
        self._pending = None
        self._last = n / ng
        return W
