#!/usr/bin/env python
"""getrates throughput on B200: Mpoints/s of the 53-species / 325-reaction
workload (2^20 points per GPU), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one getrates pass over the GPU's 2^20 points (inputs resident in
HBM; Y alone is 445 MB, larger than the 126 MB L2, so no flush is needed).
`value` is the headline form -- the fastest arithmetic mode whose error
against the FP64 oracle meets 1e-6 (normwise) -- and the FP64 kernel is
reported beside it.  Under torchrun every rank runs its own 2^20 points
(weak scaling, no collective on the data path); times are the max over
ranks.  `--impl reference` times the FP64 CPU restatement of the reference's
generated getrates on all host cores instead.

On one GPU the line also carries `surrogate`: the learned MLP surrogate of
the same mechanism, trained on exact-kernel samples, evaluated on 2^22
points -- its normwise error against the FP64 kernel, the fused tensor-core
inference kernel's points/s, the error gate's fallback rate at
--surrogate-tol and the gain with fallback over the exact kernels.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "getrates Mpoints/s on 1 B200: mixed/surrogate vs FP64 kernel at ≤1e-6 rel err"
WORKLOAD = "synthetic mechanism, 53 species / 325 reactions (28 three-body, 29 Troe, ~70% reversible), 2^20 points per GPU"
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ng", type=int, default=1 << 20)
    ap.add_argument("--modes", default="fp64,mixed,mixed_tc")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--clock-ms", type=float, default=1500.0, help="length of the clock-sampled timed pass")
    ap.add_argument("--e2e-steps", type=int, default=-1, help="host-path steps (default min(steps, 50))")
    ap.add_argument("--table", action="store_true", help="table-driven kernels instead of the generated ones")
    ap.add_argument("--surrogate-samples", type=int, default=10_000_000,
                    help="exact-kernel training samples of the learned surrogate (0 skips the surrogate leg)")
    ap.add_argument("--surrogate-epochs", type=int, default=16)
    ap.add_argument("--surrogate-points", type=int, default=1 << 22)
    ap.add_argument("--surrogate-tol", type=float, default=0.05,
                    help="normwise tolerance of the surrogate's error gate (points above it fall back)")
    ap.add_argument("--head", default="auto", choices=["auto", "fp64", "mixed", "mixed_tc"],
                    help="headline mode; auto = the fastest mode within 1e-6 (under a profiler, whose "
                         "serialised launches distort the timings that choose it, pass it explicitly)")
    ap.add_argument("--configs-only", action="store_true",
                    help="run only the other configurations and print them (for profiling their kernels)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (real GRI30, mini-app states, 348/2163, Jacobian)")
    return ap.parse_args()


# --------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and throttle reasons sampled every ~5 ms through NVML while running."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            idx = device
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            if vis:
                ids = [v.strip() for v in vis.split(",") if v.strip()]
                if device < len(ids) and ids[device].isdigit():
                    idx = int(ids[device])
            self._h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self._nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nv = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for name, bit in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self._nv is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t is not None:
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def _profile_row(fname: str, mode: str, ns: int, nr: int):
    """Numbers after `mode ns nr` on the matching row of a committed ncu summary table."""
    path = os.path.join(REPO, "profiles", fname)
    if not os.path.exists(path):
        return None
    for line in open(path):
        p = line.split()
        if len(p) >= 4 and not line.startswith("#") and p[0] == mode and int(p[1]) == ns and int(p[2]) == nr:
            return [float(x) for x in p[3:]]
    return None


def ncu_traffic(mode: str, ns: int, nr: int):
    """DRAM bytes per point of the getrates kernel from the committed ncu summary."""
    row = _profile_row("getrates_traffic.txt", mode, ns, nr)
    return None if row is None else row[0]


def ncu_issue(mode: str, ns: int, nr: int):
    """Warp instructions issued per point, and the FP64 / FMA (FP32) / XU (MUFU) pipes'
    active fractions, of the generated kernel from the committed ncu summary."""
    row = _profile_row("getrates_issue.txt", mode, ns, nr)
    if row is None or len(row) < 4:
        return None
    return {"warp_inst_per_point": row[0], "pipe_fp64": row[1], "pipe_fma": row[2], "pipe_xu": row[3]}


# ------------------------------------------------------------ reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return
    from chemgen_b200 import pack, synthetic
    from oracle import oracle
    mech = synthetic.gri_shape()
    blob = pack.pack(mech).to_blob()
    cores = os.cpu_count() or 1
    P, T, Y = synthetic.states(mech.ns, 4096, seed=1000)
    t0 = time.perf_counter()
    oracle.getrates(blob, P[:512], T[:512], Y[:, :512].copy(), nthreads=cores)
    pilot = 512 / (time.perf_counter() - t0)
    sample = int(min(args.ng, max(1024, pilot * 2.0)))
    P, T, Y = synthetic.states(mech.ns, sample, seed=1000)
    for _ in range(max(args.warmup, 0)):
        oracle.getrates(blob, P, T, Y, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.getrates(blob, P, T, Y, nthreads=cores)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    value = sample / dt / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mpoints/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "mechanism": mech.name, "points_per_step": sample},
            "cpu_baseline": {"value": value, "unit": "Mpoints/s", "cores": cores, "kind": "port",
                             "sample": f"{sample} points of the workload per step (FP64 C restatement of the "
                                       f"reference's generated getrates, OpenMP over points)"},
            "e2e": {"value": value, "unit": "Mpoints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def link_step_seconds(Ph, Th, Yh, Wh, Pd, Td, Yd, Wd, reps: int = 5) -> float:
    """Seconds for one step's host-link traffic alone: the inputs host to
    device on one stream while wdot goes device to host on another (the
    ceiling of the end-to-end leg, which overlaps the same copies with the
    kernel)."""
    import torch
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    cur = torch.cuda.current_stream()

    def step():
        s1.wait_stream(cur)
        s2.wait_stream(cur)
        with torch.cuda.stream(s1):
            Pd.copy_(Ph, non_blocking=True)
            Td.copy_(Th, non_blocking=True)
            Yd.copy_(Yh, non_blocking=True)
        with torch.cuda.stream(s2):
            Wh.copy_(Wd, non_blocking=True)
        cur.wait_stream(s1)
        cur.wait_stream(s2)

    times = []
    for r in range(reps + 2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step()
        torch.cuda.synchronize()
        if r >= 2:
            times.append(time.perf_counter() - t0)
    return sorted(times)[len(times) // 2]


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The maximum of a per-rank time over all ranks (every rank calls it)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_mpts(points_per_rank: int, world: int, ms_max: float) -> float:
    """Mpoints/s of the job: every rank's points over the slowest rank's time."""
    return points_per_rank * world / (ms_max * 1e-3) / 1e6


def choose_head(modes, results, err, head_arg: str, world: int, device=None) -> str:
    """The headline mode: the fastest whose error against the oracle (checked
    on rank 0) is within 1e-6 normwise, or `head_arg` when it names a mode.
    Under several ranks rank 0's choice is broadcast, so that every rank times
    the same kernel whatever its own timings say."""
    ok = [m for m in modes if m in err and err[m]["norm_max"] <= 1e-6] or modes[:1]
    head = max(ok, key=lambda m: results[m]["value"]) if head_arg == "auto" or head_arg not in modes else head_arg
    if world > 1:
        import torch
        import torch.distributed as dist
        hv = torch.tensor([modes.index(head)], dtype=torch.int64, device=device)
        dist.broadcast(hv, src=0)
        head = modes[int(hv.item())]
    return head


def rank_states(ns: int, ng: int, rank: int):
    """The points rank `rank` evaluates: its own seeded draw (weak scaling)."""
    from chemgen_b200 import synthetic
    return synthetic.states(ns, ng, seed=1000 + rank)


def surrogate_leg(args, gm, stream):
    """Train the MLP surrogate on exact-kernel samples, then report its
    accuracy (normwise, measured against the FP64 kernel), the fused kernel's
    points/s, the error gate's fallback rate and what the surrogate with
    fallback gains over the exact kernels at that tolerance."""
    import torch
    from chemgen_b200 import surrogate as S
    sur = S.Surrogate(gm, seed=0)
    info = sur.fit(S.TrainConfig(samples=args.surrogate_samples, epochs=args.surrogate_epochs))
    n = args.surrogate_points
    P, T, Y = sur.sample_states(n, torch.Generator(device="cuda").manual_seed(4242))
    W64 = torch.empty((gm.ns, n), dtype=torch.float64, device="cuda")
    W = torch.empty_like(W64)
    est = torch.empty(n, dtype=torch.float32, device="cuda")
    steps = max(3, min(args.steps, 20))
    ms_fp64 = time_steps(lambda: gm.getrates(P, T, Y, out=W64, mode="fp64", stream=stream), steps, 3, stream)
    ms_mixed = time_steps(lambda: gm.getrates(P, T, Y, out=W, mode="mixed", stream=stream), steps, 3, stream)
    gm.getrates(P, T, Y, out=W64, mode="fp64", stream=stream)
    ms_fused = time_steps(lambda: sur.predict_fused(P, T, Y, W, est), steps, 3, stream)
    err = ((W - W64).abs().max(dim=0).values / W64.abs().max(dim=0).values).cpu().numpy()
    q = lambda a, v: float(np.quantile(a, v))
    mp = lambda ms: n / (ms * 1e-3) / 1e6

    def gate(margin, exact_mode):
        run = S.SurrogateGetrates(sur, tol=args.surrogate_tol, exact_mode=exact_mode, margin=margin)
        Wg = torch.empty_like(W64)
        ms = time_steps(lambda: run(P, T, Y, out=Wg), steps, 2, stream)
        run(P, T, Y, out=Wg)
        e = ((Wg - W64).abs().max(dim=0).values / W64.abs().max(dim=0).values).cpu().numpy()
        return ms, e, {"tol": args.surrogate_tol, "margin": margin, "exact_mode": exact_mode,
                       "exact_path": "counted batch (staged FP64, no host wait)" if run._counted else
                       "batch of cap points, count read at the end of the call",
                       "fallback_rate": run.last_fallback,
                       "mpts_with_fallback": mp(ms),
                       "err_after_fallback": {"median": q(e, 0.5), "p99": q(e, 0.99), "p99.9": q(e, 0.999),
                                              "max": float(e.max()),
                                              "points_above_tol": int((e > args.surrogate_tol).sum())},
                       "vs_mixed": ms_mixed / ms}
    # at its tolerance the gate sends back a few tenths of a percent: the
    # counted FP64 batch; the strict gate sends back ~6 %: the mixed kernel
    ms_gate, e_after, g0 = gate(0.0, "fp64")
    _, _, g_strict = gate(0.5, "mixed")
    return {"workload": f"53 species / 325 reactions, {n} points (states drawn on the GPU from the workload's "
                        f"distributions)",
            "network": "inputs 1000/T, ln T, ln P, 53 ln X (BF16 hi+lo); 3 x 256 GELU; 53 + 2 outputs; "
                       "BF16 weights, FP32 accumulation",
            "training": {"samples": info["samples"], "epochs": args.surrogate_epochs, "steps": info["steps"],
                         "data_s": info["t_data_s"], "train_s": info["t_train_s"],
                         "error_head_s": info["t_error_head_s"], "final_loss": info["final_loss"]},
            "err_normwise": {"median": q(err, 0.5), "p90": q(err, 0.9), "p99": q(err, 0.99), "max": float(err.max())},
            "fused_kernel_mpts": mp(ms_fused), "fp64_kernel_mpts": mp(ms_fp64), "mixed_kernel_mpts": mp(ms_mixed),
            "gate": g0,
            "gate_strict": g_strict,
            "gain": {"fused_vs_fp64": ms_fp64 / ms_fused, "fused_vs_mixed": ms_mixed / ms_fused,
                     "with_fallback_vs_fp64": ms_fp64 / ms_gate, "with_fallback_vs_mixed": ms_mixed / ms_gate}}


def normwise(W, Wref):
    """Per point max_k |W - Wref| / max_k |Wref| (species-major tensors)."""
    return ((W - Wref).abs().max(dim=0).values / Wref.abs().max(dim=0).values.clamp_min(1e-300)).cpu().numpy()


def other_configs(args, stream):
    """The configurations beside the headline workload, each timed with CUDA
    events on resident inputs (states with the workload's distributions
    unless stated): the real GRI30 mechanism; the reference mini-app's own
    state distribution (chemistry_mini_app.j2:37-44); 348 species / 2163
    reactions at 2^18 points on the tensor-core mixed kernel against the
    table-driven FP64 kernel; and the analytic Jacobian at 65536 points."""
    import torch
    from chemgen_b200 import synthetic
    from chemgen_b200.mechanism import Mechanism
    from chemgen_b200.runtime import GpuMechanism
    steps = max(3, min(args.steps, 20))
    dev = torch.device("cuda")
    out = {}

    def rate_legs(gm, ng, P, T, Y, modes=("fp64", "mixed")):
        W64 = torch.empty_like(Y)
        W = torch.empty_like(Y)
        res = {}
        for m in modes:
            ms = time_steps(lambda: gm.getrates(P, T, Y, out=W, mode=m, stream=stream), steps, 3, stream)
            res[m] = {"mpts": ng / (ms * 1e-3) / 1e6, "ms_per_step": ms, "kernel": gm.kernel_kind(m)}
        gm.getrates(P, T, Y, out=W64, mode="fp64", stream=stream)
        gm.getrates(P, T, Y, out=W, mode="mixed", stream=stream)
        e = normwise(W, W64)
        res["mixed"]["err_vs_fp64_kernel"] = {"max": float(e.max()), "median": float(np.median(e))}
        return res

    ng = 1 << 20
    # real GRI30 (the reference's own mechanism file, as its emitter sees it: 322 reactions)
    gri = Mechanism.from_json(str(np.load(os.path.join(REPO, "tests", "golden", "gri30.npz"))["mech"]))
    gm = GpuMechanism(gri, generated=True)
    P, T, Y = (torch.from_numpy(x).to(dev) for x in synthetic.states(gri.ns, ng, seed=2000))
    out["gri30"] = dict(points=ng, ns=gri.ns, nr=gri.nr, **rate_legs(gm, ng, P, T, Y))
    # the reference mini-app's state distribution on the headline mechanism
    mech = synthetic.gri_shape()
    gm = GpuMechanism(mech, generated=True)
    P, T, Y = (torch.from_numpy(x).to(dev) for x in synthetic.miniapp_states(mech.ns, ng, seed=2001))
    out["miniapp_states_53_325"] = dict(points=ng, distribution="T ~ U(300, 2000) K, P = 1 atm, Y_k ~ U(0, 1/(ns-1)), "
                                        "last species the remainder", **rate_legs(gm, ng, P, T, Y))
    del P, T, Y
    # 348 species / 2163 reactions at 2^18 points: tensor-core mixed vs table FP64
    big = synthetic.jetsurf_shape()
    gm = GpuMechanism(big)
    n3 = 1 << 18
    P, T, Y = (torch.from_numpy(x).to(dev) for x in synthetic.states(big.ns, n3, seed=2002))
    legs = rate_legs(gm, n3, P, T, Y)
    npad, kdim = (big.ns + 31) // 32 * 32, (big.nr + 15) // 16 * 16
    dense = 2.0 * 3 * npad * kdim
    nnz = sum(len(r.reactants) + len(r.products) for r in big.reactions)
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            bf16 = float(json.load(f)["bf16_tflops"])
    except Exception:
        bf16 = 1590.0
    tf = dense * legs["mixed"]["mpts"] * 1e6 / 1e12
    legs["mixed"]["tensor"] = {"dense_flop_per_point": dense, "dense_tflops": tf, "bf16_peak_tflops": bf16,
                               "frac_of_bf16_peak": tf / bf16, "sparse_equivalent_flop_per_point": 2.0 * nnz,
                               "note": "BF16 x3 split of q: 3 MMAs of M=128, N=npad, K=16 per 16-reaction chunk"}
    # per-species error of the tensor-core mixed kernel against the FP64 kernel (itself within 1e-10 of
    # the oracle): max over points of |dW_k| relative to the species' own largest |W_k|, and relative to
    # the point's largest |W| (the normwise measure, split by species)
    W64 = torch.empty_like(Y)
    Wm = torch.empty_like(Y)
    gm.getrates(P, T, Y, out=W64, mode="fp64", stream=stream)
    gm.getrates(P, T, Y, out=Wm, mode="mixed", stream=stream)
    dW = (Wm - W64).abs()
    own = (dW.max(dim=1).values / W64.abs().max(dim=1).values.clamp_min(1e-300)).cpu().numpy()
    nrm = (dW / W64.abs().max(dim=0).values.clamp_min(1e-300)).max(dim=1).values.cpu().numpy()
    legs["mixed"]["err_per_species"] = {
        "relative_to_species_max": [float(f"{x:.2g}") for x in own],
        "relative_to_point_max": [float(f"{x:.2g}") for x in nrm],
        "worst_species": [mech_sp for mech_sp in (big.species[int(k)].name for k in np.argsort(-nrm)[:5])]}
    del W64, Wm, dW
    out["c3_348_2163"] = dict(points=n3, ns=big.ns, nr=big.nr, **legs)
    del P, T, Y
    # analytic Jacobian at 65536 points on the headline mechanism
    gm = GpuMechanism(mech)
    n4 = 65536
    P, T, Y = (torch.from_numpy(x).to(dev) for x in synthetic.states(mech.ns, n4, seed=2003))
    jac = {}
    for prec in ("fp64", "fp32"):
        J = gm.jacobian(P, T, Y, precision=prec)
        ms = time_steps(lambda: gm.jacobian(P, T, Y, precision=prec, out=J, stream=stream), steps, 3, stream)
        jac[prec] = {"mpts": n4 / (ms * 1e-3) / 1e6, "ms_per_step": ms,
                     "J_write_gbs": J.numel() * J.element_size() / (ms * 1e-3) / 1e9}
    G = torch.randn_like(Y)
    ms = time_steps(lambda: gm.vjp(P, T, Y, G, stream=stream), steps, 3, stream)
    jac["vjp_fp64"] = {"mpts": n4 / (ms * 1e-3) / 1e6, "ms_per_step": ms}
    out["c4_jacobian_53_325"] = dict(points=n4, **jac)
    return out


def time_steps(fn, steps, warmup, stream):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / max(steps, 1)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from chemgen_b200 import ops, pack, synthetic
    from chemgen_b200.runtime import GpuMechanism, lib
    import ctypes

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if args.configs_only:
        if rank == 0:
            print(json.dumps({"configs": other_configs(args, torch.cuda.current_stream())}), flush=True)
        return
    mech = synthetic.gri_shape()
    blob = pack.pack(mech).to_blob()
    gm = GpuMechanism(mech, device=local_rank, generated=not args.table)
    ng = args.ng
    P, T, Y = rank_states(mech.ns, ng, rank)
    Pd, Td, Yd = (torch.from_numpy(x).to(dev) for x in (P, T, Y))
    W = torch.empty_like(Yd)
    stream = torch.cuda.current_stream()

    # the table-driven tensor-core mixed kernel on its own handle
    gm_tc = GpuMechanism(blob, device=local_rank)
    gm_tc.use_generated(False)
    modes = []
    for m in args.modes.split(","):
        try:
            gm.getrates(Pd[:64].contiguous(), Td[:64].contiguous(), Yd[:, :64].contiguous(), mode=m)
            modes.append(m)
        except Exception:
            pass
    torch.cuda.synchronize()

    # FP64 roofline denominators, measured on this GPU
    fma_tf, c_exp, c_log, c_rcp = (ctypes.c_double() for _ in range(4))
    lib().chemgen_probe_fp64(local_rank, ctypes.byref(fma_tf), ctypes.byref(c_exp), ctypes.byref(c_log),
                             ctypes.byref(c_rcp))
    inv = ops.inventory(mech)
    flop_pt = ops.flop_equivalents(inv, c_exp.value, c_log.value, c_rcp.value)
    bytes_pt = ops.bytes_per_point(mech.ns)
    hbm_peak, hbm_src = measured_peaks()

    def runner(m):
        if m == "mixed_tc":
            return lambda: gm_tc.getrates(Pd, Td, Yd, out=W, mode="mixed", stream=stream)
        return lambda: gm.getrates(Pd, Td, Yd, out=W, mode=m, stream=stream)

    if "mixed_tc" in args.modes.split(",") and gm_tc.kernel_kind("mixed") == "table":
        modes.append("mixed_tc")
    results = {}
    for m in modes:
        fn = runner(m)
        if world > 1:
            dist.barrier()
        ms = max_over_ranks(time_steps(fn, args.steps, args.warmup, stream), world, dev)
        kind = gm_tc.kernel_kind("mixed") + "-tensorcore" if m == "mixed_tc" else gm.kernel_kind(m)
        results[m] = {"ms_per_step": ms, "value": whole_job_mpts(ng, world, ms), "kernel": kind}

    # errors against the oracle on a bounded sample (rank 0; every world size,
    # so that the headline mode is chosen the same way at any N) and the CPU
    # baseline (rank 0, single GPU only)
    err = {}
    cpu = None
    if rank == 0:
        from oracle import oracle
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.getrates(blob, P[:512], T[:512], np.ascontiguousarray(Y[:, :512]), nthreads=cores)
        pilot = 512 / (time.perf_counter() - t0)
        sample = int(min(ng, max(2048, pilot * args.cpu_seconds))) if world == 1 else min(ng, 8192)
        idx = np.sort(np.random.default_rng(7).choice(ng, sample, replace=False))
        Ps, Ts, Ys = P[idx], T[idx], np.ascontiguousarray(Y[:, idx])
        t0 = time.perf_counter()
        r = oracle.rates(blob, Ps, Ts, Ys, mech.nr, nthreads=cores) if sample <= 65536 else None
        t_rates = time.perf_counter() - t0
        t0 = time.perf_counter()
        w_ref = oracle.getrates(blob, Ps, Ts, Ys, nthreads=cores)
        dt = time.perf_counter() - t0
        n1 = min(sample, 16384)
        t0 = time.perf_counter()
        oracle.getrates(blob, Ps[:n1], Ts[:n1], np.ascontiguousarray(Ys[:, :n1]), nthreads=1)
        dt1 = time.perf_counter() - t0
        if world == 1:
            cpu = {"value": sample / dt / 1e6, "unit": "Mpoints/s", "cores": cores, "kind": "port",
                   "sample": f"{sample} random points of the workload, FP64 C restatement of the reference's "
                             f"generated getrates, OpenMP over points ({dt:.1f} s)",
                   "single_core": {"value": n1 / dt1 / 1e6, "unit": "Mpoints/s", "points": n1}}
        idx_t = torch.from_numpy(idx).to(dev)
        for m in modes:
            runner(m)()
            w = W.index_select(1, idx_t).cpu().numpy()
            S = r["S"] if r is not None else None
            err[m] = oracle.errors(w, w_ref, S)
        del t_rates

    head = choose_head(modes, results, err, args.head, world, dev)

    # clocks during a timed pass of the headline mode
    sampler = ClockSampler(local_rank)
    fn = runner(head)
    steps_c = max(args.steps, int(math.ceil(args.clock_ms / max(results[head]["ms_per_step"], 1e-3))))
    with sampler:
        ms_c = time_steps(fn, steps_c, 2, stream)
    clocks = sampler.summary()
    clocks["timed_ms_per_step"] = ms_c

    # end to end through the host-pointer API: pinned inputs in, wdot back on the host
    Ph, Th, Yh = (torch.from_numpy(x).pin_memory() for x in (P, T, Y))
    Wh = torch.empty_like(Yh).pin_memory()
    gm_e2e = gm_tc if head == "mixed_tc" else gm
    mode_e2e = "mixed" if head == "mixed_tc" else head
    for _ in range(2):
        gm_e2e.getrates_host(Ph, Th, Yh, out=Wh.numpy(), mode=mode_e2e)
    k_e2e = max(1, min(args.steps, 50)) if args.e2e_steps < 0 else args.e2e_steps
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        gm_e2e.getrates_host(Ph, Th, Yh, out=Wh.numpy(), mode=mode_e2e)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / max(k_e2e, 1), world, dev)
    link_s = max_over_ranks(link_step_seconds(Ph, Th, Yh, Wh, Pd, Td, Yd, W), world, dev)

    if rank != 0:
        return
    sur = None
    if world == 1 and args.surrogate_samples > 0 and mech.ns + 2 <= 64:
        del Ph, Th, Yh, Wh
        sur = surrogate_leg(args, gm, stream)
    configs = None
    if world == 1 and not args.no_configs:
        del W, Pd, Td, Yd
        configs = other_configs(args, stream)
    sm_count = torch.cuda.get_device_properties(local_rank).multi_processor_count

    def roof(m):
        """The roofline of the kernel timed in mode m.  FP64 kernel: bound by
        its FP64 pipe, work = the rate law's FP64 flop-equivalents.  Mixed
        kernel: its exponents run in FP64, 2^f on the SFU and the products in
        FP32, so no single pipe carries the work; what bounds it is the issue
        rate (4 warp instructions per clock per SM), achieved = the warp
        instructions it issues per point (ncu, committed) x points/s, peak at
        the SM clock sampled while it ran.  Both report the other measure
        beside it, and the HBM fraction."""
        ms = results[m]["ms_per_step"]
        fp64_achieved = flop_pt * ng / (ms * 1e-3) / 1e12
        fp64 = {"achieved": fp64_achieved, "peak": fma_tf.value, "unit": "TFLOP/s",
                "frac": fp64_achieved / fma_tf.value,
                "peak_source": "FP64 FMA rate measured live on this GPU (chemgen_probe_fp64)",
                "flop_equiv_per_point": flop_pt,
                "transcendental_cost_fma": {"exp": c_exp.value, "log": c_log.value, "rcp": c_rcp.value}}
        traffic = ncu_traffic(m, mech.ns, mech.nr)
        hbm = {"achieved_gbs": bytes_pt * ng / (ms * 1e-3) / 1e9, "peak_gbs": hbm_peak,
               "frac": bytes_pt * ng / (ms * 1e-3) / 1e9 / hbm_peak, "peak_source": hbm_src,
               "bytes_per_point": bytes_pt}
        iss = ncu_issue(m, mech.ns, mech.nr) if results[m]["kernel"] == "generated" else None
        issue = None
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
        if iss is not None and mhz:
            a = iss["warp_inst_per_point"] * ng / (ms * 1e-3) / 1e9
            pk = 4.0 * sm_count * mhz * 1e6 / 1e9
            issue = {"achieved": a, "peak": pk, "unit": "Gwarp-inst/s", "frac": a / pk,
                     "warp_inst_per_point": iss["warp_inst_per_point"],
                     "peak_source": f"4 warp instructions per clock x {sm_count} SMs x {mhz:.0f} MHz "
                                    "(SM clock sampled during the timed region)",
                     "pipes_ncu": {k: iss[k] for k in ("pipe_fp64", "pipe_fma", "pipe_xu")}}
        if m == "fp64" or issue is None:
            out = {"bound": "fp64", **fp64, "traffic": None if traffic is None else traffic * ng}
            if issue is not None:
                out["issue"] = issue
        else:
            out = {"bound": "issue", **{k: issue[k] for k in ("achieved", "peak", "unit", "frac")},
                   "traffic": None if traffic is None else traffic * ng,
                   "peak_source": issue["peak_source"], "warp_inst_per_point": issue["warp_inst_per_point"],
                   "pipes_ncu": issue["pipes_ncu"],
                   "fp64_equivalent_frac": fp64["frac"], "fp64_equivalent": fp64}
        out["hbm"] = hbm
        return out
    line = {"metric": METRIC, "value": results[head]["value"], "unit": "Mpoints/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": results[head]["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head == "fp64" else "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "mechanism": mech.name, "points_per_gpu": ng, "mode": head,
                       "l2": "inputs larger than L2 (Y is 445 MB per GPU per step)"},
            "roofline": roof(head),
            "cpu_baseline": cpu,
            "e2e": {"value": ng * world / e2e_s / 1e6, "unit": "Mpoints/s",
                    "h2d_bytes_per_step": (2 + mech.ns) * ng * 8, "d2h_bytes_per_step": mech.ns * ng * 8,
                    "api": "chemgen_getrates_host (pinned host buffers, 3-stream chunked copies)",
                    "link": {"ceiling": ng * world / link_s / 1e6, "unit": "Mpoints/s",
                             "both_directions_gbs": (2 + 2 * mech.ns) * ng * 8 / link_s / 1e9,
                             "frac": link_s / e2e_s,
                             "how": "the step's inputs host->device and wdot device->host as plain pinned "
                                    "copies on two streams at once, no kernel (median of 5)"}},
            "gpu_launches": args.steps,
            "clocks": clocks,
            "modes": {m: dict(results[m], err=err.get(m), roofline=roof(m)) for m in modes},
            "surrogate": sur,
            "configs": configs}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
