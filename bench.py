#!/usr/bin/env python
"""LAKER B200 solve-path benchmark.

Workload (one "step"): one exact-kernel PCG solve of (lambda I + exp(E E^T)) a = y
at n = 100,000 on the synthetic path-loss field (seed = rank), d = 10
PositionEmbedding outputs, CCCP preconditioner with N_r = 256 probes built
beforehand, tol 1e-6 on the TRUE relative residual (FP64 operator).  Inputs
are resident in HBM for `value`; `e2e` repeats the solve through the public
Python API with y copied from pinned host memory and alpha read back.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU under torchrun; every rank solves its own
instance (replicas, weak scaling); timing is the max over ranks.
`--workload sharded` instead solves ONE system row-sharded over the ranks
(strong scaling: p all-gathered over NCCL, three exchanges per iteration).
`--impl reference` times the float64 CPU oracle of the reference path on the
host cores (bounded sample, extrapolated) and prints the same JSON line.
"""

from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "PCG solves/sec & kernel entries/sec at n=100k @1e-6 resid; p50/p99 solve latency"


def solve_workload(n: int) -> str:
    """The default workload's description, the same string in both arms."""
    return (f"exact-kernel PCG solve n={n} d={EMBED_DIM} N_r={NUM_PROBES} tol={TOL} (true float64 "
            "residual), synthetic path-loss field, seed = rank (seed 0 at one GPU)")
N_DEFAULT = 100_000
EMBED_DIM = 10
NUM_PROBES = 256
LAMBDA = 1e-2
TOL = 1e-6
MAX_ITER = 1000

# Iterations the float64 reference recurrence (solve_1d, laker/solvers.py:189-295)
# needs on the n=100,000 seed-0 system with the same CCCP preconditioner,
# counted with `python bench.py --count-reference-iterations` on a B200 (the
# float64 fused matvec applies the operator, the recurrence runs in numpy).
# Used to extrapolate the bounded CPU samples to one full solve.
REFERENCE_ITERATIONS = {100_000: 306}  # true relres 6.29e-7 at stop
REFERENCE_ITERATIONS_FALLBACK = 300


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples SM clock and clock-event reasons every 100 ms (NVML)."""

    REASONS = {
        0x4: "sw_power_cap",
        0x8: "hw_slowdown",
        0x20: "sw_thermal_slowdown",
        0x40: "hw_thermal_slowdown",
        0x80: "hw_power_brake_slowdown",
    }

    def __init__(self, device: torch.device) -> None:
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None
        try:
            import pynvml

            pynvml.nvmlInit()
            handle = None
            try:
                uuid = str(torch.cuda.get_device_properties(device).uuid)
                handle = pynvml.nvmlDeviceGetHandleByUUID(
                    uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                handle = pynvml.nvmlDeviceGetHandleByIndex(device.index or 0)
            self._nvml = pynvml
            self._h = handle
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nvml = None

    def _reasons(self):
        f = getattr(self._nvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or getattr(
            self._nvml, "nvmlDeviceGetCurrentClocksThrottleReasons")
        return int(f(self._h))

    def _run(self):
        while not self._stop.is_set():
            try:
                mhz = self._nvml.nvmlDeviceGetClockInfo(self._h, self._nvml.NVML_CLOCK_SM)
                util = self._nvml.nvmlDeviceGetUtilizationRates(self._h).gpu
                self.samples.append((mhz, self._reasons(), util))
            except Exception:
                pass
            self._stop.wait(0.1)

    def start(self):
        if self._nvml is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()

    def stop(self):
        self._stop.set()
        if self._thread is not None:
            self._thread.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        loaded = [s for s in self.samples if s[2] > 50] or self.samples
        reasons = set()
        for _, bits, _ in self.samples:
            for bit, name in self.REASONS.items():
                if bits & bit:
                    reasons.add(name)
        return {
            "sm_mhz": float(statistics.median(s[0] for s in loaded)),
            "sm_max_mhz": self.max_mhz,
            "reasons": sorted(reasons),
            "samples": len(self.samples),
        }


def ncu_traffic_per_launch(n: int, kernel_id: int = 1):
    """DRAM bytes per FP32 operator launch from the committed ncu summary of
    that kernel, if any."""
    name = "k1t_matvec_n100000.md" if kernel_id == 2 else "k1_matvec_f32_n100000.md"
    path = REPO / "profiles" / name
    if not path.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch_n%d:\s*([0-9.eE+]+)" % n, path.read_text())
    return float(m.group(1)) if m else None


def build_problem(n: int, seed: int, dev: torch.device):
    import laker_b200 as L

    x, y, _ = L.synthetic_field(n, seed)
    emb = L.PositionEmbedding(2, EMBED_DIM, device=dev, dtype=torch.float32)
    with torch.no_grad():
        E = emb(x.to(dev))
    op = L.AttentionKernelOperator(E, lambda_reg=LAMBDA)
    tm = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pre = L.CCCPPreconditioner(num_probes=NUM_PROBES, gamma=0.1, verbose=False, device=dev,
                               dtype=torch.float32).build(op.matvec, n, seed=0, timings=tm)
    torch.cuda.synchronize()
    tm["total"] = time.perf_counter() - t0
    build_problem.last_cccp = tm
    return op, pre, y.double()


# ---------------------------------------------------------------------------
# CPU reference (float64 oracle of the reference path) -- bounded sample
# ---------------------------------------------------------------------------
def reference_iterations(n: int) -> tuple[int, str]:
    v = REFERENCE_ITERATIONS.get(n)
    if v:
        return int(v), "float64 reference recurrence iteration count measured on this system"
    return REFERENCE_ITERATIONS_FALLBACK, "assumed float64 iteration count (not yet measured)"


def cpu_reference_sample(n: int, seed: int, target_s: float) -> dict:
    """Time one float64 PCG iteration of the reference path on the host.

    Bounded: the n^2 matvec is timed on the first m rows (m sized so the sample
    takes ~target_s) and scaled by n/m; the CCCP apply (n x 256 factors) and
    the vector updates are timed in full.  solves/s = 1 / (t_iter * iters).
    """
    if not (REPO / "oracle" / "liblaker_oracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(REPO / "oracle")], check=True)
    from oracle import laker_oracle as O
    import laker_b200 as L

    x, y, _ = L.synthetic_field(n, seed)
    emb = L.PositionEmbedding(2, EMBED_DIM, device=torch.device("cpu"), dtype=torch.float32)
    with torch.no_grad():
        E = emb(x).double().numpy()
    rng = np.random.default_rng(0)
    v = rng.standard_normal(n)
    m = 256
    t = 0.0
    while True:
        t0 = time.perf_counter()
        O.rect_matvec(E[:m], E, v)
        t = time.perf_counter() - t0
        if t >= 0.5 or m >= n:
            break
        m = min(n, m * 4)
    m = int(min(n, max(m, m * target_s / max(t, 1e-6))))
    t0 = time.perf_counter()
    O.rect_matvec(E[:m], E, v)
    t_rows = time.perf_counter() - t0
    t_matvec = t_rows * n / m
    q = rng.standard_normal((n, NUM_PROBES)) / math.sqrt(n)
    state = {"isotropic_coef": 0.01, "q_basis": q, "q_eigenvalues": np.linspace(0.01, 1, NUM_PROBES),
             "q_eigenvectors": np.eye(NUM_PROBES)}
    t0 = time.perf_counter()
    z = O.cccp_apply(state, v)
    xx = v + 0.5 * z
    rr = v - 0.5 * z
    _ = float(rr @ z), float(np.linalg.norm(rr)), xx
    t_rest = time.perf_counter() - t0
    iters, how = reference_iterations(n)
    t_iter = t_matvec + t_rest
    return {
        "solves_per_s": 1.0 / (t_iter * iters),
        "t_iter_s": t_iter,
        "iters": iters,
        "cores": O.c_threads(),
        "sample": (f"float64 oracle: {m} of {n} rows of one fused matvec ({t_rows:.1f} s, scaled "
                   f"x{n / m:.1f}) + one N_r={NUM_PROBES} CCCP apply and vector updates = one PCG "
                   f"iteration ({t_iter:.2f} s), x {iters} iterations ({how})"),
    }


def run_reference(args) -> None:
    rank, world, _ = dist_info()
    if rank != 0:
        return
    n = args.n
    for _ in range(args.warmup):
        cpu_reference_sample(n, 0, args.ref_sample_s)
    vals = []
    last = None
    t_begin = time.perf_counter()
    for _ in range(args.steps):
        last = cpu_reference_sample(n, 0, args.ref_sample_s)
        vals.append(last["solves_per_s"])
    wall = time.perf_counter() - t_begin
    value = float(statistics.median(vals))
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {
            "workload": solve_workload(n),
            "method": "extrapolated: one float64 PCG iteration timed on the host cores "
                      "(matvec on a row sample, scaled) x the float64 reference iteration count",
            "n": n,
            "precision": "float64 (the reference's float32 default does not reach a 1e-6 true "
                         "residual: 1e-2 at n=20k)",
            "sample_wall_s": wall,
        },
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": last["cores"],
                         "kind": "port", "sample": last["sample"]},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args) -> None:
    import torch.distributed as dist

    import laker_b200 as L
    from laker_b200 import _lib

    rank, world, local = dist_info()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
    n = args.n
    op, pre, y = build_problem(n, seed=rank, dev=dev)
    y_dev = y.to(dev)
    peaks = _lib.measure_peaks(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    pcg = L.PreconditionedConjugateGradient(tol=TOL, max_iter=MAX_ITER, verbose=False)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        flush.zero_()
        pcg.solve(op.matvec, pre.apply, y_dev)
    torch.cuda.synchronize()

    clocks = ClockSampler(dev)
    step_ms, iters, accurate, launches = [], [], [], 0
    k1_ms, k1_count, k4_ms = 0.0, 0, 0.0
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record()
        alpha = pcg.solve(op.matvec, pre.apply, y_dev)
        ev[i][1].record()
        res = pcg.last_result
        iters.append(res.iterations)
        accurate.append(res.accurate_matvecs)
        launches += res.kernel_launches
    torch.cuda.synchronize()
    barrier()
    clocks.stop()
    # per-launch operator times for the roofline: one more solve, outside the
    # timed region, with the kernels launched one by one and timed by events
    # (the timed solves replay each iteration as a CUDA graph)
    prof = L.PreconditionedConjugateGradient(tol=TOL, max_iter=MAX_ITER, verbose=False, profile=True)
    flush.zero_()
    prof.solve(op.matvec, pre.apply, y_dev)
    pres_ = prof.last_result
    k1_ms, k1_count, k4_ms = pres_.fp32_matvec_ms, pres_.fp32_matvec_launches, pres_.fp64_matvec_ms
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    relres = pcg.residual_norm / float(torch.linalg.norm(y_dev))

    # ---- end to end through the public API: pinned host y -> solve -> host alpha
    y_host = y.clone().pin_memory()
    e2e_ms = []
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        yd = y_host.to(dev, non_blocking=True)
        a = pcg.solve(op.matvec, pre.apply, yd)
        a_host = a.to("cpu")
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_total = sum(e2e_ms)

    if world > 1:
        t = torch.tensor([total_ms, e2e_total], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_total = float(t[0]), float(t[1])
        ent = torch.tensor([float(sum(iters) + sum(accurate))], device=dev, dtype=torch.float64)
        dist.all_reduce(ent, op=dist.ReduceOp.SUM)
        matvecs_all = float(ent[0])
        lt = torch.tensor([launches], device=dev, dtype=torch.int64)
        dist.all_reduce(lt, op=dist.ReduceOp.SUM)
        launches_all = int(lt[0])
    else:
        matvecs_all = float(sum(iters) + sum(accurate))
        launches_all = launches

    if rank == 0:
        solves = world * args.steps
        value = solves / (total_ms / 1e3)
        k1_avg_ms = k1_ms / max(k1_count, 1)
        # algorithmic work of the FP32 operator as the library evaluates it
        # (symmetric kernel: each off-diagonal entry once and used twice)
        work = _lib.fp32_matvec_work(n, EMBED_DIM)
        kernel_id = _lib.fp32_operator_kernel(n, EMBED_DIM)
        flops_per_launch = work["flops"]
        achieved = flops_per_launch / (k1_avg_ms * 1e-3) / 1e12
        exps_per_s = work["exps"] / (k1_avg_ms * 1e-3)
        traffic = ncu_traffic_per_launch(n, _lib.fp32_operator_kernel(n, EMBED_DIM))
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": solve_workload(n),
                "n": n,
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "precision": "FP32 fused operator in the recurrence; FP64 vectors, inner "
                             "products, scalars and residual recomputation",
                "l2": "flushed between steps (256 MB write)",
            },
            "kernel_entries_per_s": matvecs_all * n * n / (total_ms / 1e3),
            "p50_ms": float(np.percentile(step_ms, 50)),
            "p99_ms": float(np.percentile(step_ms, 99)),
            "iterations": iters,
            "fp64_residual_recomputations": accurate,
            "relres_true": relres,
            "e2e": {
                "value": solves / (e2e_total / 1e3),
                "unit": "solves/s",
                "h2d_bytes_per_step": int(y_host.numel() * y_host.element_size()),
                "d2h_bytes_per_step": int(a_host.numel() * a_host.element_size()),
            },
            "roofline": roofline_block(kernel_id, work, k1_avg_ms, achieved, exps_per_s, peaks,
                                       traffic, n, k4_ms),
            "clocks": clocks.summary(),
            "gpu_launches": launches_all,
        }
        line["relres_true_cpu_oracle"], line["oracle_check"] = oracle_relres(op, alpha, y)
        line["cccp_build_s"] = getattr(build_problem, "last_cccp", None)
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_reference_sample(n, 0, args.cpu_sample_s)
            line["cpu_baseline"] = {"value": cb["solves_per_s"], "unit": "solves/s",
                                    "cores": cb["cores"], "kind": "port", "sample": cb["sample"]}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def oracle_relres(op, alpha, y) -> tuple:
    """||y - A alpha|| / ||y|| with the float64 CPU oracle (OpenMP C on the
    host cores), the check the reference's pipeline logs after a solve
    (laker/core.py:565-574), on the embeddings the GPU used."""
    from oracle import laker_oracle as O

    E64 = op.embeddings.detach().double().cpu().numpy()
    a = alpha.detach().double().cpu().numpy()
    yh = y.detach().double().cpu().numpy()
    t0 = time.perf_counter()
    r = yh - O.attention_matvec(E64, op.lambda_reg, a)
    dt = time.perf_counter() - t0
    rel = float(np.linalg.norm(r) / np.linalg.norm(yh))
    return rel, {"seconds": dt, "cores": O.c_threads(),
                 "what": "float64 oracle operator applied to the returned solution on the host"}


def roofline_block(kernel_id, work, k1_avg_ms, achieved, exps_per_s, peaks, traffic, n, k4_ms):
    """Roofline of the FP32 operator kernel that dominates the solve.

    Tensor-core logits (kernel 2): per entry evaluated the CUDA cores do one
    MUFU exp2 and two FMAs (one for an entry on a diagonal block pair), so the
    binding unit is the exp2 rate; the logits add 3 split products x 2 x 16
    flops per entry on the tensor cores (split FP16 by default, kind::f16,
    against the dense FP16 rate = the bf16 figure; split TF32 against half of
    it).  CUDA-core logits (kernel 1): d + 2 FMAs per entry, bound by the FFMA
    rate."""
    from laker_b200 import _lib
    common = {
        "traffic": traffic,
        "avg_launch_ms": k1_avg_ms,
        "entries_evaluated_per_launch": work["entries"],
        "logical_entries_per_s": n * n / (k1_avg_ms * 1e-3),
        "fp64_matvec_ms_total": k4_ms,
    }
    if kernel_id == 2:
        peak = peaks["mufu_tops"] * 1e12
        f16 = _lib.get_variant(_lib.VARIANT_K1T_LOGITS) == 1
        tf32 = work["entries"] * 96.0 / (k1_avg_ms * 1e-3) / 1e12
        tf32_peak, tf32_src = _tf32_peak()
        if f16:
            tf32_peak, tf32_src = 2.0 * tf32_peak, tf32_src.replace("half the", "the").replace(
                "TF32 dense rate", "FP16 dense rate")
        return dict(common, **{
            "bound": "mufu",
            "kernel": "k1t_matvec (symmetric FP32 operator, split-%s tcgen05 logits)"
                      % ("FP16" if f16 else "TF32"),
            "achieved": exps_per_s / 1e12, "peak": peaks["mufu_tops"], "unit": "Texp2/s",
            "frac": exps_per_s / peak,
            "peak_source": "MUFU ex2 microbenchmark measured in this run (laker_measure_peaks)",
            "fma_flops_per_launch": work["flops"], "fma_frac": achieved / peaks["ffma_tflops"],
            "tensor_tf32_tflops": tf32, "tensor_frac": tf32 / tf32_peak,
            "tensor_peak_source": tf32_src,
        })
    return dict(common, **{
        "bound": "fma",
        "kernel": "k1s_matvec_f32 (symmetric FP32 fused matvec)" if kernel_id == 1
                  else "k1_matvec_f32 (plain FP32 fused matvec)",
        "achieved": achieved, "peak": peaks["ffma_tflops"], "unit": "TFLOP/s",
        "frac": achieved / peaks["ffma_tflops"],
        "algorithmic_flops_per_launch": work["flops"],
        "peak_source": "FFMA microbenchmark measured in this run (laker_measure_peaks); "
                       "nominal 148 SM x 128 FMA/clk x 2 flop x clock for context",
        "mufu_frac": exps_per_s / (peaks["mufu_tops"] * 1e12),
    })


def kernel_only(args) -> None:
    """One fused matvec alone on the bench embeddings (a clean ncu target):
    the FP32 single-RHS operator, or with --rhs k > 1 the tensor-core
    multi-RHS operator; with --kernel-precision f64 the FP64 (residual)
    operator instead."""
    import laker_b200 as L

    dev = torch.device("cuda", 0)
    x, _, _ = L.synthetic_field(args.n, 0)
    emb = L.PositionEmbedding(2, EMBED_DIM, device=dev, dtype=torch.float32)
    with torch.no_grad():
        E = emb(x.to(dev))
    op = L.AttentionKernelOperator(E, lambda_reg=LAMBDA)
    f64 = args.kernel_precision == "f64"
    dt = torch.float64 if f64 else torch.float32
    v = (torch.randn(args.n, device=dev, dtype=dt) if args.rhs <= 1
         else torch.randn(args.n, args.rhs, device=dev, dtype=dt))
    apply = op.matvec_f64 if f64 else op.matvec
    for _ in range(args.warmup):
        apply(v)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        apply(v)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    k = max(args.rhs, 1)
    name = ("fp64 fused matvec" if k == 1 else "fp64 multi-RHS matvec") if f64 else \
        ("fp32 fused matvec" if k == 1 else "tensor-core multi-RHS matvec")
    out = {"kernel": name, "n": args.n,
           "rhs": k, "ms": ms, "entries_per_s": args.n * args.n / (ms * 1e-3)}
    if k > 1 and not f64:
        out["tf32_tflops_3_products"] = 3 * 2.0 * args.n * args.n * k / (ms * 1e-3) / 1e12
    print(json.dumps(out))


def count_reference_iterations(args) -> None:
    """Iterations of the float64 reference recurrence on the bench system."""
    import laker_b200  # noqa: F401
    from oracle import laker_oracle as O

    dev = torch.device("cuda", 0)
    op, pre, y = build_problem(args.n, 0, dev)
    state = {"isotropic_coef": pre.isotropic_coef, "q_basis": pre.q_basis.double().cpu().numpy(),
             "q_eigenvalues": pre.q_eigenvalues.double().cpu().numpy(),
             "q_eigenvectors": pre.q_eigenvectors.double().cpu().numpy()}

    def apply_a(v):
        return op.matvec_f64(torch.as_tensor(v, device=dev)).cpu().numpy()

    x, iters, rn = O.pcg_solve(apply_a, lambda v: O.cccp_apply(state, v), y.numpy(), tol=TOL,
                               max_iter=MAX_ITER)
    true_rel = float(np.linalg.norm(y.numpy() - apply_a(x)) / np.linalg.norm(y.numpy()))
    print(json.dumps({"n": args.n, "reference_iterations": iters, "recurrence_relres":
                      rn / float(np.linalg.norm(y.numpy())), "true_relres": true_rel}))


# ---------------------------------------------------------------------------
# other workloads (one JSON line each; the default workload is the solve above)
# ---------------------------------------------------------------------------
def _tf32_peak() -> tuple:
    """TF32 dense peak (TFLOP/s) and where it comes from: half the measured
    cuBLAS bf16 burst of MEASURED_PEAKS.json, else half the pool's fallback
    bf16 figure (1.59 PFLOP/s)."""
    pk = _peaks_file()
    if "bf16_tflops" in pk:
        return pk["bf16_tflops"] / 2.0, ("half the measured cuBLAS bf16 burst (MEASURED_PEAKS.json): "
                                        "TF32 dense rate, of measured")
    return 1590.0 / 2.0, "half the fallback bf16 figure (1.59 PFLOP/s; MEASURED_PEAKS.json absent), of fallback"


def _peaks_file() -> dict:
    try:
        return json.loads((REPO / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


def _event_ms(fn, reps: int = 3) -> float:
    fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return min(out)


def _base_line(metric, value, unit, args, ms, dtype, config, higher=True):
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": higher, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic", "config": config}


def workload_sharded(args) -> None:
    """One n-point solve row-sharded over the ranks (strong scaling).

    Every rank builds the same system (seed 0) and the same CCCP factors, then
    the ranks solve it together with sharded_pcg_solve: rows [r0, r1) of A p
    per rank with the fused kernel, p all-gathered and the inner products
    all-reduced over NCCL.  On one GPU the single shard holds every row and
    takes the symmetric kernel, which shows the host-driven loop's cost against
    the fused solve's CUDA-graph replay."""
    import torch.distributed as dist

    import laker_b200 as L
    from laker_b200 import _lib
    from laker_b200.distributed import ShardedPreconditioner, sharded_pcg_solve

    rank, world, local = dist_info()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    n = args.n
    op, pre, y = build_problem(n, seed=0, dev=dev)
    dop = L.DistributedAttentionKernelOperator(op.embeddings, lambda_reg=op.lambda_reg)
    ex, shard = dop.exchange, dop.shard
    spre = ShardedPreconditioner.from_cccp(pre, ex.r0, ex.r1)
    y_dev = y.to(dev)
    peaks = _lib.measure_peaks(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def solve(b):
        return sharded_pcg_solve(shard, ex, b, precond=spre, tol=TOL, max_iter=MAX_ITER)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        flush.zero_()
        solve(y_dev)
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    iters, accurate = [], []
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record()
        x, info = solve(y_dev)
        ev[i][1].record()
        iters.append(info.iterations)
        accurate.append(info.accurate_matvecs)
    torch.cuda.synchronize()
    barrier()
    clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    relres = info.residual_norm / info.rhs_norm

    y_host = y.clone().pin_memory()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        xd, _ = solve(y_host.to(dev, non_blocking=True))
        x_host = xd.to("cpu")
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_total = sum(e2e_ms)

    # this rank's operator product alone, for the roofline
    pf = torch.randn(n, device=dev, dtype=torch.float32)
    k_ms = _event_ms(lambda: shard.apply32(pf, 0.0), reps=5)
    if world > 1:
        t = torch.tensor([total_ms, e2e_total, k_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_total, k_ms = (float(v) for v in t)
    if rank == 0:
        full = ex.rows == n
        kernel_id = _lib.fp32_operator_kernel(n, EMBED_DIM) if full else 0
        if full:
            work = _lib.fp32_matvec_work(n, EMBED_DIM)
        else:  # plain rectangular kernel over the largest shard: d + 1 FMAs and one exp2 per entry
            ent = float(ex.chunk) * n
            work = {"entries": ent, "flops": ent * 2.0 * (EMBED_DIM + 1), "exps": ent}
        achieved = work["flops"] / (k_ms * 1e-3) / 1e12
        roof = roofline_block(kernel_id, work, k_ms, achieved, work["exps"] / (k_ms * 1e-3), peaks,
                              None, n, None)
        roof["logical_entries_per_s"] = float(ex.chunk) * n / (k_ms * 1e-3)
        roof["shard_rows"] = ex.chunk
        # kernels of ours per solve: the operator (plain: k1 + finish; symmetric
        # with tensor-core logits: pack + k1t + finish) per iteration and the
        # FP64 residual (k4 + finish) per recomputation; vector updates are torch ops
        per_op = 3 if kernel_id == 2 else 2
        launches = sum(per_op * a + 2 * b for a, b in zip(iters, accurate))
        line = {
            "metric": METRIC + " (one system row-sharded over the GPUs)",
            "value": args.steps / (total_ms / 1e3),
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": f"exact-kernel PCG solve n={n} d={EMBED_DIM} N_r={NUM_PROBES} tol={TOL} "
                            f"(true float64 residual), one system (seed 0) row-sharded over "
                            f"{world} GPU(s)",
                "n": n,
                "parallelism": f"row shards x{world} (all_gather p, all_reduce scalars, NCCL)"
                               if world > 1 else "single GPU, one shard (host-driven loop)",
                "l2": "flushed between steps (256 MB write)",
            },
            "iterations": iters,
            "fp64_residual_recomputations": accurate,
            "relres_true": relres,
            "p50_ms": float(np.percentile(step_ms, 50)),
            "e2e": {"value": args.steps / (e2e_total / 1e3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(y_host.numel() * y_host.element_size()),
                    "d2h_bytes_per_step": int(x_host.numel() * x_host.element_size())},
            "roofline": roof,
            "clocks": clocks.summary(),
            "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def workload_fit(args) -> None:
    """Config: n=2000 fit + predict at 2000 points through LAKERRegressor."""
    import laker_b200 as L
    from oracle import laker_oracle as O

    dev = torch.device("cuda", 0)
    n = 2000
    x, y, xq = L.synthetic_field(n, 0, m=2000)

    def step():
        model = L.LAKERRegressor(embedding_dim=EMBED_DIM, lambda_reg=LAMBDA, gamma=0.1, pcg_tol=TOL,
                                 pcg_max_iter=MAX_ITER, device=dev, dtype=torch.float32, verbose=False)
        model.fit(x, y, seed=0)
        pred = model.predict(xq)
        torch.cuda.synchronize()
        return model, pred

    for _ in range(args.warmup):
        step()
    times = []
    clocks = ClockSampler(dev)
    clocks.start()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        model, pred = step()
        times.append((time.perf_counter() - t0) * 1e3)
    clocks.stop()
    ms = float(statistics.median(times))
    # float64 oracle with the same probes and FP32-computed embeddings
    E = model.embeddings.double().cpu().numpy()
    Eq = model.embedding_model(xq.to(dev)).detach().double().cpu().numpy()
    probes = L.preconditioner.draw_probes(n, model.preconditioner.nr, torch.float32, dev, 0)
    t0 = time.perf_counter()
    alpha_o, iters_o, _ = O.fit(E, y.double().numpy(), lam=LAMBDA, probes=probes.double().cpu().numpy(),
                                pcg_tol=TOL)
    pred_o = O.predict(Eq, E, alpha_o)
    cpu_s = time.perf_counter() - t0
    line = _base_line("fits+predicts/sec (n=2000 fit, 2000 predictions)", 1e3 / ms, "fits/s", args, ms,
                      "f32", {"workload": "LAKERRegressor.fit + predict, n=2000 train / 2000 test, d=10, "
                              "lambda=1e-2, CCCP default N_r=200, tol 1e-6 (true float64 residual), seed 0",
                              "n": n})
    line["pcg_iterations"] = int(model.pcg_iterations_)
    line["prediction_relerr_vs_float64_oracle"] = float(
        np.linalg.norm(pred.double().cpu().numpy() - pred_o) / np.linalg.norm(pred_o))
    line["relres_true"] = O.relres(E, LAMBDA, model.alpha.double().cpu().numpy(), y.double().numpy())
    line["clocks"] = clocks.summary()
    line["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": "fits/s", "cores": O.c_threads(), "kind": "port",
                            "sample": f"float64 oracle fit + predict, full workload ({cpu_s:.2f} s, "
                                      f"{iters_o} PCG iterations)"}
    print(json.dumps(line), flush=True)


def workload_variance(args) -> None:
    """Config: n=20000, predictive variance at 512 query points (512 RHS)."""
    import laker_b200 as L
    from laker_b200 import _lib
    from oracle import laker_oracle as O

    dev = torch.device("cuda", 0)
    n, m = 20000, 512
    x, y, xq = L.synthetic_field(n, 0, m=m)
    emb = L.PositionEmbedding(2, EMBED_DIM, device=dev, dtype=torch.float32)
    with torch.no_grad():
        E = emb(x.to(dev))
    op = L.AttentionKernelOperator(E, lambda_reg=LAMBDA)
    pre = L.CCCPPreconditioner(gamma=0.1, verbose=False, device=dev, dtype=torch.float32).build(
        op.matvec, n, seed=0)
    core = L.LAKERCore(embedding_dim=EMBED_DIM, pcg_tol=TOL, pcg_max_iter=MAX_ITER, device=dev,
                       dtype=torch.float32, verbose=False)
    xq_d = xq.to(dev)

    def step():
        return core.predict_variance(xq_d, emb, E, op, pre, None, LAMBDA)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clocks.start()
    for i in range(args.steps):
        ev[i][0].record()
        var = step()
        ev[i][1].record()
    torch.cuda.synchronize()
    clocks.stop()
    ms_steps = [a.elapsed_time(b) for a, b in ev]
    ms = float(statistics.median(ms_steps))
    pcg = core.last_pcg
    oracle = variance_oracle_checks(op, pre, emb, xq_d, var, m)
    # the dominant kernel: the tensor-core 512-RHS matvec alone
    X = torch.randn(n, m, device=dev)
    k2_ms = _event_ms(lambda: op.matvec(X))
    tf32 = 3 * 2.0 * n * n * m / (k2_ms * 1e-3) / 1e12
    tf32_peak, tf32_src = _tf32_peak()
    # CPU: one 512-RHS float64 matvec on a row sample, x iterations
    import numpy as _np
    Eh = E.double().cpu().numpy()
    Xh = _np.random.default_rng(0).standard_normal((n, m))
    rows = 256
    while True:  # a sample of about 2 s or more
        t0 = time.perf_counter()
        O.rect_matvec(Eh[:rows], Eh, Xh)
        t_rows = time.perf_counter() - t0
        if t_rows >= 2.0 or rows >= n:
            break
        rows = min(n, rows * 4)
    t_iter = t_rows * n / rows
    cpu_rate = m / (t_iter * max(pcg.iterations, 1))
    line = _base_line("variance queries/sec (n=20k, 512 queries, 1e-6 resid)", m / (ms * 1e-3),
                      "queries/s", args, ms, "f32",
                      {"workload": f"LAKERCore.predict_variance, n={n} train, m={m} queries (512 RHS), "
                                   "d=10, CCCP default N_r, tol 1e-6 (float64 residual, global Frobenius "
                                   "norm as solve_2d)", "n": n, "m": m})
    line.update({
        "pcg_iterations": pcg.iterations, "fp64_residual_recomputations": pcg.accurate_matvecs,
        "relres_frobenius": pcg.residual_norm / max(getattr(pcg, "rhs_norm", 0.0), 1e-300),
        "oracle_checks": oracle,
        "roofline": {"bound": "tensor", "kernel": "k2_tc_matvec (tcgen05 kind::tf32, 3 split products)",
                     "achieved": tf32, "peak": tf32_peak, "unit": "TFLOP/s", "frac": tf32 / tf32_peak,
                     "traffic": None, "avg_launch_ms": k2_ms,
                     "peak_source": tf32_src},
        "clocks": clocks.summary(),
        "cpu_baseline": {"value": cpu_rate, "unit": "queries/s", "cores": O.c_threads(), "kind": "port",
                         "sample": f"float64 oracle 512-RHS matvec on {rows} of {n} rows ({t_rows:.2f} s) "
                                   f"scaled to one iteration x {pcg.iterations} iterations (extrapolated)"},
    })
    print(json.dumps(line), flush=True)


def variance_oracle_checks(op, pre, emb, xq_d, var, m) -> dict:
    """Every one of the m variance solves checked with the float64 CPU oracle.

    The solve of the bench step (k(X, x*) for all m queries, global Frobenius
    stop as solve_2d) is repeated to get its solution V; the oracle applies
    the float64 operator to V on the host (blocked BLAS) for each column's
    true residual.  A converged float64 solve (tol 1e-11, its own residual
    also checked by the oracle) gives the reference sigma^2 of every column,
    against which the bench step's sigma^2 and those of the per-column stop
    (column_stop=True, every column to 1e-6 of its own norm) are compared.
    sigma^2 = k(q,q) - k_q^T A^-1 k_q cancels about 4 digits, so errors are
    also given relative to k(q,q)."""
    import laker_b200 as L
    from laker_b200 import _lib
    from oracle import laker_oracle as O

    dev = op.embeddings.device
    n = op.n
    with torch.no_grad():
        Eq = emb(xq_d).detach()
    q64 = _lib.pack_f64(Eq.double())
    kxq = _lib.kernel_eval(op.packed.packed64, n, q64, m, EMBED_DIM, 0, torch.float64, dev)
    kqq = torch.exp((Eq.double() ** 2).sum(dim=1)).cpu().numpy()
    E64 = op.embeddings.double().cpu().numpy()
    K = kxq.cpu().numpy()

    def solve(tol, column_stop):
        pcg = L.PreconditionedConjugateGradient(tol=tol, max_iter=5000, verbose=False,
                                                column_stop=column_stop)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        V = pcg.solve(op.matvec, pre.apply, kxq)
        v = _lib.variance_finalize(q64, m, EMBED_DIM, kxq, V.to(torch.float64))
        torch.cuda.synchronize()
        return V.double().cpu().numpy(), v.cpu().numpy(), time.perf_counter() - t0, pcg

    def col_relres(V):
        R = K - O.attention_matvec(E64, op.lambda_reg, V)
        return np.linalg.norm(R, axis=0) / np.linalg.norm(K, axis=0), \
            float(np.linalg.norm(R) / np.linalg.norm(K))

    t0 = time.perf_counter()
    V, _, _, _ = solve(TOL, False)
    col, fro = col_relres(V)
    Vt, vt, _, pt = solve(1e-11, False)
    col_t, fro_t = col_relres(Vt)
    Vc, vc, t_c, pc = solve(TOL, True)
    col_c, fro_c = col_relres(Vc)
    ours = var.double().cpu().numpy()

    def errs(v):
        d = np.abs(v - vt)
        return {"max_relerr": float((d / np.maximum(np.abs(vt), 1e-300)).max()),
                "median_relerr": float(np.median(d / np.maximum(np.abs(vt), 1e-300))),
                "max_err_over_kqq": float((d / kqq).max())}

    return {
        "columns_checked": m,
        "oracle_cores": O.c_threads(),
        "oracle_seconds": time.perf_counter() - t0,
        "step_solve": {"relres_frobenius": fro, "max_column_relres": float(col.max()),
                       "median_column_relres": float(np.median(col)),
                       "sigma2_vs_converged": errs(ours)},
        "converged_reference": {"tol": 1e-11, "relres_frobenius": fro_t,
                                "max_column_relres": float(col_t.max()),
                                "iterations": pt.iterations},
        "column_stop": {"seconds": t_c, "iterations": pc.iterations,
                        "relres_frobenius": fro_c, "max_column_relres": float(col_c.max()),
                        "sigma2_vs_converged": errs(vc)},
    }


def workload_batch(args) -> None:
    """Config: 1024 independent regressions, n log-uniform in [500, 20000]."""
    import laker_b200 as L
    from oracle import laker_oracle as O

    dev = torch.device("cuda", 0)
    count = args.count
    ns, lams = L.batch_instances(count)
    ops, ys = [], []
    emb = L.PositionEmbedding(2, EMBED_DIM, device=dev, dtype=torch.float32)
    for i, (n, lam) in enumerate(zip(ns, lams)):
        x, y, _ = L.synthetic_field(n, i)
        with torch.no_grad():
            E = emb(x.to(dev))
        ops.append(L.AttentionKernelOperator(E, lambda_reg=lam))
        ys.append(y.to(dev).double())
    torch.cuda.synchronize()
    tm = {}
    t0 = time.perf_counter()
    pres = L.build_cccp_batched(ops, seeds=list(range(count)), timings=tm)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    pcg = L.BatchedPCG(tol=TOL, max_iter=MAX_ITER)
    for _ in range(args.warmup):
        pcg.solve(ops, pres, ys)
    clocks = ClockSampler(dev)
    clocks.start()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xs = pcg.solve(ops, pres, ys)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    clocks.stop()
    solve_s = float(statistics.median(times))
    # every instance's true residual with the float64 CPU oracle (host cores)
    t_or = time.perf_counter()
    rels = []
    for k in range(count):
        Eh = ops[k].embeddings.double().cpu().numpy()
        yk = ys[k].cpu().numpy()
        r = yk - O.attention_matvec(Eh, lams[k], xs[k].double().cpu().numpy())
        rels.append(float(np.linalg.norm(r) / np.linalg.norm(yk)))
    t_or = time.perf_counter() - t_or
    # the plain single-instance path on an evenly spaced subset, scaled by count
    sub = list(range(0, count, max(1, count // args.plain_subset)))[:args.plain_subset]
    single = L.PreconditionedConjugateGradient(tol=TOL, max_iter=MAX_ITER, verbose=False)
    t_plain = 0.0
    for k in sub:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        single.solve(ops[k].matvec, pres[k].apply, ys[k])
        torch.cuda.synchronize()
        t_plain += time.perf_counter() - t0
    plain_rate = len(sub) / t_plain
    # CPU: float64 oracle iteration cost on a few instances, x their iterations
    cpu_t = 0.0
    csub = sub[: max(1, len(sub) // 8)]
    for k in csub:
        Eh = ops[k].embeddings.double().cpu().numpy()
        v = np.random.default_rng(k).standard_normal(ops[k].n)
        t0 = time.perf_counter()
        O.attention_matvec(Eh, lams[k], v)
        cpu_t += (time.perf_counter() - t0) * pcg.iterations[k]
    cpu_rate = len(csub) / cpu_t
    line = _base_line("batched PCG solves/sec (1024 uneven instances @1e-6 resid)", count / solve_s,
                      "solves/s", args, solve_s * 1e3, "f32",
                      {"workload": f"{count} independent regressions, n log-uniform in [500, 20000], "
                                   "lambda log-uniform in [1e-3, 1e-1], d=10, CCCP default N_r per "
                                   "instance (built beforehand, batched), tol 1e-6 true float64 residual",
                       "instances": count, "total_points": int(sum(ns))})
    line.update({
        "iterations_max": max(pcg.iterations), "iterations_mean": sum(pcg.iterations) / count,
        "oracle_relres": {"instances": count, "max": max(rels), "median": float(np.median(rels)),
                          "above_tol": sum(1 for r in rels if r > TOL), "seconds": t_or,
                          "cores": O.c_threads(),
                          "what": "float64 CPU oracle operator applied to every returned solution"},
        "statuses_ok": sum(1 for s in pcg.statuses if s == 0),
        "batched_cccp_build_s": build_s, "build_phases_s": tm,
        "plain_single_instance_solves_per_s": plain_rate,
        "speedup_vs_plain": (count / solve_s) / plain_rate,
        "gpu_launches": pcg.kernel_launches, "clocks": clocks.summary(),
        "cpu_baseline": {"value": cpu_rate, "unit": "solves/s", "cores": O.c_threads(), "kind": "port",
                         "sample": f"float64 oracle matvec of {len(csub)} instances x their iteration "
                                   "counts (extrapolated)"},
    })
    print(json.dumps(line), flush=True)


def serve_cpu_estimate(trace, recs, n_sample: int = 8) -> dict:
    """CPU baseline of a served trace: the float64 oracle's operator cost for
    an evenly spaced sample of the requests, extrapolated.  Per request: the
    operator on 256 of its n rows (all k right-hand sides: 1 for a fit, m for a
    variance query), scaled to n rows, times the PCG iterations the GPU solve
    of that request took, plus for a fit the CCCP build's operator on its N_r
    probes.  Timing depends only on the shapes, so seeded random embeddings
    of the request's size stand in."""
    from oracle import laker_oracle as O

    rng = np.random.default_rng(0)
    by_rid = {r.rid: r for r in trace}
    sample = trace[:: max(1, len(trace) // n_sample)][:n_sample]
    total = 0.0

    def timed_rows(E, X, rows):
        t0 = time.perf_counter()
        O.rect_matvec(E[:rows], E, X)
        return (time.perf_counter() - t0) * E.shape[0] / rows

    for r in sample:
        n = r.n if r.kind == "fit" else by_rid[r.target].n
        k = 1 if r.kind == "fit" else r.m
        rows = min(n, 256)
        E = rng.standard_normal((n, EMBED_DIM)) * 0.3
        X = rng.standard_normal(n) if k == 1 else rng.standard_normal((n, k))
        total += max(1, recs[r.rid].iterations) * timed_rows(E, X, rows)
        if r.kind == "fit":
            nr = min(n, max(200, int(2 * n ** 0.5)))
            total += timed_rows(E, rng.standard_normal((n, nr)), rows)
    return {"value": len(sample) / total, "unit": "requests/s", "cores": O.c_threads(),
            "kind": "port",
            "sample": f"float64 oracle operator for {len(sample)} of {len(trace)} requests "
                      f"(256 rows per request scaled to n, x the request's PCG iterations, + the "
                      f"CCCP probe product of fits): {total:.1f} s extrapolated"}


def workload_serve(args) -> None:
    """Config: Poisson trace of fit (70 %) and variance (30 %) requests."""
    import laker_b200  # noqa: F401
    from laker_b200.serving import Server, make_trace, run_plain, summarize

    dev = torch.device("cuda", 0)
    rates = [float(r) for r in args.rates.split(",")]
    out = []
    for rate in rates:
        trace = make_trace(args.requests, rate, seed=0, n_range=(1000, 50000), m_range=(16, 256))
        srv = Server(device=dev, hbm_budget=150e9)
        warm = make_trace(6, 1e4, seed=99, n_range=(1000, 4000), m_range=(16, 32))
        srv.run(warm)
        clocks = ClockSampler(dev)
        clocks.start()
        recs = srv.run(trace)
        clocks.stop()
        last_trace, last_recs = trace, recs
        s = summarize(recs)
        s["activity_s"] = dict(srv.stats)
        s["clocks"] = clocks.summary()
        plain = run_plain(srv, trace)
        p = summarize(plain)
        out.append({"rate": rate, "served": s, "plain": p,
                    "speedup_requests_per_s": s["requests_per_s"] / p["requests_per_s"]})
        srv.engine.release()
        del srv
        torch.cuda.empty_cache()
    best = out[-1]
    line = _base_line("served requests/sec with p50/p99 latency (Poisson fit/variance trace)",
                      best["served"]["requests_per_s"], "requests/s", args,
                      best["served"]["makespan_s"] * 1e3, "f32",
                      {"workload": f"{args.requests} requests per rate, Poisson arrivals, 70 % fit "
                                   "(n log-uniform in [1000, 50000]) / 30 % variance (16-256 query "
                                   "points) against a resident model, HBM budget 150 GB, tol 1e-6",
                       "rates": rates})
    line.update({"p50_ms": best["served"]["p50_ms"], "p99_ms": best["served"]["p99_ms"],
                 "clocks": best["served"]["clocks"], "by_rate": out})
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = serve_cpu_estimate(last_trace, last_recs)
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-s", type=float, default=12.0)
    ap.add_argument("--ref-sample-s", type=float, default=5.0)
    ap.add_argument("--count-reference-iterations", action="store_true")
    ap.add_argument("--kernel-only", action="store_true",
                    help="time the FP32 fused matvec alone (profiling target)")
    ap.add_argument("--workload", choices=("solve", "fit", "variance", "batch", "serve", "sharded"),
                    default="solve", help="solve: n=100k PCG solve (the default line); fit: n=2000 "
                    "fit+predict; variance: n=20k x 512 queries; batch: 1024 instances; serve: "
                    "Poisson request trace; sharded: one n=100k solve row-sharded over the GPUs")
    ap.add_argument("--rhs", type=int, default=1, help="--kernel-only: right-hand sides")
    ap.add_argument("--kernel-precision", choices=("f32", "f64"), default="f32",
                    help="--kernel-only: the FP32 operator or the FP64 (residual) operator")
    ap.add_argument("--count", type=int, default=1024, help="batch: instances")
    ap.add_argument("--plain-subset", type=int, default=64, help="batch: single-path sample")
    ap.add_argument("--requests", type=int, default=120, help="serve: requests per rate")
    ap.add_argument("--rates", default="100", help="serve: comma-separated arrival rates (req/s)")
    args = ap.parse_args()
    if args.workload != "solve" and args.impl == "ours":
        {"fit": workload_fit, "variance": workload_variance, "batch": workload_batch,
         "serve": workload_serve, "sharded": workload_sharded}[args.workload](args)
        return
    if args.warmup < 3 and args.impl == "ours" and not args.kernel_only:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.kernel_only:
        kernel_only(args)
    elif args.count_reference_iterations:
        count_reference_iterations(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
