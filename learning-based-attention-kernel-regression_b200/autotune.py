"""Measuring autotuner for the kernel variants.

The fused kernels have a few tile and pipeline choices whose best value
depends on the problem size and the GPU (include/laker_b200.h,
LAKER_VARIANT_*): the logit operands of the tensor-core symmetric operator
(split FP16 or split TF32), its TMEM unit with split TF32 (4 or 2 row tiles
per accumulator buffer) and, per class of multi-RHS chunk width
(<= 32, 33..128, > 128 right-hand sides), whether the multi-RHS kernel takes
its logits from the tensor cores or the CUDA cores.  `autotune` times every
candidate with CUDA events on a synthetic problem of the caller's size (the
same kernel launches the solvers make), checks that the candidates agree to
the FP32 operator's tolerance, keeps the fastest in the library (for the rest
of the process) and returns the choices with their timings.  No counterpart in
the reference (its operator has no kernel variants).
"""

from __future__ import annotations

from typing import Dict, Optional, Sequence

import torch

from . import _lib
from .kernels import AttentionKernelOperator

# agreement required between two variants of the same product (relative,
# per output column): the split-TF32 / split-FP16 products differ at ~1e-6
AGREE_RTOL = 1e-4


def _time_ms(fn, reps: int) -> float:
    fn()  # warm-up (and the first-call set-up of a variant)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _colrel(a: torch.Tensor, b: torch.Tensor) -> float:
    a, b = a.double(), b.double()
    if a.dim() == 1:
        a, b = a.unsqueeze(1), b.unsqueeze(1)
    num = torch.linalg.norm(a - b, dim=0)
    den = torch.linalg.norm(b, dim=0).clamp(min=1e-300)
    return float((num / den).max())


def _k2_slot(k: int) -> int:
    n_chunk = min(((k + 31) // 32) * 32, 256)
    if n_chunk <= 32:
        return _lib.VARIANT_K2_LOGITS_N32
    return _lib.VARIANT_K2_LOGITS_N128 if n_chunk <= 128 else _lib.VARIANT_K2_LOGITS_WIDE


def autotune(n: int = 20000, d: int = 10, ks: Sequence[int] = (16, 64, 256), reps: int = 5,
             device: Optional[torch.device] = None, seed: int = 0) -> Dict[str, dict]:
    """Time the kernel variants at n points (d dimensions) and keep the fastest.

    Args:
        n, d: problem size to tune for (the operator's points and dimension).
        ks: right-hand-side counts of the multi-RHS products to tune (one
            decision per chunk-width class; the widest k of a class decides).
        reps: timed repetitions per candidate.
    Returns:
        {"k1t_unit": {"choice": u, "ms": {2: t2, 4: t4}}, "k2_logits_n32": ...}
    Raises:
        RuntimeError: if two variants of the same product disagree.
    """
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device="cpu").manual_seed(int(seed))
    E = (torch.randn(n, d, generator=g) * (0.5 if d >= 4 else 0.3)).to(dev, torch.float32)
    op = AttentionKernelOperator(E, lambda_reg=1e-2)
    out: Dict[str, dict] = {}

    def pick(name: str, which: int, values: Sequence[int], fn) -> None:
        prev = _lib.get_variant(which)
        times, results = {}, {}
        try:
            for v in values:
                _lib.set_variant(which, v)
                times[v] = _time_ms(fn, reps)
                results[v] = fn()
        finally:
            _lib.set_variant(which, prev)
        ref = results[values[0]]
        for v in values[1:]:
            err = _colrel(results[v], ref)
            if err > AGREE_RTOL:
                raise RuntimeError(f"kernel variants of {name} disagree: {v} vs {values[0]} "
                                   f"({err:.2e} relative)")
        best = min(times, key=times.get)
        _lib.set_variant(which, best)
        out[name] = {"choice": best, "ms": times}

    if _lib.fp32_operator_kernel(n, d) == 2:
        x = torch.randn(n, generator=g).to(dev, torch.float32)
        if op.skip_clamp:  # clamped operators always take split TF32
            pick("k1t_logits", _lib.VARIANT_K1T_LOGITS, (1, 0), lambda: op.matvec(x))
        if _lib.get_variant(_lib.VARIANT_K1T_LOGITS) == 0 or not op.skip_clamp:
            pick("k1t_unit", _lib.VARIANT_K1T_UNIT, (4, 2), lambda: op.matvec(x))
    by_slot: Dict[int, int] = {}
    for k in ks:
        if k > 1:
            slot = _k2_slot(int(k))
            by_slot[slot] = max(by_slot.get(slot, 0), int(k))
    names = {_lib.VARIANT_K2_LOGITS_N32: "k2_logits_n32", _lib.VARIANT_K2_LOGITS_N128: "k2_logits_n128",
             _lib.VARIANT_K2_LOGITS_WIDE: "k2_logits_wide"}
    for slot, k in sorted(by_slot.items()):
        X = torch.randn(n, k, generator=g).to(dev, torch.float32)
        pick(names[slot], slot, (0, 1), lambda X=X: op.matvec(X))
    return out
