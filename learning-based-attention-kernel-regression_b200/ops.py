"""The library's entry points as torch custom ops (namespace `laker_b200`).

Each `torch.ops.laker_b200.<name>` wraps one call of liblaker_b200.so's C ABI
(include/laker_b200.h) with a schema and a fake (shape-only) implementation,
so the kernels are operators torch knows: they run under their own names in
profiler traces, take part in FakeTensor / meta shape propagation, and can be
called from other torch code without this package's classes.  The operator,
preconditioner, solver and prediction paths of this package call the kernels
through these ops.

    pack(E, precision)                         -> packed32 / packed64 embeddings
    attn_matvec(rows, m, cols, n, d, lam, clamp, x)  (lam I + exp(Er Ec^T)) x
    attn_residual(rows64, m, cols64, n, d, lam, clamp, x, b)   b - (...) x, FP64
    attn_diagonal(packed64, n, d, lam)         lam + exp(|e_i|^2)
    kernel_eval(rows64, m, cols64, p, d, clamp, out_f64)   exp(Er Ec^T), m x p
    precond_apply(q32, w32, n, nr, inv_sqrt_iso, r, out_f64)   CCCP P r
    pcg_solve(...)                             fused PCG -> (x, stats)
    variance_finalize(q64, m, d, kxq, v)       max(0, exp(|q|^2) - sum K V)

`attn_matvec` runs the FP32 kernels on packed32 buffers and the FP64 kernels
on packed64 ones; the same tensor passed as rows and cols with m == n selects
the symmetric operator kernels.  Every op requires CUDA tensors and fails
loudly otherwise: there is no CPU implementation.
"""

from __future__ import annotations

from typing import Optional, Tuple

import torch

from . import _lib

STATS_FIELDS = tuple(name for name, _ in _lib.laker_pcg_result._fields_)


@torch.library.custom_op("laker_b200::pack", mutates_args=())
def pack(E: torch.Tensor, precision: int) -> torch.Tensor:
    """Pair-interleaved FP32 (precision 32) or row-padded FP64 (64) layout of E (n x d)."""
    if precision == 32:
        return _lib.pack_f32(E)
    if precision == 64:
        return _lib.pack_f64(E)
    raise ValueError(f"precision must be 32 or 64, got {precision}")


@pack.register_fake
def _pack_fake(E, precision):
    n, d = int(E.shape[0]), int(E.shape[1])
    lib = _lib.load()
    if precision == 32:
        return E.new_empty(lib.laker_packed32_floats(n, d), dtype=torch.float32)
    return E.new_empty(lib.laker_packed64_doubles(n, d), dtype=torch.float64)


@torch.library.custom_op("laker_b200::attn_matvec", mutates_args=())
def attn_matvec(rows: torch.Tensor, m: int, cols: torch.Tensor, n: int, d: int, lam: float,
                clamp: bool, x: torch.Tensor) -> torch.Tensor:
    """Y = lam X[:m] + exp(Er Ec^T) X for X (n,) or (n, k); lam applies when m == n."""
    if rows.dtype == torch.float64:
        return _lib.attn_matvec_f64(rows, m, cols, n, d, lam, int(clamp), x.to(torch.float64))
    return _lib.attn_matvec_f32(rows, m, cols, n, d, lam, int(clamp), x.to(torch.float32))


@attn_matvec.register_fake
def _attn_matvec_fake(rows, m, cols, n, d, lam, clamp, x):
    return x.new_empty((m,) + tuple(x.shape[1:]), dtype=rows.dtype)


@torch.library.custom_op("laker_b200::attn_residual", mutates_args=())
def attn_residual(rows64: torch.Tensor, m: int, cols64: torch.Tensor, n: int, d: int, lam: float,
                  clamp: bool, x: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """B - (lam X[:m] + exp(Er Ec^T) X) with the FP64 kernels."""
    return _lib.attn_matvec_f64(rows64, m, cols64, n, d, lam, int(clamp), x.to(torch.float64),
                                B=b.to(torch.float64))


@attn_residual.register_fake
def _attn_residual_fake(rows64, m, cols64, n, d, lam, clamp, x, b):
    return x.new_empty((m,) + tuple(x.shape[1:]), dtype=torch.float64)


@torch.library.custom_op("laker_b200::attn_diagonal", mutates_args=())
def attn_diagonal(packed64: torch.Tensor, n: int, d: int, lam: float) -> torch.Tensor:
    """lam + exp(|e_i|^2) in FP64."""
    return _lib.attn_diagonal(packed64, n, d, lam, packed64.device)


@attn_diagonal.register_fake
def _attn_diagonal_fake(packed64, n, d, lam):
    return packed64.new_empty((n,), dtype=torch.float64)


@torch.library.custom_op("laker_b200::kernel_eval", mutates_args=())
def kernel_eval(rows64: torch.Tensor, m: int, cols64: torch.Tensor, p: int, d: int, clamp: bool,
                out_f64: bool) -> torch.Tensor:
    """exp(Er Ec^T) (m x p) from FP64 logits, FP64 or FP32 output."""
    return _lib.kernel_eval(rows64, m, cols64, p, d, int(clamp),
                            torch.float64 if out_f64 else torch.float32, rows64.device)


@kernel_eval.register_fake
def _kernel_eval_fake(rows64, m, cols64, p, d, clamp, out_f64):
    return rows64.new_empty((m, p), dtype=torch.float64 if out_f64 else torch.float32)


@torch.library.custom_op("laker_b200::precond_apply", mutates_args=())
def precond_apply(q32: torch.Tensor, w32: torch.Tensor, n: int, nr: int, inv_sqrt_iso: float,
                  r: torch.Tensor, out_f64: bool) -> torch.Tensor:
    """Z = c^-1/2 R + Q W Q^T R (q32: Q padded to a multiple of 4 columns)."""
    pc = _lib.precond_struct(q32, w32, n, nr, inv_sqrt_iso)
    return _lib.precond_apply(pc, r, torch.float64 if out_f64 else torch.float32)


@precond_apply.register_fake
def _precond_apply_fake(q32, w32, n, nr, inv_sqrt_iso, r, out_f64):
    return r.new_empty(r.shape, dtype=torch.float64 if out_f64 else torch.float32)


@torch.library.custom_op("laker_b200::pcg_solve", mutates_args=())
def pcg_solve(packed32: torch.Tensor, packed64: torch.Tensor, n: int, d: int, lam: float,
              clamp: bool, q32: Optional[torch.Tensor], w32: Optional[torch.Tensor], nr: int,
              inv_sqrt_iso: float, b: torch.Tensor, x0: Optional[torch.Tensor], tol: float,
              max_iter: int, reliable_delta: float, breakdown_eps: float, check_every: int,
              profile: bool, column_stop: bool = False) -> Tuple[torch.Tensor, torch.Tensor]:
    """Fused mixed-precision PCG for b of shape (n,) or (n, k): returns x
    (FP64, b's shape) and the solve's report as a float64 CPU tensor in the
    order of STATS_FIELDS (status, iterations, ...).  For k right-hand sides
    alpha and beta are per column and the stop test is the Frobenius one of
    the reference's solve_2d, or per column with `column_stop`.  A breakdown,
    non-finite value or the iteration cap is reported in the status, not
    raised."""
    op = _lib.laker_operator(packed32.data_ptr(), packed64.data_ptr(), n, d, float(lam), int(clamp))
    pc = _lib.precond_struct(q32, w32, n, nr, inv_sqrt_iso) if q32 is not None else None
    bb = b.to(torch.float64).contiguous()
    x = x0.to(device=b.device, dtype=torch.float64).clone().contiguous() if x0 is not None \
        else torch.empty_like(bb)
    params = _lib.laker_pcg_params(float(tol), int(max_iter), float(reliable_delta),
                                   float(breakdown_eps), int(check_every), int(x0 is not None),
                                   int(profile), int(column_stop))
    res = _lib.pcg_solve(op, pc, bb, x, params)
    stats = torch.tensor([float(getattr(res, f)) for f in STATS_FIELDS], dtype=torch.float64)
    return x, stats


@pcg_solve.register_fake
def _pcg_solve_fake(packed32, packed64, n, d, lam, clamp, q32, w32, nr, inv_sqrt_iso, b, x0, tol,
                    max_iter, reliable_delta, breakdown_eps, check_every, profile,
                    column_stop=False):
    return (b.new_empty(b.shape, dtype=torch.float64),
            torch.empty(len(STATS_FIELDS), dtype=torch.float64, device="cpu"))


def result_from_stats(stats: torch.Tensor) -> _lib.laker_pcg_result:
    """The laker_pcg_result struct of a pcg_solve report."""
    res = _lib.laker_pcg_result()
    for (name, ctype), v in zip(_lib.laker_pcg_result._fields_, stats.tolist()):
        setattr(res, name, int(v) if ctype is _lib.c_int else float(v))
    return res


@torch.library.custom_op("laker_b200::variance_finalize", mutates_args=())
def variance_finalize(q64: torch.Tensor, m: int, d: int, kxq: torch.Tensor,
                      v: torch.Tensor) -> torch.Tensor:
    """sigma^2_q = max(0, exp(|e_q|^2) - sum_i K[i, q] V[i, q]) for m queries."""
    return _lib.variance_finalize(q64, m, d, kxq, v.to(torch.float64))


@variance_finalize.register_fake
def _variance_finalize_fake(q64, m, d, kxq, v):
    return kxq.new_empty((m,), dtype=torch.float64)


OPS = ("pack", "attn_matvec", "attn_residual", "attn_diagonal", "kernel_eval", "precond_apply",
       "pcg_solve", "variance_finalize")
