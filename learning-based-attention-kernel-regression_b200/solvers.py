"""Preconditioned conjugate gradient on the B200 path.

Drop-in for laker.solvers.PreconditionedConjugateGradient
(laker/solvers.py:48-394): same constructor arguments, `solve(operator,
preconditioner, rhs, x0)` signature, `iterations` / `residual_norm`
attributes, ValueError for a rhs that is not 1-D or 2-D, RuntimeError on
breakdown, zero RHS returned as is, and a warning when max_iter is reached.

When `operator` is the bound `matvec` of an AttentionKernelOperator and
`preconditioner` the bound `apply` of a CCCPPreconditioner (or None), the
solve runs entirely on the device through laker_pcg_solve: FP32 fused
operator inside the recurrence, FP64 vectors / inner products / scalars, and
reliable updates that replace the recurrence residual by the FP64 residual
b - A x, so the stop test `||b - A x|| <= tol ||b||` holds for the float64
operator.  2-D right-hand sides take the same device loop with column-wise
alpha / beta and the global Frobenius stop test of solve_2d (or, with
`column_stop=True`, a per-column stop).  With a row-sharded operator 2-D
right-hand sides run the same mixed-precision recurrence driven from torch
over the sharded products.  Any other callables run the reference recurrence
unchanged on their CUDA tensors.
"""

from __future__ import annotations

import logging
from typing import Callable, Optional

import torch

from . import _lib, ops
from .distributed import (DistributedAttentionKernelOperator, ShardedPreconditioner,
                          ShardedSolveInfo, sharded_pcg_solve)
from .kernels import AttentionKernelOperator
from .preconditioner import CCCPPreconditioner

logger = logging.getLogger(__name__)

BREAKDOWN_MSG = (
    "PCG breakdown: non-positive curvature detected (p^T A p <= 0). "
    "The operator may be indefinite or the preconditioner may be unsuitable."
)


def _bound_self(fn, cls, names):
    obj = getattr(fn, "__self__", None)
    func = getattr(fn, "__func__", None)
    if isinstance(obj, cls) and func is not None and func.__name__ in names:
        return obj
    return None


class PreconditionedConjugateGradient:
    """PCG solver (laker/solvers.py:48-394) with a fused device path.

    Extra arguments (not in the reference):
        reliable_delta: the FP64 residual is recomputed whenever the
            recurrence residual fell by this factor since the last
            recomputation (mixed-precision reliable update).
        check_every: host polls of the device status (0 = automatic).
        column_stop: 2-D right-hand sides only: stop each column on its own
            FP64 residual (||b_c - A x_c|| <= tol ||b_c||, the column is then
            frozen) instead of the reference's global Frobenius test.

    Extra attributes after solve: `accurate_matvecs` (FP64 residual
    recomputations), `recurrence_norm`, `status` (laker status code).
    """

    def __init__(
        self,
        tol: float = 1e-10,
        max_iter: Optional[int] = None,
        verbose: bool = True,
        restart_freq: Optional[int] = None,
        breakdown_eps: Optional[float] = None,
        autograd_safe: bool = False,
        reliable_delta: float = 0.03,
        check_every: int = 0,
        profile: bool = False,
        column_stop: bool = False,
    ) -> None:
        self.tol = float(tol)
        self.max_iter = max_iter
        self.verbose = verbose
        self.restart_freq = restart_freq
        self.breakdown_eps = breakdown_eps
        self.autograd_safe = autograd_safe
        self.reliable_delta = float(reliable_delta)
        self.check_every = int(check_every)
        self.profile = bool(profile)
        self.column_stop = bool(column_stop)
        self.last_result: Optional[_lib.laker_pcg_result] = None
        self.iterations: int = 0
        self.residual_norm: float = float("inf")
        self.accurate_matvecs: int = 0
        self.recurrence_norm: float = float("inf")
        self.status: int = _lib.LAKER_OK

    def _eps(self, dtype: torch.dtype) -> float:
        if self.breakdown_eps is not None:
            return float(self.breakdown_eps)
        return torch.finfo(dtype).eps ** 0.5

    def solve(
        self,
        operator: Callable[[torch.Tensor], torch.Tensor],
        preconditioner: Optional[Callable[[torch.Tensor], torch.Tensor]],
        rhs: torch.Tensor,
        x0: Optional[torch.Tensor] = None,
    ) -> torch.Tensor:
        if rhs.dim() not in (1, 2):
            raise ValueError(f"rhs must be 1-D or 2-D, got shape {rhs.shape}")
        _lib.require_cuda(rhs, "rhs")
        n = rhs.shape[0]
        max_iter = self.max_iter if self.max_iter is not None else n
        op = _bound_self(operator, AttentionKernelOperator, ("matvec",))
        pc = None
        fused_pc = preconditioner is None
        if preconditioner is not None:
            pc = _bound_self(preconditioner, CCCPPreconditioner, ("apply", "apply_1d", "apply_impl"))
            fused_pc = pc is not None
        if op is not None and fused_pc and not self.autograd_safe and self.restart_freq is None:
            if isinstance(op, DistributedAttentionKernelOperator) and not op.single_device:
                if rhs.dim() == 1:
                    return self._solve_sharded(op, pc, rhs, x0, max_iter)
                return self._solve_mixed_2d(op, preconditioner, rhs, x0, max_iter)
            return self._solve_fused(op, pc, rhs, x0, max_iter)
        if preconditioner is None:
            preconditioner = lambda v: v  # noqa: E731
        x = self._solve_generic(operator, preconditioner, rhs, x0, max_iter)
        _lib.raise_device_status(rhs.device)
        return x

    # ------------------------------------------------------------------
    def _finish(self, status: int, rel: float) -> None:
        if status == _lib.LAKER_ERR_BREAKDOWN:
            raise RuntimeError(BREAKDOWN_MSG)
        if status == _lib.LAKER_ERR_TIMEOUT:
            raise _lib.LakerError(status, "PCG", _lib.status_string(status) +
                                  " (a bounded wait on the GPU expired; the solve was stopped)")
        if status == _lib.LAKER_ERR_NONFINITE:
            raise RuntimeError("PCG encountered a non-finite inner product (NaN/Inf in the data)")
        if status == _lib.LAKER_ERR_NOT_CONVERGED:
            if self.verbose:
                logger.warning("PCG did not converge in %d iterations, rel_res=%.3e",
                               self.iterations, rel)
        elif self.verbose:
            logger.info("PCG converged in %d iterations, rel_res=%.3e", self.iterations, rel)

    def _solve_fused(self, op: AttentionKernelOperator, pc: Optional[CCCPPreconditioner],
                     rhs: torch.Tensor, x0: Optional[torch.Tensor], max_iter: int) -> torch.Tensor:
        p = op.packed
        q32, w32, nr, cis = pc.apply_factors() if pc is not None else (None, None, 0, 0.0)
        x, stats = ops.pcg_solve(
            p.packed32, p.packed64, op.n, op.embedding_dim, op.lambda_reg, not op.skip_clamp,
            q32, w32, nr, cis, rhs, x0, self.tol, int(max_iter), self.reliable_delta,
            self._eps(rhs.dtype), self.check_every, self.profile, self.column_stop)
        res = ops.result_from_stats(stats)
        self.last_result = res
        self.iterations = int(res.iterations)
        self.accurate_matvecs = int(res.accurate_matvecs)
        self.residual_norm = float(res.residual_norm)
        self.rhs_norm = float(res.rhs_norm)
        self.recurrence_norm = float(res.recurrence_norm)
        self.status = int(res.status)
        if res.rhs_norm == 0.0:
            return x.to(rhs.dtype)
        self._finish(res.status, res.residual_norm / res.rhs_norm)
        return x.to(rhs.dtype)

    def _solve_sharded(self, op: DistributedAttentionKernelOperator,
                       pc: Optional[CCCPPreconditioner], rhs: torch.Tensor,
                       x0: Optional[torch.Tensor], max_iter: int) -> torch.Tensor:
        """Row-sharded solve over the operator's process group (every rank
        calls it with the same rhs and gets the full solution)."""
        e = op.exchange
        pre = ShardedPreconditioner.from_cccp(pc, e.r0, e.r1) if pc is not None else None
        info = ShardedSolveInfo()
        try:
            x, _ = sharded_pcg_solve(op.shard, e, rhs, precond=pre, x0=x0, tol=self.tol,
                                     max_iter=max_iter, reliable_delta=self.reliable_delta,
                                     breakdown_eps=self._eps(rhs.dtype), info=info)
        finally:
            self.iterations = info.iterations
            self.accurate_matvecs = info.accurate_matvecs
            self.residual_norm = info.residual_norm
            self.rhs_norm = info.rhs_norm
            self.recurrence_norm = info.recurrence_norm
            self.status = info.status
        if info.rhs_norm > 0.0:
            self._finish(info.status, info.residual_norm / info.rhs_norm)
        return x.to(rhs.dtype)

    def _solve_mixed_2d(self, op: AttentionKernelOperator, preconditioner, rhs, x0, max_iter):
        """Mixed-precision 2-D recurrence (solve_2d semantics, FP64 residual)
        driven from torch, for the row-sharded operator whose products
        exchange rows between ranks on the host side."""
        b = rhs.to(torch.float64)
        pre = preconditioner if preconditioner is not None else (lambda v: v)
        if x0 is None:
            x = torch.zeros_like(b)
            r = b.clone()
        else:
            x = x0.to(device=b.device, dtype=torch.float64).clone()
            r = op.residual_f64(x, b)
        bn = torch.linalg.norm(b).item()
        self.rhs_norm = bn
        self.accurate_matvecs = 0 if x0 is None else 1
        if bn == 0:
            self.iterations = 0
            self.residual_norm = 0.0
            return x.to(rhs.dtype)
        eps = self._eps(rhs.dtype)
        z = pre(r).to(torch.float64)
        p = z.clone()
        rz = torch.sum(r * z, dim=0)
        rmax = torch.linalg.norm(r).item()
        rn = rmax
        status = _lib.LAKER_ERR_NOT_CONVERGED
        it = 0
        for it in range(1, max_iter + 1):
            ap = op.matvec(p.to(torch.float32)).to(torch.float64)
            pap = torch.sum(p * ap, dim=0)
            if torch.any(pap <= -eps * torch.linalg.norm(p, dim=0) * torch.linalg.norm(ap, dim=0)):
                self.iterations = it
                raise RuntimeError(BREAKDOWN_MSG)
            alpha = rz / pap
            x.add_(p * alpha.unsqueeze(0))
            r.sub_(ap * alpha.unsqueeze(0))
            rn = torch.linalg.norm(r).item()
            _lib.raise_device_status(r.device)
            self.recurrence_norm = rn
            rmax = max(rmax, rn)  # running max since the last FP64 recomputation
            if rn <= self.reliable_delta * rmax or rn <= self.tol * bn or it == max_iter:
                r = op.residual_f64(x, b)
                self.accurate_matvecs += 1
                rn = torch.linalg.norm(r).item()
                rmax = rn
                if rn <= self.tol * bn:
                    status = _lib.LAKER_OK
                    break
            z = pre(r).to(torch.float64)
            rz_new = torch.sum(r * z, dim=0)
            beta = rz_new / rz
            p = z + p * beta.unsqueeze(0)
            rz = rz_new
        self.iterations = it
        self.residual_norm = rn
        self.status = status
        self._finish(status, rn / bn)
        return x.to(rhs.dtype)

    def _solve_generic(self, operator, preconditioner, rhs, x0, max_iter):
        """Reference recurrence (solve_1d / solve_2d) for arbitrary callables."""
        if x0 is None:
            x = torch.zeros_like(rhs)
            r = rhs.clone()
        else:
            x = x0.clone()
            r = rhs - operator(x)
        z = preconditioner(r)
        p = z.clone()
        rhs_norm = torch.linalg.norm(rhs).item()
        if rhs_norm == 0:
            self.iterations = 0
            self.residual_norm = 0.0
            return x
        eps = self._eps(p.dtype)
        one_d = rhs.dim() == 1
        rz = torch.dot(r, z) if one_d else torch.sum(r * z, dim=0)
        rel = float("inf")
        for it in range(max_iter):
            ap = operator(p)
            if one_d:
                pap = torch.dot(p, ap)
                bad = (pap <= -eps * torch.linalg.norm(p) * torch.linalg.norm(ap)).item()
            else:
                pap = torch.sum(p * ap, dim=0)
                bad = torch.any(
                    pap <= -eps * torch.linalg.norm(p, dim=0) * torch.linalg.norm(ap, dim=0)
                ).item()
            if bad:
                raise RuntimeError(BREAKDOWN_MSG)
            alpha = rz / pap
            if self.autograd_safe:
                x = x + (alpha * p if one_d else p * alpha.unsqueeze(0))
                r = r - (alpha * ap if one_d else ap * alpha.unsqueeze(0))
            else:
                x.add_(alpha * p if one_d else p * alpha.unsqueeze(0))
                r.sub_(alpha * ap if one_d else ap * alpha.unsqueeze(0))
            if self.restart_freq is not None and (it + 1) % self.restart_freq == 0:
                r = rhs - operator(x)
            self.residual_norm = torch.linalg.norm(r).item()
            rel = self.residual_norm / rhs_norm
            if rel <= self.tol:
                self.iterations = it + 1
                if self.verbose:
                    logger.info("PCG converged in %d iterations, rel_res=%.3e", self.iterations, rel)
                return x
            z = preconditioner(r)
            rz_new = torch.dot(r, z) if one_d else torch.sum(r * z, dim=0)
            beta = rz_new / rz
            if self.autograd_safe:
                p = z + (beta * p if one_d else p * beta.unsqueeze(0))
            else:
                (p.mul_(beta) if one_d else p.mul_(beta.unsqueeze(0))).add_(z)
            rz = rz_new
        self.iterations = max_iter
        if self.verbose:
            logger.warning("PCG did not converge in %d iterations, rel_res=%.3e", max_iter, rel)
        return x
