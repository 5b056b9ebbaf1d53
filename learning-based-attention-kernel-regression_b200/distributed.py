"""Row-sharded multi-GPU operator and PCG solve, one process per GPU.

Drop-in for laker.distributed_kernels.DistributedAttentionKernelOperator
(laker/distributed_kernels.py:41-339): same constructor arguments
(embeddings, lambda_reg, master_device, dtype), the same attributes
(single_device, devices, chunk_sizes, master_device) and methods (matvec,
diagonal, to_dense, kernel_eval), the same balanced split of the n points
(n // G each, one more for the first n % G shards, distributed_kernels.py:
140-182) and the same single-device fallback.  The reference drives every GPU
from one process and copies the full embeddings and vector to each device per
call; here each GPU runs its own process in a torch.distributed group (NCCL
over NVLink between GPUs, gloo for CPU tests), every rank holds the packed
embeddings once (n x 16 floats: 6.4 MB at n = 100k) and computes the rows
[r0, r1) of a product with the fused rectangular kernel, and the rows travel
by all_gather.  With one rank (no process group, or a group of one) the
operator is the single-GPU operator.

The solver path (`sharded_pcg_solve`, which PreconditionedConjugateGradient
takes for a 1-D right-hand side when the operator is this class on more than
one rank) keeps every vector sharded by rows.  One iteration exchanges:
  * all_gather of p (FP32, n values) before the local rows of A p,
  * one all_reduce of (p.Ap, |p|^2, |Ap|^2) for alpha and the breakdown test,
  * one all_reduce of (Q_loc^T r, |r|^2) for the preconditioner, where Q_loc
    is this rank's rows of the CCCP basis; r.z then follows without another
    exchange as c^-1/2 |r|^2 + s^T W s, s = Q^T r,
and the host reads the four scalars once.  Reliable updates gather x (FP64)
and recompute this rank's rows of b - A x with the FP64 kernel, exactly as
the single-GPU solve does over all rows; the stop test is on that FP64
residual.  Every rank takes the same decisions from the same all-reduced
scalars and returns the full solution.
"""

from __future__ import annotations

import logging
import math
from typing import List, Optional, Tuple

import torch
import torch.distributed as dist

from . import _lib, ops
from .kernels import AttentionKernelOperator
from .preconditioner import CCCPPreconditioner

logger = logging.getLogger(__name__)

BREAKDOWN_MSG = (
    "PCG breakdown: non-positive curvature detected (p^T A p <= 0). "
    "The operator may be indefinite or the preconditioner may be unsuitable."
)
NONFINITE_MSG = "PCG encountered a non-finite inner product (NaN/Inf in the data)"


def shard_bounds(n: int, world: int) -> List[Tuple[int, int]]:
    """Row range of every rank: n // world points each, one more for the first
    n % world ranks (laker/distributed_kernels.py:160-166)."""
    if world < 1:
        raise ValueError(f"world size must be >= 1, got {world}")
    sizes = [n // world + (1 if r < n % world else 0) for r in range(world)]
    bounds, start = [], 0
    for s in sizes:
        bounds.append((start, start + s))
        start += s
    return bounds


class RowExchange:
    """The collectives of the sharded solve over one process group."""

    def __init__(self, n: int, group=None) -> None:
        self.n = int(n)
        self.group = group
        active = dist.is_available() and dist.is_initialized()
        self.world = dist.get_world_size(group) if active else 1
        self.rank = dist.get_rank(group) if active else 0
        self.bounds = shard_bounds(self.n, self.world)
        self.r0, self.r1 = self.bounds[self.rank]
        self.rows = self.r1 - self.r0
        self.chunk = max(e - s for s, e in self.bounds)
        self.nccl = self.world > 1 and dist.get_backend(group) == "nccl"

    def sum_(self, t: torch.Tensor) -> torch.Tensor:
        """In-place sum over the ranks (every rank gets the same values)."""
        if self.world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t

    def gather(self, v: torch.Tensor) -> torch.Tensor:
        """The full (n, ...) tensor from every rank's rows (rows, ...)."""
        if v.shape[0] != self.rows:
            raise ValueError(f"rank {self.rank} holds {self.rows} rows, got {v.shape[0]}")
        if self.world == 1:
            return v.contiguous()
        tail = tuple(v.shape[1:])
        if self.nccl:
            # all_gather_into_tensor wants equal pieces: pad every shard to the
            # largest (ceil(n / world) rows) and drop the padding afterwards
            piece = v.new_zeros((self.chunk,) + tail)
            piece[: self.rows] = v
            out = v.new_empty((self.world * self.chunk,) + tail)
            dist.all_gather_into_tensor(out, piece, group=self.group)
            if self.chunk * self.world == self.n:
                return out
            return torch.cat([out[r * self.chunk: r * self.chunk + (e - s)]
                              for r, (s, e) in enumerate(self.bounds)])
        # gloo (CPU tensors, and CUDA tensors where it has no all_gather): a
        # sum of zero-padded copies, exact since every row has one owner
        full = v.new_zeros((self.n,) + tail)
        full[self.r0: self.r1] = v
        dist.all_reduce(full, op=dist.ReduceOp.SUM, group=self.group)
        return full


class RowShard:
    """Rows [r0, r1) of A = lambda I + exp(E E^T) on this rank's GPU: its own
    packed row embeddings against the operator's packed full embeddings, on
    the fused rectangular kernels (the whole square operator when the shard
    holds every row)."""

    def __init__(self, op: AttentionKernelOperator, r0: int, r1: int) -> None:
        self.n, self.d = op.n, op.embedding_dim
        self.lam = op.lambda_reg
        self.clamp = 0 if op.skip_clamp else 1
        self.r0, self.r1, self.rows = r0, r1, r1 - r0
        self.cols32, self.cols64 = op.packed.packed32, op.packed.packed64
        if r0 == 0 and r1 == self.n:
            self.rows32, self.rows64 = self.cols32, self.cols64
        elif self.rows > 0:
            E = op.embeddings.detach()[r0:r1]
            self.rows32, self.rows64 = ops.pack(E, 32), ops.pack(E, 64)

    def _local(self, full: torch.Tensor) -> torch.Tensor:
        return full[self.r0: self.r1]

    def apply32(self, xf: torch.Tensor, lam: float) -> torch.Tensor:
        """(A x)[r0:r1] with the FP32 kernel, lam * x added in FP32."""
        if self.rows == 0:
            return xf.new_zeros((0,) + tuple(xf.shape[1:]), dtype=torch.float32)
        xf = xf.to(torch.float32).contiguous()
        y = ops.attn_matvec(self.rows32, self.rows, self.cols32, self.n, self.d, 0.0,
                            bool(self.clamp), xf)
        return y.add_(self._local(xf), alpha=lam) if lam != 0.0 else y

    def apply64(self, xf: torch.Tensor, lam: float) -> torch.Tensor:
        """(A x)[r0:r1] with the FP64 kernel."""
        if self.rows == 0:
            return xf.new_zeros((0,) + tuple(xf.shape[1:]), dtype=torch.float64)
        xf = xf.to(torch.float64).contiguous()
        y = ops.attn_matvec(self.rows64, self.rows, self.cols64, self.n, self.d, 0.0,
                            bool(self.clamp), xf)
        return y.add_(self._local(xf), alpha=lam) if lam != 0.0 else y

    def residual64(self, xf: torch.Tensor, b_loc: torch.Tensor) -> torch.Tensor:
        """(b - A x)[r0:r1] with the FP64 kernel (b_loc: this shard's rows)."""
        if self.rows == 0:
            return b_loc.to(torch.float64).clone()
        xf = xf.to(torch.float64).contiguous()
        r = ops.attn_residual(self.rows64, self.rows, self.cols64, self.n, self.d, 0.0,
                              bool(self.clamp), xf, b_loc)
        return r.sub_(self._local(xf), alpha=self.lam)


class ShardedPreconditioner:
    """This rank's rows of the factored CCCP apply P = c^-1/2 I + Q W Q^T
    (laker/preconditioner.py:52-68 with W = V diag(l^-1/2 - c^-1/2) V^T
    folded): Q_loc (rows x nr), W (nr x nr), c^-1/2, held in FP64 but with Q
    and W taken from the fused apply's FP32 factors (apply_factors()), so the
    sharded apply carries the same FP32 rounding of Q and W as the
    single-GPU apply."""

    def __init__(self, q_loc: torch.Tensor, w: torch.Tensor, inv_sqrt_iso: float) -> None:
        self.q = q_loc.to(torch.float64).contiguous()
        self.w = w.to(torch.float64).contiguous()
        self.cis = float(inv_sqrt_iso)
        self.nr = int(self.w.shape[0])

    @classmethod
    def from_cccp(cls, pc: CCCPPreconditioner, r0: int, r1: int) -> "ShardedPreconditioner":
        _, w32, _, cis = pc.apply_factors()  # raises before the first build
        return cls(pc.q_basis[r0:r1], w32, cis)


def _precondition(r: torch.Tensor, pre: Optional[ShardedPreconditioner], exch: RowExchange):
    """z = P r on this shard, with r.z and |r|^2 summed over the ranks in one
    all_reduce (device tensors; nothing is read on the host)."""
    rr_loc = torch.dot(r, r).reshape(1)
    if pre is None:
        rr = exch.sum_(rr_loc)[0]
        return r, rr, rr
    buf = exch.sum_(torch.cat([pre.q.T @ r, rr_loc]))
    s, rr = buf[: pre.nr], buf[pre.nr]
    ws = pre.w @ s
    z = torch.addmv(r * pre.cis, pre.q, ws)
    rz = pre.cis * rr + torch.dot(s, ws)
    return z, rz, rr


class ShardedSolveInfo:
    """What a sharded solve reports (the fields of laker_pcg_result it shares)."""

    def __init__(self) -> None:
        self.status = _lib.LAKER_ERR_NOT_CONVERGED
        self.iterations = 0
        self.accurate_matvecs = 0
        self.residual_norm = float("inf")
        self.rhs_norm = 0.0
        self.recurrence_norm = float("inf")


def sharded_pcg_solve(shard, exch: RowExchange, b: torch.Tensor, *,
                      precond: Optional[ShardedPreconditioner] = None,
                      x0: Optional[torch.Tensor] = None, tol: float = 1e-10,
                      max_iter: Optional[int] = None, reliable_delta: float = 0.03,
                      breakdown_eps: Optional[float] = None,
                      info: Optional[ShardedSolveInfo] = None,
                      ) -> Tuple[torch.Tensor, ShardedSolveInfo]:
    """Row-sharded mixed-precision PCG for one right-hand side.

    `shard` gives this rank's rows of the operator: apply32(x_full, lam) (FP32
    operator, the recurrence), residual64(x_full, b_loc) (FP64, the reliable
    update) and `lam`.  b (n,) is the full right-hand side on every rank, x0
    the full initial guess.  The recurrence is the reference's solve_1d
    (laker/solvers.py:189-295: alpha = r.z / p.Ap, beta = r.z new / old,
    breakdown when p.Ap <= -eps |p| |Ap|, at least one iteration) with the
    single-GPU fused solve's reliable updates.  Returns the full x (FP64) on
    every rank and the solve's report (filled into `info` when given, so a
    caller still has it after an exception); raises RuntimeError on breakdown
    or non-finite values, on every rank alike.
    """
    n = b.shape[0]
    if n != exch.n:
        raise ValueError(f"rhs has {n} rows, the exchange was set up for {exch.n}")
    max_iter = n if max_iter is None else int(max_iter)
    eps = math.sqrt(torch.finfo(torch.float64).eps) if breakdown_eps is None else breakdown_eps
    info = ShardedSolveInfo() if info is None else info
    b_loc = b[exch.r0: exch.r1].to(torch.float64)
    bn = math.sqrt(exch.sum_(torch.dot(b_loc, b_loc).reshape(1)).item())
    info.rhs_norm = bn
    if not math.isfinite(bn):
        info.status = _lib.LAKER_ERR_NONFINITE
        raise RuntimeError(NONFINITE_MSG)
    if bn == 0.0:
        info.status, info.residual_norm = _lib.LAKER_OK, 0.0
        return torch.zeros(n, dtype=torch.float64, device=b.device), info
    if x0 is not None:
        x0f = x0.to(device=b.device, dtype=torch.float64)
        x = x0f[exch.r0: exch.r1].clone()
        r = shard.residual64(x0f, b_loc)
        info.accurate_matvecs = 1
    else:
        x = torch.zeros_like(b_loc)
        r = b_loc.clone()
    z, rz, rr = _precondition(r, precond, exch)
    p = z.clone()
    rn = rmax = math.sqrt(rr.item())
    lam = shard.lam
    it = 0
    for it in range(1, max_iter + 1):
        pf = exch.gather(p.to(torch.float32))
        q = shard.apply32(pf, 0.0).to(torch.float64).add_(p, alpha=lam)
        red = exch.sum_(torch.stack([torch.dot(p, q), torch.dot(p, p), torch.dot(q, q)]))
        alpha = rz / red[0]
        x.add_(alpha * p)
        r.sub_(alpha * q)
        z, rz_new, rr = _precondition(r, precond, exch)
        pap, pp, qq, rr_h = torch.stack([red[0], red[1], red[2], rr]).tolist()
        if not all(math.isfinite(v) for v in (pap, pp, qq, rr_h)):
            info.status, info.iterations = _lib.LAKER_ERR_NONFINITE, it
            raise RuntimeError(NONFINITE_MSG)
        if pap <= -eps * math.sqrt(pp * qq):
            info.status, info.iterations = _lib.LAKER_ERR_BREAKDOWN, it
            raise RuntimeError(BREAKDOWN_MSG)
        rn = math.sqrt(rr_h)
        info.recurrence_norm = rn
        rmax = max(rmax, rn)
        if rn <= reliable_delta * rmax or rn <= tol * bn or it == max_iter:
            r = shard.residual64(exch.gather(x), b_loc)
            info.accurate_matvecs += 1
            z, rz_new, rr = _precondition(r, precond, exch)
            rn = math.sqrt(rr.item())
            rmax = rn
            if rn <= tol * bn:
                info.status = _lib.LAKER_OK
                break
        p = z + (rz_new / rz) * p
        rz = rz_new
    info.iterations = it
    info.residual_norm = rn
    return exch.gather(x), info


class DistributedAttentionKernelOperator(AttentionKernelOperator):
    """A = lambda I + exp(E E^T) row-sharded over the ranks of a process group.

    Every rank constructs it with the same full embeddings and calls every
    method collectively (matvec and the solves exchange rows); results are the
    full tensors on every rank.  Products go through this rank's RowShard and
    an all_gather, including under autograd (the backward's products are the
    same sharded products).  diagonal, to_dense and kernel_eval are computed
    on each rank from its replicated embeddings.

    Args:
        embeddings: full (n, d) embeddings on this rank's CUDA device.
        lambda_reg: Tikhonov regularisation lambda.
        master_device: device of inputs and outputs (default: the embeddings').
        dtype: operator dtype (default: the embeddings').
        group: torch.distributed process group (default: the world group).
    """

    def __init__(self, embeddings: torch.Tensor, lambda_reg: float = 1e-2,
                 master_device: Optional[torch.device] = None,
                 dtype: Optional[torch.dtype] = None, group=None) -> None:
        super().__init__(embeddings, lambda_reg=lambda_reg, chunk_size=None,
                         device=master_device, dtype=dtype)
        self.master_device = self.device
        self.group = group
        self.exchange = RowExchange(self.n, group)
        self.world_size, self.rank = self.exchange.world, self.exchange.rank
        self.single_device = self.world_size == 1
        self.chunk_sizes = [e - s for s, e in self.exchange.bounds]
        if self.single_device:
            self.devices = [self.device]
            self.local_op = self
        else:
            names: list = [None] * self.world_size
            dist.all_gather_object(names, str(self.device), group=group)
            self.devices = [torch.device(s) for s in names]
        self.shard = RowShard(self, self.exchange.r0, self.exchange.r1)

    def shard_embeddings(self, embeddings: torch.Tensor) -> None:
        """Re-shard new embeddings of the same shape (distributed_kernels.py:140-182)."""
        if tuple(embeddings.shape) != (self.n, self.embedding_dim):
            raise ValueError(f"expected embeddings of shape {(self.n, self.embedding_dim)}, "
                             f"got {tuple(embeddings.shape)}")
        self.__init__(embeddings, self.lambda_reg, self.master_device, self.dtype, self.group)

    def _apply(self, x: torch.Tensor, lam: float) -> torch.Tensor:
        if self.single_device:
            return super()._apply(x, lam)
        x = x.detach()
        if self.dtype == torch.float64:
            y = self.shard.apply64(x, lam)
        else:
            y = self.shard.apply32(x, lam)
        y = self.exchange.gather(y)
        return y.to(x.dtype) if x.dtype in (torch.float32, torch.float64) else y

    def matvec_f64(self, x: torch.Tensor) -> torch.Tensor:
        if self.single_device:
            return super().matvec_f64(x)
        _lib.require_cuda(x, "x")
        return self.exchange.gather(self.shard.apply64(x, self.lambda_reg))

    def residual_f64(self, x: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        if self.single_device:
            return super().residual_f64(x, b)
        _lib.require_cuda(x, "x")
        e = self.exchange
        return e.gather(self.shard.residual64(x, b.to(torch.float64)[e.r0: e.r1]))
