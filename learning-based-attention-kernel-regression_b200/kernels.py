"""Exact attention-kernel operator on the B200 kernels.

Drop-in for laker.kernels.AttentionKernelOperator (laker/kernels.py:133-354):
same constructor, attributes (n, embedding_dim, lambda_reg, chunk_size,
device, dtype, embeddings, shape, skip_clamp) and methods (matvec, diagonal,
to_dense, kernel_eval).  The operator is applied by fused CUDA kernels that
never store the n x n kernel: float32 operators use the FP32 flash-style
matvec, float64 operators the FP64 one.  `chunk_size` is accepted and kept for
API compatibility; the fused kernels tile on chip and need no memory budget.
"""

from __future__ import annotations

import logging
from typing import Optional, Protocol, Tuple

import torch

from . import _lib, ops

logger = logging.getLogger(__name__)

MAX_EMBEDDING_DIM = 16


class KernelOperator(Protocol):
    """Protocol for matrix-free kernel operators (laker/kernels.py:43-72)."""

    n: int
    embedding_dim: int
    lambda_reg: float
    dtype: torch.dtype
    device: torch.device
    shape: Tuple[int, int]

    def matvec(self, x: torch.Tensor) -> torch.Tensor: ...

    def diagonal(self) -> torch.Tensor: ...

    def to_dense(self) -> torch.Tensor: ...

    def kernel_eval(
        self, x: torch.Tensor, y: Optional[torch.Tensor] = None, chunk_size: Optional[int] = None
    ) -> torch.Tensor: ...


def _safe_limit(dtype: torch.dtype) -> float:
    # exp_safe clamp level (laker/kernels.py:98-99)
    return 80.0 if dtype == torch.float32 else 700.0


class PackedEmbeddings:
    """Device copies of an embedding matrix in the two kernel layouts."""

    def __init__(self, E: torch.Tensor) -> None:
        _lib.require_cuda(E, "embeddings")
        if E.dim() != 2:
            raise ValueError(f"embeddings must be 2-D, got shape {tuple(E.shape)}")
        if not 1 <= E.shape[1] <= MAX_EMBEDDING_DIM:
            raise ValueError(
                f"embedding_dim must be in [1, {MAX_EMBEDDING_DIM}] for the fused kernels, "
                f"got {E.shape[1]}"
            )
        self.n, self.d = int(E.shape[0]), int(E.shape[1])
        self.packed32 = ops.pack(E.detach(), 32)
        self.packed64 = ops.pack(E.detach(), 64)


class _AttnMatvec(torch.autograd.Function):
    """y = (lambda I + G) x with G = exp(E E^T), differentiable in E and x.

    For a loss with upstream gradient Y' (same shape as y):
      dL/dx = (lambda I + G) Y'                        (G is symmetric)
      dL/de_i = sum_c [ Y'_ic (G (x_c * E))_i + x_ic (G (Y'_c * E))_i ]
    (d/de_i of exp(e_i . e_j) = exp(e_i . e_j) e_j, and e_i appears in row i
    and column i).  The E gradient is one multi-RHS product of G with the 2 k d
    columns x_c * E and Y'_c * E -- the fused multi-RHS kernel, in chunks.
    Entries clamped before exp (operators that do not skip the clamp) have
    zero derivative, which this backward does not mask: it raises instead."""

    @staticmethod
    def forward(ctx, E, x, op):  # noqa: D401
        ctx.op = op
        ctx.save_for_backward(x)
        return op._apply(x, op.lambda_reg)

    @staticmethod
    def backward(ctx, gy):
        op = ctx.op
        (x,) = ctx.saved_tensors
        gE = gx = None
        if ctx.needs_input_grad[1]:
            gx = op._apply(gy, op.lambda_reg).to(x.dtype)
        if ctx.needs_input_grad[0]:
            if not op.skip_clamp:
                raise NotImplementedError(
                    "embedding gradient of a clamped attention kernel is not implemented")
            E = op.embeddings.detach()
            X2 = x.detach().reshape(op.n, -1).to(op.dtype)
            G2 = gy.detach().reshape(op.n, -1).to(op.dtype)
            d = op.embedding_dim
            gE = torch.zeros_like(E)
            cols_per_chunk = max(1, 256 // (2 * d))  # right-hand sides per product
            for c0 in range(0, X2.shape[1], cols_per_chunk):
                c1 = min(c0 + cols_per_chunk, X2.shape[1])
                xs, gs = X2[:, c0:c1], G2[:, c0:c1]  # (n, c)
                R = torch.cat([(xs.unsqueeze(2) * E.unsqueeze(1)).reshape(op.n, -1),
                               (gs.unsqueeze(2) * E.unsqueeze(1)).reshape(op.n, -1)], dim=1)
                KR = op._apply(R.contiguous(), 0.0).reshape(op.n, 2, c1 - c0, d)
                gE += (gs.unsqueeze(2) * KR[:, 0]).sum(dim=1) + (xs.unsqueeze(2) * KR[:, 1]).sum(dim=1)
            gE = gE.to(op.embeddings.dtype)
        return gE, gx, None


class AttentionKernelOperator:
    """Matrix-free operator A = lambda*I + exp(E E^T) on the GPU.

    Args:
        embeddings: (n, embedding_dim) tensor on a CUDA device, embedding_dim <= 16.
        lambda_reg: Tikhonov regularisation lambda.
        chunk_size: accepted for compatibility (unused by the fused kernels).
        device / dtype: default to the embeddings' own.

    Raises:
        ValueError: if embeddings is not 2-D.
        RuntimeError: if the device is not CUDA.
    """

    def __init__(
        self,
        embeddings: torch.Tensor,
        lambda_reg: float = 1e-2,
        chunk_size: Optional[int] = None,
        device: Optional[torch.device] = None,
        dtype: Optional[torch.dtype] = None,
    ) -> None:
        if embeddings.dim() != 2:
            raise ValueError(f"embeddings must be 2-D, got shape {embeddings.shape}")
        self.n = embeddings.shape[0]
        self.embedding_dim = embeddings.shape[1]
        self.lambda_reg = float(lambda_reg)
        self.chunk_size = chunk_size
        if device is None:
            device = embeddings.device
        if dtype is None:
            dtype = embeddings.dtype
        self.device = torch.device(device)
        self.dtype = dtype
        self.embeddings = embeddings.to(device=self.device, dtype=dtype)
        _lib.require_cuda(self.embeddings, "embeddings")
        self.shape = (self.n, self.n)
        self._packed = PackedEmbeddings(self.embeddings)
        max_sq_norm = torch.sum(self.embeddings.detach() ** 2, dim=1).max().item() if self.n else 0.0
        self.skip_clamp = max_sq_norm < _safe_limit(self.dtype)

    # -- device-level handles used by the fused solver ---------------------
    @property
    def packed(self) -> PackedEmbeddings:
        return self._packed

    def c_operator(self) -> _lib.laker_operator:
        return _lib.laker_operator(
            self._packed.packed32.data_ptr(),
            self._packed.packed64.data_ptr(),
            self.n,
            self.embedding_dim,
            self.lambda_reg,
            0 if self.skip_clamp else 1,
        )

    # -- KernelOperator protocol ---------------------------------------------
    def matvec(self, x: torch.Tensor) -> torch.Tensor:
        """Apply (lambda I + G) to x of shape (n,) or (n, k).

        Differentiable (laker/kernels.py:209-270 runs under autograd in the
        reference's training code): with grad enabled and the embeddings or x
        requiring grad, the product goes through _AttnMatvec, whose backward
        runs on the same fused kernels."""
        if x.dim() not in (1, 2):
            raise ValueError(f"x must be 1-D or 2-D, got shape {x.shape}")
        if x.shape[0] != self.n:
            raise ValueError(f"x has {x.shape[0]} rows, operator has n={self.n}")
        _lib.require_cuda(x, "x")
        if self.n == 0:
            return torch.zeros_like(x)
        if torch.is_grad_enabled() and (self.embeddings.requires_grad or x.requires_grad):
            return _AttnMatvec.apply(self.embeddings, x, self)
        return self._apply(x, self.lambda_reg)

    def _apply(self, x: torch.Tensor, lam: float) -> torch.Tensor:
        """(lam I + G) x on the fused kernels (no autograd)."""
        p = self._packed
        x = x.detach()
        packed = p.packed64 if self.dtype == torch.float64 else p.packed32
        y = ops.attn_matvec(packed, self.n, packed, self.n, self.embedding_dim, lam,
                            not self.skip_clamp, x)
        return y.to(x.dtype) if x.dtype in (torch.float32, torch.float64) else y

    def matvec_f64(self, x: torch.Tensor) -> torch.Tensor:
        """FP64 (accurate) application regardless of the operator dtype."""
        _lib.require_cuda(x, "x")
        p = self._packed
        return ops.attn_matvec(p.packed64, self.n, p.packed64, self.n, self.embedding_dim,
                               self.lambda_reg, not self.skip_clamp, x)

    def residual_f64(self, x: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        """b - A x with the FP64 operator."""
        _lib.require_cuda(x, "x")
        p = self._packed
        return ops.attn_residual(p.packed64, self.n, p.packed64, self.n, self.embedding_dim,
                                 self.lambda_reg, not self.skip_clamp, x, b)

    def diagonal(self) -> torch.Tensor:
        """diag(lambda I + G) = lambda + exp(||e_i||^2)."""
        d = ops.attn_diagonal(self._packed.packed64, self.n, self.embedding_dim, self.lambda_reg)
        return d.to(self.dtype)

    def to_dense(self) -> torch.Tensor:
        """Materialise lambda I + G (O(n^2) memory: small n only)."""
        p = self._packed
        g = ops.kernel_eval(p.packed64, self.n, p.packed64, self.n, self.embedding_dim, False,
                            self.dtype == torch.float64)
        g.diagonal().add_(self.lambda_reg)
        return g

    def kernel_eval(
        self, x: torch.Tensor, y: Optional[torch.Tensor] = None, chunk_size: Optional[int] = None
    ) -> torch.Tensor:
        """exp(x y^T) for x (m, d) and y (p, d) (y defaults to the embeddings)."""
        del chunk_size  # the kernel tiles on chip
        if x.dim() != 2:
            raise ValueError(f"x must be 2-D, got shape {x.shape}")
        _lib.require_cuda(x, "x")
        if y is None:
            cols64, p = self._packed.packed64, self.n
        else:
            if y.dim() != 2 or y.shape[1] != x.shape[1]:
                raise ValueError(f"y must be 2-D with {x.shape[1]} columns, got {tuple(y.shape)}")
            _lib.require_cuda(y, "y")
            cols64, p = ops.pack(y.to(self.dtype), 64), y.shape[0]
        rows64 = ops.pack(x.to(self.dtype), 64)
        return ops.kernel_eval(rows64, x.shape[0], cols64, p, x.shape[1], not self.skip_clamp,
                               self.dtype == torch.float64)
