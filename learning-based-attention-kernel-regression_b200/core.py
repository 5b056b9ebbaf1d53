"""LAKERCore: the solve / predict / variance pipeline on the B200 kernels.

Mirrors the hot-path methods of laker.core.LAKERCore (laker/core.py:77-777):
compute_embeddings, build_kernel_operator, build_preconditioner, solve_pcg,
predict and predict_variance, with the same constructor.  The exact kernel
operator, the fused PCG and the fused preconditioner apply replace the torch
op chains.  Approximate kernels, the multi-device operator and the adaptive
preconditioner are outside this path and raise NotImplementedError.

Precision contract: alpha is solved and kept in float64 whatever `dtype` is
(its norm is ~90x ||y|| on the standard field, so rounding it to float32 would
cost ~1e-3 relative prediction error); predictions and variances use the FP64
fused kernels and are returned in `dtype`.
"""

from __future__ import annotations

import logging
from typing import Optional, Tuple, Union

import torch
import torch.nn as nn

from . import _lib, ops
from .backend import get_default_device, get_default_dtype
from .embeddings import PositionEmbedding
from .distributed import DistributedAttentionKernelOperator
from .kernels import AttentionKernelOperator, KernelOperator
from .preconditioner import CCCPPreconditioner
from .solvers import PreconditionedConjugateGradient

logger = logging.getLogger(__name__)

# Largest number of query columns solved in one batched-RHS PCG.
VARIANCE_BLOCK = 1024


class LAKERCore:
    """Pipeline root (laker/core.py:77-245)."""

    def __init__(
        self,
        embedding_dim: int = 10,
        lambda_reg: float = 1e-2,
        gamma: float = 1e-1,
        num_probes: Optional[int] = None,
        epsilon: float = 1e-8,
        base_rho: float = 0.05,
        cccp_max_iter: int = 200,
        cccp_tol: float = 1e-6,
        pcg_tol: float = 1e-6,
        pcg_max_iter: int = 1000,
        chunk_size: Optional[int] = None,
        embedding_module: Optional[nn.Module] = None,
        kernel_approx: Optional[str] = None,
        num_landmarks: Optional[int] = None,
        num_features: Optional[int] = None,
        k_neighbors: Optional[int] = None,
        grid_size: Optional[int] = None,
        distributed: bool = False,
        twoscale_alpha: float = 0.5,
        landmark_method: str = "greedy",
        landmark_pilot_size: int = 1000,
        spectral_knots: int = 5,
        preconditioner_strategy: str = "cccp",
        embedding_dtype: Optional[torch.dtype] = None,
        device: Optional[Union[str, torch.device]] = None,
        dtype: Optional[torch.dtype] = None,
        verbose: bool = True,
    ) -> None:
        self.embedding_dim = embedding_dim
        self.lambda_reg = lambda_reg
        self.gamma = gamma
        self.num_probes = num_probes
        self.epsilon = epsilon
        self.base_rho = base_rho
        self.cccp_max_iter = cccp_max_iter
        self.cccp_tol = cccp_tol
        self.pcg_tol = pcg_tol
        self.pcg_max_iter = pcg_max_iter
        self.chunk_size = chunk_size
        self.embedding_module = embedding_module
        self.kernel_approx = kernel_approx
        self.num_landmarks = num_landmarks
        self.num_features = num_features
        self.k_neighbors = k_neighbors
        self.grid_size = grid_size
        self.distributed = distributed
        self.twoscale_alpha = twoscale_alpha
        self.landmark_method = landmark_method
        self.landmark_pilot_size = landmark_pilot_size
        self.spectral_knots = spectral_knots
        self.preconditioner_strategy = preconditioner_strategy
        self.verbose = verbose
        if device is None:
            device = get_default_device()
        elif isinstance(device, str):
            device = torch.device(device)
        if dtype is None:
            dtype = get_default_dtype()
        self.device = device
        self.dtype = dtype
        self.embedding_dtype = embedding_dtype if embedding_dtype is not None else dtype
        self.last_pcg: Optional[PreconditionedConjugateGradient] = None

    # ------------------------------------------------------------------
    def compute_embeddings(
        self, x: torch.Tensor, embedding_model: Optional[nn.Module] = None
    ) -> Tuple[torch.Tensor, nn.Module]:
        """Spatial locations -> embeddings (laker/core.py:247-305)."""
        n, input_dim = x.shape[0], x.shape[1]
        if self.verbose:
            logger.info("Fitting LAKER on n=%d, dx=%d", n, input_dim)
        embedded_input = x.to(dtype=self.embedding_dtype)
        if self.embedding_module is not None:
            model = self.embedding_module.to(self.device)
        elif embedding_model is None:
            model = PositionEmbedding(input_dim=input_dim, embedding_dim=self.embedding_dim,
                                      device=self.device, dtype=self.embedding_dtype)
        else:
            model = embedding_model
        with torch.no_grad():
            embeddings = model(embedded_input)
        if self.embedding_dtype != self.dtype:
            embeddings = embeddings.to(dtype=self.dtype)
        return embeddings, model

    def build_kernel_operator(
        self, embeddings: torch.Tensor, lambda_reg: Optional[float] = None,
        chunk_size: Optional[int] = None,
    ) -> KernelOperator:
        """Exact attention-kernel operator (laker/core.py:307-367)."""
        if self.kernel_approx is not None:
            raise NotImplementedError(
                f"kernel_approx={self.kernel_approx!r} is outside the B200 exact-kernel path"
            )
        lam = float(lambda_reg) if lambda_reg is not None else self.lambda_reg
        if self.distributed:
            # rows sharded over the ranks of the default process group (one
            # process per GPU); a single device when there is no group
            op = DistributedAttentionKernelOperator(embeddings=embeddings, lambda_reg=lam,
                                                    master_device=self.device, dtype=self.dtype)
            if self.verbose:
                logger.info("Using distributed kernel on %d device(s)", len(op.devices))
            return op
        n = embeddings.shape[0]
        chunk = chunk_size
        if chunk is None and n > 5000:
            chunk = max(1024, min(n // 10, 8192))
        return AttentionKernelOperator(embeddings=embeddings, lambda_reg=lam, chunk_size=chunk,
                                       device=self.device, dtype=self.dtype)

    def build_preconditioner(
        self, matvec, n: int, gamma: Optional[float] = None, num_probes: Optional[int] = None,
        seed: Optional[int] = None, diagonal: Optional[torch.Tensor] = None,
    ) -> CCCPPreconditioner:
        """CCCP preconditioner (laker/core.py:461-521)."""
        del diagonal  # used only by the adaptive strategy
        if self.preconditioner_strategy != "cccp":
            raise NotImplementedError(
                f"preconditioner={self.preconditioner_strategy!r} is outside the B200 path"
            )
        pre = CCCPPreconditioner(
            num_probes=num_probes if num_probes is not None else self.num_probes,
            gamma=gamma if gamma is not None else self.gamma,
            epsilon=self.epsilon,
            base_rho=self.base_rho,
            max_iter=self.cccp_max_iter,
            tol=self.cccp_tol,
            verbose=self.verbose,
            device=self.device,
            dtype=self.dtype,
        )
        pre.build(matvec, n, seed=seed)
        return pre

    def solve_pcg(
        self, kernel_operator: KernelOperator, preconditioner: CCCPPreconditioner,
        rhs: torch.Tensor, x0: Optional[torch.Tensor] = None,
    ) -> Tuple[torch.Tensor, int]:
        """Solve (lambda I + G) alpha = rhs (laker/core.py:526-575); alpha in float64."""
        pcg = PreconditionedConjugateGradient(tol=self.pcg_tol, max_iter=self.pcg_max_iter,
                                              verbose=self.verbose)
        alpha = pcg.solve(kernel_operator.matvec, preconditioner.apply, rhs.to(torch.float64),
                          x0=x0)
        self.last_pcg = pcg
        if self.verbose:
            logger.info("LAKER fit complete: PCG iters=%d, final rel_res=%.3e", pcg.iterations,
                        pcg.residual_norm / max(torch.linalg.norm(rhs).item(), 1e-300))
        return alpha, pcg.iterations

    # ------------------------------------------------------------------
    def _query_embeddings(self, x: torch.Tensor, embedding_model: nn.Module) -> torch.Tensor:
        with torch.no_grad():
            q = embedding_model(x.to(dtype=self.embedding_dtype))
        return q.to(dtype=self.dtype)

    def predict(
        self, x: torch.Tensor, embedding_model: nn.Module, embeddings: torch.Tensor,
        kernel_operator: AttentionKernelOperator, alpha: torch.Tensor,
        residual_corrector: Optional[nn.Module] = None,
    ) -> torch.Tensor:
        """f(x*) = exp(E_q E^T) alpha with the FP64 fused kernel (laker/core.py:580-661)."""
        q = self._query_embeddings(x, embedding_model)
        _lib.require_cuda(q, "query embeddings")
        m = q.shape[0]
        op = kernel_operator
        clamp = 0
        if not op.skip_clamp or (m and torch.sum(q.double() ** 2, dim=1).max().item() >= 700.0):
            clamp = 1
        q64 = ops.pack(q, 64)
        out = ops.attn_matvec(q64, m, op.packed.packed64, op.n, op.embedding_dim, 0.0, bool(clamp),
                              alpha)
        _lib.raise_device_status(out.device)
        out = out.to(self.dtype)
        if residual_corrector is not None:
            residual_corrector.eval()
            with torch.no_grad():
                out = out + residual_corrector(x).squeeze()
        return out

    def predict_variance(
        self, x: torch.Tensor, embedding_model: nn.Module, embeddings: torch.Tensor,
        kernel_operator: AttentionKernelOperator, preconditioner: CCCPPreconditioner,
        alpha: torch.Tensor, lambda_reg: float,
    ) -> torch.Tensor:
        """sigma^2(x) = k(x,x) - k(x,X)^T A^{-1} k(x,X) (laker/core.py:666-777)."""
        del alpha, lambda_reg, embeddings
        q = self._query_embeddings(x, embedding_model)
        _lib.require_cuda(q, "query embeddings")
        op = kernel_operator
        m, d = q.shape
        var = torch.empty(m, dtype=torch.float64, device=q.device)
        pcg = PreconditionedConjugateGradient(tol=self.pcg_tol, max_iter=self.pcg_max_iter,
                                              verbose=False)
        for start in range(0, m, VARIANCE_BLOCK):
            end = min(start + VARIANCE_BLOCK, m)
            qb = q[start:end]
            q64 = ops.pack(qb, 64)
            kxq = ops.kernel_eval(op.packed.packed64, op.n, q64, end - start, d, not op.skip_clamp,
                                  True)
            v = pcg.solve(op.matvec, preconditioner.apply, kxq)
            var[start:end] = ops.variance_finalize(q64, end - start, d, kxq, v)
        _lib.raise_device_status(var.device)
        self.last_pcg = pcg
        return var.to(self.dtype)
