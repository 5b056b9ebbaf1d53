"""Factored CCCP preconditioner with a fused GPU apply.

Drop-in for laker.preconditioner.CCCPPreconditioner
(laker/preconditioner.py:71-379).  The build follows the reference step by
step on the GPU in the operator's dtype (probes, operator(probes) through the
fused multi-RHS matvec, column normalisation, economy QR, the CCCP fixed point
on N_r x N_r matrices with eigh, final eigh).  After the build the apply
P = c^-1/2 I + Q V diag(lambda^-1/2 - c^-1/2) V^T Q^T is folded into
W = V diag(lambda^-1/2 - c^-1/2) V^T (symmetrised) and applied by the fused
two-pass kernel (laker_precond_apply), which the fused PCG also uses.

Probe draws come from a CPU generator (moved to the device), so a seeded build
matches the CPU float64 oracle; the reference draws on the target device.
"""

from __future__ import annotations

import logging
from typing import Callable, Optional

import torch

from . import _lib
from .backend import get_default_device, get_default_dtype

logger = logging.getLogger(__name__)


def adaptive_shrinkage_rho(num_probes: int, problem_size: int, gamma: float,
                           base_rho: float = 0.05) -> float:
    """Shrinkage rho from the undersampling ratio (laker/utils.py:68-106)."""
    if num_probes >= problem_size:
        return base_rho
    ratio = num_probes / problem_size
    rho = base_rho + (1.0 - base_rho) * (1.0 - ratio) * min(1.0, gamma * 10.0)
    return float(min(rho, 0.5))


def eigh_stable(mat: torch.Tensor, eps: float = 1e-10):
    """eigh with eigenvalues clamped at eps (laker/utils.py:109-134)."""
    w, v = torch.linalg.eigh(mat)
    return w.clamp(min=eps), v


def preconditioner_apply_core(x, isotropic_coef, q_basis, q_eigenvalues, q_eigenvectors):
    """Unfused reference form of the apply (laker/preconditioner.py:52-68)."""
    inv = isotropic_coef ** (-0.5)
    proj = q_basis.T @ x
    coeffs = q_eigenvectors.T @ proj
    scale = q_eigenvalues.rsqrt() - inv
    coeffs = scale * coeffs if x.dim() == 1 else scale.unsqueeze(-1) * coeffs
    return inv * x + q_basis @ (q_eigenvectors @ coeffs)


class CCCPPreconditioner:
    """Learned data-dependent preconditioner P = Sigma^{-1/2} (factored form)."""

    def __init__(
        self,
        num_probes: Optional[int] = None,
        gamma: float = 1e-1,
        epsilon: float = 1e-8,
        base_rho: float = 0.05,
        max_iter: int = 200,
        tol: float = 1e-6,
        verbose: bool = True,
        device: Optional[torch.device] = None,
        dtype: Optional[torch.dtype] = None,
        probe_strategy: str = "gaussian",
        power_iter_steps: int = 3,
    ) -> None:
        self.num_probes = num_probes
        self.gamma = float(gamma)
        self.epsilon = float(epsilon)
        self.base_rho = float(base_rho)
        self.max_iter = int(max_iter)
        self.tol = float(tol)
        self.verbose = verbose
        self.probe_strategy = probe_strategy
        self.power_iter_steps = int(power_iter_steps)
        self.device = torch.device(device) if device is not None else get_default_device()
        self.dtype = dtype if dtype is not None else get_default_dtype()
        self.n: Optional[int] = None
        self.nr: Optional[int] = None
        self.q_basis: Optional[torch.Tensor] = None
        self.qr_r: Optional[torch.Tensor] = None
        self.isotropic_coef: Optional[float] = None
        self.q_basis_matrix: Optional[torch.Tensor] = None
        self.q_eigenvalues: Optional[torch.Tensor] = None
        self.q_eigenvectors: Optional[torch.Tensor] = None
        self.cccp_iterations: int = 0
        self._q32: Optional[torch.Tensor] = None
        self._w32: Optional[torch.Tensor] = None
        self._c: Optional[_lib.laker_precond] = None

    # ------------------------------------------------------------------
    def build(self, operator: Callable[[torch.Tensor], torch.Tensor], n: int,
              seed: Optional[int] = None) -> "CCCPPreconditioner":
        """Learn the preconditioner (laker/preconditioner.py:144-284)."""
        if self.device.type != "cuda":
            raise RuntimeError("CCCPPreconditioner on the B200 path requires a CUDA device")
        dev, dt = self.device, self.dtype
        self.n = n
        nr = self.num_probes if self.num_probes is not None else max(200, int(2 * n**0.5))
        self.nr = min(nr, n)
        if self.nr > 1024:
            raise ValueError(f"num_probes must be <= 1024 for the fused apply, got {self.nr}")
        if self.verbose:
            logger.info("Building CCCP preconditioner: n=%d, N_r=%d", n, self.nr)

        gen = torch.Generator(device="cpu")
        if seed is not None:
            gen.manual_seed(seed)
        # drawn in float64 (as the float64 reference does) and cast to the
        # operator dtype, so a float32 build sees the same directions
        probes = torch.randn(n, self.nr, dtype=torch.float64, generator=gen).to(dev, dt)

        if self.probe_strategy == "power_iter":
            n_power = max(1, int(self.nr * 0.25))
            block = probes[:, :n_power]
            for _ in range(self.power_iter_steps):
                block = operator(block)
                block = torch.linalg.qr(block, mode="reduced")[0]
            probes = torch.cat([block, probes[:, n_power:]], dim=1)

        # operator(probes) through the fused multi-RHS kernel; QR and the
        # N_r x N_r fixed point then run in float64 on the GPU
        op_probes = operator(probes).to(torch.float64)
        dt = torch.float64
        norms = torch.linalg.norm(op_probes, dim=0, keepdim=True)
        normalized = op_probes / norms.clamp(min=self.epsilon)
        q_basis, qr_r = torch.linalg.qr(normalized, mode="reduced")
        self.q_basis, self.qr_r = q_basis, qr_r

        shrinkage = adaptive_shrinkage_rho(self.nr, n, self.gamma, self.base_rho)
        reg_scale = 1.0 + self.gamma / n
        iso = 1.0
        qbm = torch.zeros(self.nr, self.nr, device=dev, dtype=dt)
        eye = torch.eye(self.nr, device=dev, dtype=dt)
        it = 0
        for it in range(self.max_iter):
            iso_prev = iso
            qbm_prev = qbm.clone()
            m_mat = eye * iso + qbm
            evals, evecs = eigh_stable(m_mat, eps=self.epsilon)
            proj = evecs.T @ self.qr_r
            inv_m_r = proj.T @ (evals.reciprocal().unsqueeze(-1) * proj)
            denom = torch.diagonal(inv_m_r) + self.epsilon
            weights = (n / self.nr) / denom
            wrr = (self.qr_r * weights.unsqueeze(0)) @ self.qr_r.T
            f_gamma = (wrr + self.gamma * eye) * (1.0 / reg_scale)
            shrunk = torch.lerp(f_gamma, eye, shrinkage)
            shrunk_iso = (1.0 - shrinkage) * self.gamma / reg_scale + shrinkage
            trace = shrunk_iso * (n - self.nr) + shrunk.diagonal().sum()
            scale = n / trace
            iso = float(scale * shrunk_iso)
            qbm = shrunk * scale
            qbm.diagonal().sub_(iso)
            iso_rel = abs(iso - iso_prev) / (abs(iso_prev) + 1e-12)
            q_rel = (torch.norm(qbm - qbm_prev, p="fro") / (torch.norm(qbm_prev, p="fro") + 1e-12)).item()
            if self.verbose and (it % 10 == 0 or max(iso_rel, q_rel) < self.tol):
                logger.info("CCCP iter %d: isotropic_rel=%.3e, q_basis_rel=%.3e, isotropic_coef=%.6f",
                            it, iso_rel, q_rel, iso)
            if max(iso_rel, q_rel) < self.tol:
                break
        self.cccp_iterations = it + 1
        self.isotropic_coef = iso
        self.q_basis_matrix = qbm
        self.q_eigenvalues, self.q_eigenvectors = eigh_stable(eye * iso + qbm, eps=self.epsilon)
        self._prepare_apply()
        if self.verbose:
            logger.info("CCCP preconditioner built in %d iterations", it + 1)
        return self

    def _prepare_apply(self) -> None:
        v = self.q_eigenvectors.to(torch.float64)
        scale = self.q_eigenvalues.to(torch.float64).rsqrt() - self.isotropic_coef ** (-0.5)
        w = (v * scale.unsqueeze(0)) @ v.T
        w = 0.5 * (w + w.T)
        self._q32 = _lib.padded_q(self.q_basis)
        self._w32 = w.to(torch.float32).contiguous()
        self._c = _lib.precond_struct(self._q32, self._w32, self.n, self.nr,
                                      self.isotropic_coef ** (-0.5))

    def c_precond(self) -> _lib.laker_precond:
        if self._c is None:
            raise RuntimeError("Preconditioner has not been built. Call build() first.")
        return self._c

    # ------------------------------------------------------------------
    def apply(self, x: torch.Tensor) -> torch.Tensor:
        """Apply P to (n,) or (n, k) (laker/preconditioner.py:286-310)."""
        if self.q_basis is None:
            raise RuntimeError("Preconditioner has not been built. Call build() first.")
        if x.dim() == 1:
            return self.apply_1d(x)
        if x.dim() == 2:
            return self.apply_2d(x)
        raise ValueError(f"x must be 1-D or 2-D, got shape {x.shape}")

    def apply_1d(self, x: torch.Tensor) -> torch.Tensor:
        _lib.require_cuda(x, "x")
        return _lib.precond_apply(self.c_precond(), x, x.dtype)

    def apply_2d(self, x: torch.Tensor) -> torch.Tensor:
        _lib.require_cuda(x, "x")
        # k right-hand sides: three plain GEMMs (cuBLAS) with the same folded W
        q = self._q32[:, : self.nr].to(x.dtype)
        w = self._w32.to(x.dtype)
        return (self.isotropic_coef ** (-0.5)) * x + q @ (w @ (q.T @ x))

    def apply_impl(self, x: torch.Tensor) -> torch.Tensor:
        return self.apply(x)

    def to_dense(self) -> torch.Tensor:
        """Dense P = Sigma^{-1/2} (O(n^2); debugging only)."""
        if self.q_basis is None:
            raise RuntimeError("Preconditioner has not been built.")
        n = self.q_basis.shape[0]
        cov = self.isotropic_coef * torch.eye(n, device=self.device, dtype=self.dtype)
        cov = cov + self.q_basis @ self.q_basis_matrix @ self.q_basis.T
        w, v = torch.linalg.eigh(cov)
        w = w.clamp(min=self.epsilon)
        return v @ torch.diag(w.rsqrt()) @ v.T
