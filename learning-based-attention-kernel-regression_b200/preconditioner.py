"""Factored CCCP preconditioner with a fused GPU apply.

Drop-in for laker.preconditioner.CCCPPreconditioner
(laker/preconditioner.py:71-379).  The build follows the reference step by
step on the GPU in the operator's dtype (probes, operator(probes) through the
fused multi-RHS matvec, column normalisation, economy QR, the CCCP fixed point
on N_r x N_r matrices with eigh, final eigh).  After the build the apply
P = c^-1/2 I + Q V diag(lambda^-1/2 - c^-1/2) V^T Q^T is folded into
W = V diag(lambda^-1/2 - c^-1/2) V^T (symmetrised) and applied by the fused
two-pass kernel (laker_precond_apply), which the fused PCG also uses.

Probes are drawn as the reference draws them (laker/preconditioner.py:168-171):
torch.randn in the preconditioner's dtype from a generator on its device, so a
seeded build on a CUDA device sees the probes the reference sees on that
device.  probe_device="cpu" draws from a CPU generator instead, which
reproduces a reference build run on the CPU (the float64 goldens).
"""

from __future__ import annotations

import logging
import time
from typing import Callable, Optional

import torch

from . import _lib, ops
from .backend import get_default_device, get_default_dtype

logger = logging.getLogger(__name__)


class PhaseClock:
    """Accumulates synchronised wall time per phase into a dict (or nothing)."""

    def __init__(self, out: Optional[dict], device: torch.device) -> None:
        self.out, self.device, self.t = out, device, 0.0

    def start(self) -> None:
        if self.out is not None:
            torch.cuda.synchronize(self.device)
            self.t = time.perf_counter()

    def stop(self, phase: str) -> None:
        if self.out is not None:
            torch.cuda.synchronize(self.device)
            now = time.perf_counter()
            self.out[phase] = self.out.get(phase, 0.0) + now - self.t
            self.t = now


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


def draw_probes(n: int, nr: int, dtype: torch.dtype, device: torch.device,
                seed: Optional[int]) -> torch.Tensor:
    """Gaussian probes U (n, N_r) as laker/preconditioner.py:168-171 draws them."""
    gen = torch.Generator(device=device)
    if seed is not None:
        gen.manual_seed(int(seed))
    return torch.randn(n, nr, device=device, dtype=dtype, generator=gen)


def orthonormal_basis(U: torch.Tensor):
    """Economy QR U = Q R of a tall float64 matrix (laker/preconditioner.py:191).

    CholeskyQR2 (two passes of G = Q^T Q, G = L L^T, Q <- Q L^-T; R = R2 R1):
    two GEMMs and two triangular solves instead of Householder QR, orthogonal
    to rounding while cond(U) < ~1e8.  Householder QR (torch.linalg.qr) is the
    fallback when a Cholesky factorisation fails.  R has a positive diagonal,
    so Q and R can differ from Householder's by column signs Q D, D R; the CCCP
    weights diag(R^T M^-1 R) and the apply Q V f(Lambda) V^T Q^T do not see D.
    """
    Q, R = U, None
    for _ in range(2):
        L, info = torch.linalg.cholesky_ex(Q.T @ Q)
        if int(info.item()) != 0:
            return torch.linalg.qr(U, mode="reduced")
        Q = torch.linalg.solve_triangular(L.T, Q, upper=True, left=False)
        R = L.T if R is None else L.T @ R
    return Q, R


def inv_sqrt_spd_batched(M: torch.Tensor, max_iter: int = 100, tol: float = 1e-14) -> torch.Tensor:
    """M^{-1/2} for a batch of SPD float64 matrices (B, m, m).

    Coupled Newton-Schulz iteration on M / s with s = ||M||_F >= lambda_max:
    T = (3 I - Z Y) / 2, Y <- Y T, Z <- T Z, so Z -> (M / s)^{-1/2}; only
    batched GEMMs, no eigensolver.  Stops when every ||I - Z Y||_F <= tol.
    """
    s = torch.linalg.matrix_norm(M).clamp(min=1e-300)
    eye = torch.eye(M.shape[-1], dtype=M.dtype, device=M.device).expand_as(M)
    Y = M / s.view(-1, 1, 1)
    Z = eye.clone()
    for it in range(max_iter):
        ZY = Z @ Y
        if it % 4 == 0 and float(torch.linalg.matrix_norm(eye - ZY).max()) <= tol:
            break
        T = 1.5 * eye - 0.5 * ZY
        Y = Y @ T
        Z = T @ Z
    return Z / s.sqrt().view(-1, 1, 1)


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
        probe_device: Optional[torch.device] = None,
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
        self.probe_device = torch.device(probe_device) if probe_device is not None else self.device
        self.n: Optional[int] = None
        self.nr: Optional[int] = None
        self.q_basis: Optional[torch.Tensor] = None
        self.qr_r: Optional[torch.Tensor] = None
        self.isotropic_coef: Optional[float] = None
        self.q_basis_matrix: Optional[torch.Tensor] = None
        self._q_eig = None  # (eigenvalues, eigenvectors) of c I + B, computed on demand
        self.cccp_iterations: int = 0
        self._q32: Optional[torch.Tensor] = None
        self._w32: Optional[torch.Tensor] = None
        self._c: Optional[_lib.laker_precond] = None

    # ------------------------------------------------------------------
    def build(self, operator: Callable[[torch.Tensor], torch.Tensor], n: int,
              seed: Optional[int] = None, timings: Optional[dict] = None) -> "CCCPPreconditioner":
        """Learn the preconditioner (laker/preconditioner.py:144-284).

        `timings`, when given, receives the seconds spent in each phase
        (probes, operator, qr, fixed_point, apply_factors) and the fixed
        point's iteration count under "iterations"."""
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

        clock = PhaseClock(timings, dev)
        clock.start()
        probes = draw_probes(n, self.nr, dt, self.probe_device, seed).to(dev)
        clock.stop("probes")

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
        _lib.raise_device_status(dev)
        clock.stop("operator")
        dt = torch.float64
        norms = torch.linalg.norm(op_probes, dim=0, keepdim=True)
        normalized = op_probes / norms.clamp(min=self.epsilon)
        q_basis, qr_r = orthonormal_basis(normalized)
        self.q_basis, self.qr_r = q_basis, qr_r
        clock.stop("qr")

        shrinkage = adaptive_shrinkage_rho(self.nr, n, self.gamma, self.base_rho)
        iso, qbm, iters = self._fixed_point_device(n, shrinkage)
        if iso is None:
            # M = c I + B was not positive definite at some iteration (not met
            # on the configs): the reference's eigh formulation, one host
            # synchronisation per iteration
            iso, qbm, iters = self._fixed_point_eigh(n, shrinkage)
        it = iters - 1
        eye = torch.eye(self.nr, device=dev, dtype=torch.float64)
        self.cccp_iterations = it + 1
        self.isotropic_coef = iso
        self.q_basis_matrix = qbm
        clock.stop("fixed_point")
        if timings is not None:
            timings["iterations"] = timings.get("iterations", 0) + it + 1
        self.q_eigenvalues, self.q_eigenvectors = eigh_stable(eye * iso + qbm, eps=self.epsilon)
        self._prepare_apply()
        clock.stop("apply_factors")
        if self.verbose:
            logger.info("CCCP preconditioner built in %d iterations", it + 1)
        return self

    def _fixed_point_device(self, n: int, shrinkage: float):
        """The N_r x N_r CCCP fixed point (laker/preconditioner.py:207-273)
        with its scalars, convergence test and iteration count kept on the
        device: the state freezes at the iteration the reference stops at
        (max(iso_rel, q_rel) < tol), and the host polls every 4 iterations
        instead of once per iteration.  diag(R^T M^-1 R) comes from a Cholesky
        solve (the reference's eigh gives the same quantity for SPD M).
        Returns (c, B, iterations), or (None, None, 0) if a Cholesky
        factorisation failed (M not positive definite)."""
        dev, dt = self.device, torch.float64
        nr = self.nr
        reg_scale = 1.0 + self.gamma / n
        eye = torch.eye(nr, device=dev, dtype=dt)
        iso = torch.ones((), device=dev, dtype=dt)
        qbm = torch.zeros(nr, nr, device=dev, dtype=dt)
        active = torch.ones((), device=dev, dtype=torch.bool)
        failed = torch.zeros((), device=dev, dtype=torch.bool)
        iters = torch.zeros((), device=dev, dtype=torch.int64)
        shrunk_iso = (1.0 - shrinkage) * self.gamma / reg_scale + shrinkage
        for it in range(self.max_iter):
            chol, info = torch.linalg.cholesky_ex(eye * iso + qbm)
            failed |= info != 0
            denom = (self.qr_r * torch.cholesky_solve(self.qr_r, chol)).sum(dim=0) + self.epsilon
            weights = (n / nr) / denom
            wrr = (self.qr_r * weights.unsqueeze(0)) @ self.qr_r.T
            f_gamma = (wrr + self.gamma * eye) * (1.0 / reg_scale)
            shrunk = torch.lerp(f_gamma, eye, shrinkage)
            trace = shrunk_iso * (n - nr) + shrunk.diagonal().sum()
            scale = n / trace
            iso_new = scale * shrunk_iso
            qbm_new = shrunk * scale
            qbm_new.diagonal().sub_(iso_new)
            iso_rel = (iso_new - iso).abs() / (iso.abs() + 1e-12)
            q_rel = torch.norm(qbm_new - qbm, p="fro") / (torch.norm(qbm, p="fro") + 1e-12)
            iso = torch.where(active, iso_new, iso)
            qbm = torch.where(active, qbm_new, qbm)
            iters = iters + active.to(torch.int64)
            active = active & ~(torch.maximum(iso_rel, q_rel) < self.tol)
            if it % 4 == 3 or it == self.max_iter - 1:
                done, bad = bool((~active) | failed), bool(failed)
                if self.verbose:
                    logger.info("CCCP iter %d: isotropic_coef=%.6f (active=%s)", it,
                                float(iso), bool(active))
                if bad:
                    return None, None, 0
                if done:
                    break
        return float(iso), qbm, int(iters)

    def _fixed_point_eigh(self, n: int, shrinkage: float):
        """The fixed point with eigh-based diag(R^T M^-1 R), as the reference
        computes it, synchronising once per iteration."""
        dev, dt = self.device, torch.float64
        reg_scale = 1.0 + self.gamma / n
        iso = 1.0
        qbm = torch.zeros(self.nr, self.nr, device=dev, dtype=dt)
        eye = torch.eye(self.nr, device=dev, dtype=dt)
        it = 0
        for it in range(self.max_iter):
            iso_prev = iso
            qbm_prev = qbm.clone()
            evals, evecs = eigh_stable(eye * iso + qbm, eps=self.epsilon)
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
            if max(iso_rel, q_rel) < self.tol:
                break
        return iso, qbm, it + 1

    # eigen-decomposition of c I + B (reference state attributes); a batched
    # build leaves it to be computed on first access
    @property
    def q_eigenvalues(self) -> Optional[torch.Tensor]:
        return self._eig()[0]

    @q_eigenvalues.setter
    def q_eigenvalues(self, value) -> None:
        self._q_eig = (value, self._q_eig[1] if self._q_eig else None)

    @property
    def q_eigenvectors(self) -> Optional[torch.Tensor]:
        return self._eig()[1]

    @q_eigenvectors.setter
    def q_eigenvectors(self, value) -> None:
        self._q_eig = (self._q_eig[0] if self._q_eig else None, value)

    def _eig(self):
        if (self._q_eig is None or self._q_eig[0] is None) and self.q_basis_matrix is not None:
            eye = torch.eye(self.nr, device=self.q_basis_matrix.device, dtype=self.q_basis_matrix.dtype)
            self._q_eig = eigh_stable(eye * self.isotropic_coef + self.q_basis_matrix, eps=self.epsilon)
        return self._q_eig if self._q_eig is not None else (None, None)

    def _prepare_apply(self, w: Optional[torch.Tensor] = None) -> None:
        """Fold the apply into (Q padded, W = V diag(lambda^-1/2 - c^-1/2) V^T);
        a batched build passes W computed as (c I + B)^-1/2 - c^-1/2 I."""
        if w is None:
            v = self.q_eigenvectors.to(torch.float64)
            scale = self.q_eigenvalues.to(torch.float64).rsqrt() - self.isotropic_coef ** (-0.5)
            w = (v * scale.unsqueeze(0)) @ v.T
        w = 0.5 * (w + w.T)
        self._q32 = _lib.padded_q(self.q_basis)
        self._w32 = w.to(torch.float32).contiguous()
        self._c = _lib.precond_struct(self._q32, self._w32, self.n, self.nr,
                                      self.isotropic_coef ** (-0.5))

    # ---- persistence ----------------------------------------------------------
    def state_dict(self) -> dict:
        """The built state, on the CPU: hyperparameters, the factors of the
        reference state (q_basis, qr_r, isotropic_coef, q_basis_matrix) and the
        folded FP32 apply core W exactly as the fused apply uses it."""
        if self._c is None:
            raise RuntimeError("Preconditioner has not been built. Call build() first.")
        cpu = lambda t: t.detach().to("cpu") if torch.is_tensor(t) else t  # noqa: E731
        return {
            "num_probes": self.num_probes, "gamma": self.gamma, "epsilon": self.epsilon,
            "base_rho": self.base_rho, "max_iter": self.max_iter, "tol": self.tol,
            "n": self.n, "nr": self.nr, "isotropic_coef": float(self.isotropic_coef),
            "cccp_iterations": int(self.cccp_iterations),
            "q_basis": cpu(self.q_basis), "qr_r": cpu(self.qr_r),
            "q_basis_matrix": cpu(self.q_basis_matrix), "w32": cpu(self._w32),
        }

    @classmethod
    def from_state(cls, state: dict, device=None, dtype=None) -> "CCCPPreconditioner":
        """A built preconditioner from state_dict() output (no rebuild: the
        apply uses the stored factors, so results are the same bits)."""
        pre = cls(num_probes=state["num_probes"], gamma=state["gamma"], epsilon=state["epsilon"],
                  base_rho=state["base_rho"], max_iter=state["max_iter"], tol=state["tol"],
                  verbose=False, device=device, dtype=dtype)
        dev = pre.device
        pre.n, pre.nr = int(state["n"]), int(state["nr"])
        pre.isotropic_coef = float(state["isotropic_coef"])
        pre.cccp_iterations = int(state["cccp_iterations"])
        pre.q_basis = state["q_basis"].to(dev)
        pre.qr_r = state["qr_r"].to(dev) if state.get("qr_r") is not None else None
        pre.q_basis_matrix = state["q_basis_matrix"].to(dev)
        pre._q32 = _lib.padded_q(pre.q_basis)
        pre._w32 = state["w32"].to(dev, torch.float32).contiguous()
        pre._c = _lib.precond_struct(pre._q32, pre._w32, pre.n, pre.nr, pre.isotropic_coef ** (-0.5))
        return pre

    def apply_factors(self):
        """(Q padded to a multiple of 4 columns in FP32, the folded W in FP32,
        N_r, c^-1/2): the factors the fused apply uses, P = c^-1/2 I + Q W Q^T."""
        if self._c is None:
            raise RuntimeError("Preconditioner has not been built. Call build() first.")
        return self._q32, self._w32, self.nr, self.isotropic_coef ** (-0.5)

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
        q32, w32, nr, cis = self.apply_factors()
        return ops.precond_apply(q32, w32, self.n, nr, cis, x, x.dtype == torch.float64)

    def apply_2d(self, x: torch.Tensor) -> torch.Tensor:
        _lib.require_cuda(x, "x")
        # k right-hand sides: the multi-RHS fused apply (the one the device
        # multi-RHS solve uses), with the same folded factors
        q32, w32, nr, cis = self.apply_factors()
        return ops.precond_apply(q32, w32, self.n, nr, cis, x, x.dtype == torch.float64)

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
