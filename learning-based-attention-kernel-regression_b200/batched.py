"""Many independent regressions solved together on one GPU.

`build_cccp_batched` builds the CCCP preconditioners of a list of operators
(laker/preconditioner.py:144-284 per instance): probes, operator(probes) and
CholeskyQR2 per instance, then the N_r x N_r fixed point for all instances at
once -- padded to the largest N_r, batched float64 Cholesky on the GPU for
diag(R^T M^-1 R) (the reference's eigh gives the same quantity; M is SPD), and
a per-instance convergence mask that freezes each instance at the iteration the
reference would stop at -- and the apply's W = M^-1/2 - c^-1/2 I for all
instances by a batched Newton-Schulz iteration.

`BatchedPCG.solve` runs laker_pcg_solve_batched: one device loop for all
instances (block-diagonal symmetric FP32 matvec over the block pairs of the
instances still running, vector steps over 512-point blocks with per-instance
reductions in a fixed order, per-instance scalars and convergence masks on the
device, the iteration replayed as a CUDA graph).
"""

from __future__ import annotations

import ctypes
import logging
from typing import List, Optional, Sequence

import torch

from . import _lib
from .kernels import AttentionKernelOperator
from .preconditioner import (CCCPPreconditioner, PhaseClock, adaptive_shrinkage_rho, draw_probes,
                             inv_sqrt_spd_batched, orthonormal_basis)

logger = logging.getLogger(__name__)


def build_cccp_batched(
    operators: Sequence[AttentionKernelOperator],
    num_probes: Optional[int] = None,
    gamma: float = 0.1,
    epsilon: float = 1e-8,
    base_rho: float = 0.05,
    max_iter: int = 200,
    tol: float = 1e-6,
    seeds: Optional[Sequence[int]] = None,
    probe_device: Optional[torch.device] = None,
    timings: Optional[dict] = None,
) -> List[CCCPPreconditioner]:
    """CCCP preconditioners for many operators (one per operator).

    Instance k draws its probes like CCCPPreconditioner.build(seed=seeds[k])
    (on the operator's device unless probe_device is given), so each result
    matches the single build up to the float64 rounding of the batched fixed
    point.  `timings`, when given, receives the seconds spent in each phase
    (probes, operator, qr, fixed_point, apply_factors)."""
    count = len(operators)
    if count == 0:
        return []
    dev = operators[0].device
    f64 = torch.float64
    clock = PhaseClock(timings, dev)
    pres, rs, ns, nrs = [], [], [], []
    for k, op in enumerate(operators):
        n = op.n
        pre = CCCPPreconditioner(num_probes=num_probes, gamma=gamma, epsilon=epsilon,
                                 base_rho=base_rho, max_iter=max_iter, tol=tol, verbose=False,
                                 device=dev, dtype=op.dtype, probe_device=probe_device)
        nr = num_probes if num_probes is not None else max(200, int(2 * n**0.5))
        nr = min(nr, n)
        if nr > 1024:
            raise ValueError(f"num_probes must be <= 1024 for the fused apply, got {nr}")
        pre.n, pre.nr = n, nr
        clock.start()
        probes = draw_probes(n, nr, op.dtype, pre.probe_device,
                             seeds[k] if seeds is not None else None).to(dev)
        clock.stop("probes")
        op_probes = op.matvec(probes).to(f64)
        clock.stop("operator")
        norms = torch.linalg.norm(op_probes, dim=0, keepdim=True)
        q, r = orthonormal_basis(op_probes / norms.clamp(min=epsilon))
        clock.stop("qr")
        pre.q_basis, pre.qr_r = q, r
        pres.append(pre)
        rs.append(r)
        ns.append(n)
        nrs.append(nr)

    clock.start()
    m = max(nrs)
    R = torch.zeros(count, m, m, dtype=f64, device=dev)
    mask = torch.zeros(count, m, dtype=f64, device=dev)
    for k in range(count):
        R[k, : nrs[k], : nrs[k]] = rs[k]
        mask[k, : nrs[k]] = 1.0
    n_t = torch.tensor(ns, dtype=f64, device=dev)
    nr_t = torch.tensor(nrs, dtype=f64, device=dev)
    shrink = torch.tensor([adaptive_shrinkage_rho(nrs[k], ns[k], gamma, base_rho)
                           for k in range(count)], dtype=f64, device=dev)
    reg = 1.0 + gamma / n_t
    eye = torch.eye(m, dtype=f64, device=dev).expand(count, m, m)
    real = mask.unsqueeze(2) * mask.unsqueeze(1)  # real (nr_k x nr_k) block
    iso = torch.ones(count, dtype=f64, device=dev)
    qbm = torch.zeros(count, m, m, dtype=f64, device=dev)
    active = torch.ones(count, dtype=torch.bool, device=dev)
    iters = torch.zeros(count, dtype=torch.int64, device=dev)
    for it in range(max_iter):
        mm = eye * iso.view(-1, 1, 1) + qbm
        chol = torch.linalg.cholesky(mm)
        z = torch.cholesky_solve(R, chol)
        denom = (R * z).sum(dim=1) + epsilon  # diag(R^T M^-1 R)
        weights = (n_t / nr_t).unsqueeze(1) / denom * mask
        wrr = (R * weights.unsqueeze(1)) @ R.transpose(1, 2)
        f_gamma = (wrr + gamma * eye) / reg.view(-1, 1, 1)
        shrunk = torch.lerp(f_gamma, eye, shrink.view(-1, 1, 1))
        shrunk_iso = (1.0 - shrink) * gamma / reg + shrink
        trace = shrunk_iso * (n_t - nr_t) + (torch.diagonal(shrunk, dim1=1, dim2=2) * mask).sum(1)
        scale = n_t / trace
        iso_new = scale * shrunk_iso
        qbm_new = (shrunk * scale.view(-1, 1, 1) - eye * iso_new.view(-1, 1, 1)) * real
        iso_rel = (iso_new - iso).abs() / (iso.abs() + 1e-12)
        q_rel = torch.linalg.matrix_norm(qbm_new - qbm) / (torch.linalg.matrix_norm(qbm) + 1e-12)
        upd = active
        iso = torch.where(upd, iso_new, iso)
        qbm = torch.where(upd.view(-1, 1, 1), qbm_new, qbm)
        iters = iters + upd.to(torch.int64)
        active = active & ~(torch.maximum(iso_rel, q_rel) < tol)
        # converged instances are frozen by the mask, so polling every few
        # iterations changes nothing but the number of host syncs
        if it % 4 == 3 and not bool(active.any()):
            break
    iso_h = iso.tolist()
    iters_h = iters.tolist()
    clock.stop("fixed_point")
    # W_k = (c_k I + B_k)^-1/2 - c_k^-1/2 I for the fused apply, for all
    # instances at once: on the padded block c_k I the batched inverse square
    # root is c_k^-1/2 I, so W vanishes there.  The eigen-decomposition (a
    # reference state attribute) is computed only if it is read.
    mm = eye * iso.view(-1, 1, 1) + qbm
    W = inv_sqrt_spd_batched(mm) - eye * iso.rsqrt().view(-1, 1, 1)
    for k in range(count):
        pre = pres[k]
        nr = nrs[k]
        pre.isotropic_coef = float(iso_h[k])
        pre.q_basis_matrix = qbm[k, :nr, :nr].clone()
        pre.cccp_iterations = int(iters_h[k])
        pre._prepare_apply(W[k, :nr, :nr])
    clock.stop("apply_factors")
    return pres


class BatchedPCG:
    """PCG for many independent systems (laker_pcg_solve_batched).

    Same stopping rule as the single solve (true FP64 relative residual <= tol
    per instance); after `solve`, `iterations`, `accurate_matvecs`,
    `residual_norms`, `rhs_norms` and `statuses` hold one entry per instance
    and `kernel_launches` the launches of the whole batch.
    """

    def __init__(self, tol: float = 1e-6, max_iter: int = 1000, reliable_delta: float = 0.03,
                 check_every: int = 8) -> None:
        self.tol = float(tol)
        self.max_iter = int(max_iter)
        self.reliable_delta = float(reliable_delta)
        self.check_every = int(check_every)
        self.iterations: List[int] = []
        self.accurate_matvecs: List[int] = []
        self.residual_norms: List[float] = []
        self.rhs_norms: List[float] = []
        self.statuses: List[int] = []
        self.kernel_launches = 0

    def solve(self, operators: Sequence[AttentionKernelOperator],
              preconditioners: Optional[Sequence[CCCPPreconditioner]],
              rhs: Sequence[torch.Tensor]) -> List[torch.Tensor]:
        count = len(operators)
        if count == 0:
            return []
        if len(rhs) != count or (preconditioners is not None and len(preconditioners) != count):
            raise ValueError("operators, preconditioners and rhs must have the same length")
        d = operators[0].embedding_dim
        dev = operators[0].device
        if any(op.embedding_dim != d for op in operators):
            raise ValueError("all operators of a batch must share the embedding dimension")
        lib = _lib.load()
        ns = (ctypes.c_int64 * count)(*[op.n for op in operators])
        offs = (ctypes.c_int64 * (count + 1))()
        total = int(lib.laker_batch_layout(count, ns, offs))
        dp = (d + 1) // 2 * 2
        packed32 = torch.zeros(total * dp, dtype=torch.float32, device=dev)
        packed64 = torch.zeros(total * dp, dtype=torch.float64, device=dev)
        b = torch.zeros(total, dtype=torch.float64, device=dev)
        for k, op in enumerate(operators):
            o = offs[k] * dp
            p32, p64 = op.packed.packed32, op.packed.packed64
            packed32[o : o + p32.numel()] = p32
            packed64[o : o + p64.numel()] = p64
            rk = rhs[k]
            if rk.dim() != 1 or rk.shape[0] != op.n:
                raise ValueError(f"rhs {k} must have shape ({op.n},), got {tuple(rk.shape)}")
            b[offs[k] : offs[k] + op.n] = rk.to(torch.float64)
        x = torch.empty(total, dtype=torch.float64, device=dev)
        lams = (ctypes.c_double * count)(*[op.lambda_reg for op in operators])
        pcs = None
        if preconditioners is not None:
            pcs = (_lib.laker_precond * count)(*[p.c_precond() for p in preconditioners])
        batch = _lib.laker_batch(count, d, int(any(not op.skip_clamp for op in operators)), ns, lams,
                                 packed32.data_ptr(), packed64.data_ptr(), pcs)
        params = _lib.laker_pcg_params(self.tol, self.max_iter, self.reliable_delta,
                                       torch.finfo(torch.float32).eps ** 0.5, self.check_every,
                                       0, 0)
        max_nr = max(p.nr for p in preconditioners) if preconditioners is not None else 0
        ws = _lib.workspace(lib.laker_pcg_batched_workspace_bytes(count, ns, d, max_nr), dev)
        results = (_lib.laker_pcg_result * count)()
        _lib.check(lib.laker_pcg_solve_batched(ctypes.byref(batch), b.data_ptr(), x.data_ptr(),
                                               ctypes.byref(params), ws.data_ptr(), ws.numel(),
                                               results, _lib.stream_handle(dev)),
                   "laker_pcg_solve_batched")
        self.iterations = [r.iterations for r in results]
        self.accurate_matvecs = [r.accurate_matvecs for r in results]
        self.residual_norms = [r.residual_norm for r in results]
        self.rhs_norms = [r.rhs_norm for r in results]
        self.statuses = [r.status for r in results]
        self.kernel_launches = results[0].kernel_launches
        return [x[offs[k] : offs[k] + operators[k].n].clone() for k in range(count)]
