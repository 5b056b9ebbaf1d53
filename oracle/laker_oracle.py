"""CPU float64 oracle of the LAKER solve path -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference algorithms, used by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline / reference arm as the
checker.  Nothing in the product imports it.  Each function cites the
reference source (package `laker`, file:line) it restates.  Pinned against
golden vectors produced by the reference itself (tests/golden/, generated by
tests/golden/make_golden.py).

Large dense work (the n^2 kernel matvec) goes through liblaker_oracle.so, an
OpenMP C restatement of the same formula built by oracle/Makefile; below
`NUMPY_MAX_N` numpy is used directly.
"""

from __future__ import annotations

import ctypes
import math
import os
from pathlib import Path
from typing import Callable, Optional

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
C_LIB_PATH = ORACLE_DIR / "liblaker_oracle.so"
NUMPY_MAX_N = 4096
_CHUNK_BYTES = 64 * 1024 * 1024

_clib = None


def _c_lib():
    global _clib
    if _clib is None and C_LIB_PATH.exists():
        lib = ctypes.CDLL(str(C_LIB_PATH))
        lib.oracle_attn_matvec.restype = None
        lib.oracle_attn_matvec.argtypes = [
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
            ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
            ctypes.c_int,
        ]
        lib.oracle_num_threads.restype = ctypes.c_int
        lib.oracle_num_threads.argtypes = []
        _clib = lib
    return _clib


def c_threads() -> int:
    lib = _c_lib()
    return int(lib.oracle_num_threads()) if lib is not None else 1


# ---------------------------------------------------------------------------
# Embedding  (laker/embeddings.py:220-242)
# ---------------------------------------------------------------------------
def embed(x, freq, phase, w1, b1, w2, b2, dtype=np.float64):
    """E = W2 tanh(W1 cos(2 pi x F + phi) + b1) + b2 (nn.Linear: y = x W^T + b)."""
    x = np.asarray(x, dtype=dtype)
    f = np.cos(2.0 * math.pi * (x @ np.asarray(freq, dtype)) + np.asarray(phase, dtype))
    h = np.tanh(f @ np.asarray(w1, dtype).T + np.asarray(b1, dtype))
    return h @ np.asarray(w2, dtype).T + np.asarray(b2, dtype)


# ---------------------------------------------------------------------------
# Exact attention kernel  (laker/kernels.py:80-130, 187-354)
# ---------------------------------------------------------------------------
def safe_limit(dtype=np.float64) -> float:
    """exp_safe clamp level (kernels.py:98-99)."""
    return 80.0 if np.dtype(dtype) == np.float32 else 700.0


def skip_clamp(E, dtype=np.float64) -> bool:
    """kernels.py:181-185."""
    E = np.asarray(E, np.float64)
    return bool(E.shape[0] == 0 or np.max(np.sum(E * E, axis=1)) < safe_limit(dtype))


def attention_matvec(E, lam, X, clamp: bool = False, clamp_value: float = 700.0):
    """(lam I + exp(E E^T)) X in float64, X (n,) or (n,k).

    dense_attention_matvec (kernels.py:121-130) / matvec_impl (:209-270); the
    row-chunked evaluation keeps peak memory at ~64 MB.
    """
    E = np.ascontiguousarray(E, dtype=np.float64)
    X = np.asarray(X, dtype=np.float64)
    n = E.shape[0]
    lib = _c_lib()
    if n > NUMPY_MAX_N and lib is not None and _narrow(X):
        return _c_matvec(lib, E, E, lam, X, clamp, clamp_value)
    return _np_matvec(E, E, lam, X, clamp, clamp_value, square=True)


def rect_matvec(Eq, E, X, clamp: bool = False, clamp_value: float = 700.0):
    """exp(Eq E^T) X (the exact-kernel prediction of core.py:633-655)."""
    Eq = np.ascontiguousarray(Eq, dtype=np.float64)
    E = np.ascontiguousarray(E, dtype=np.float64)
    X = np.asarray(X, dtype=np.float64)
    lib = _c_lib()
    if max(Eq.shape[0], E.shape[0]) > NUMPY_MAX_N and lib is not None and _narrow(X):
        return _c_matvec(lib, Eq, E, 0.0, X, clamp, clamp_value)
    return _np_matvec(Eq, E, 0.0, X, clamp, clamp_value, square=False)


def _narrow(X) -> bool:
    """Few right-hand sides take the OpenMP C loop; wide blocks the blocked
    numpy path, whose (rows x n) @ (n x k) products run as BLAS GEMMs."""
    return X.ndim == 1 or X.shape[1] <= 8


def _np_matvec(Er, Ec, lam, X, clamp, clamp_value, square):
    m = Er.shape[0]
    out = np.zeros((m,) + X.shape[1:], dtype=np.float64)
    rows = max(1, _CHUNK_BYTES // (8 * max(1, Ec.shape[0])))
    for s in range(0, m, rows):
        g = Er[s : s + rows] @ Ec.T
        if clamp:
            np.minimum(g, clamp_value, out=g)
        np.exp(g, out=g)
        out[s : s + rows] = g @ X
    if square:
        out += lam * X
    return out


def _c_matvec(lib, Er, Ec, lam, X, clamp, clamp_value):
    one_d = X.ndim == 1
    Xc = np.ascontiguousarray(X.reshape(X.shape[0], -1), dtype=np.float64)
    k = Xc.shape[1]
    out = np.empty((Er.shape[0], k), dtype=np.float64)
    lib.oracle_attn_matvec(
        Er.ctypes.data, Er.shape[0], Ec.ctypes.data, Ec.shape[0], Er.shape[1], float(lam),
        float(clamp_value) if clamp else float("inf"), Xc.ctypes.data, k, out.ctypes.data,
        int(Er is Ec or (Er.shape == Ec.shape and np.shares_memory(Er, Ec))),
    )
    return out[:, 0] if one_d else out


def diagonal(E, lam):
    """lam + exp(||e_i||^2) (kernels.py:272-283)."""
    E = np.asarray(E, np.float64)
    return lam + np.exp(np.sum(E * E, axis=1))


def kernel_eval(X, Y, clamp: bool = False, clamp_value: float = 700.0):
    """exp(X Y^T) (kernels.py:301-354)."""
    g = np.asarray(X, np.float64) @ np.asarray(Y, np.float64).T
    if clamp:
        np.minimum(g, clamp_value, out=g)
    return np.exp(g)


def to_dense(E, lam):
    """exp(E E^T) + lam I (kernels.py:285-299)."""
    g = kernel_eval(E, E)
    g[np.diag_indices_from(g)] += lam
    return g


# ---------------------------------------------------------------------------
# Helpers  (laker/utils.py:68-134)
# ---------------------------------------------------------------------------
def adaptive_shrinkage_rho(num_probes, problem_size, gamma, base_rho=0.05):
    """utils.py:68-106."""
    if num_probes >= problem_size:
        return base_rho
    ratio = num_probes / problem_size
    rho = base_rho + (1.0 - base_rho) * (1.0 - ratio) * min(1.0, gamma * 10.0)
    return float(min(rho, 0.5))


def eigh_stable(mat, eps=1e-10):
    """utils.py:109-134."""
    w, v = np.linalg.eigh(mat)
    return np.maximum(w, eps), v


# ---------------------------------------------------------------------------
# CCCP preconditioner  (laker/preconditioner.py:52-68, 144-284)
# ---------------------------------------------------------------------------
def cccp_build(apply_a: Callable, n: int, probes, gamma=0.1, epsilon=1e-8, base_rho=0.05,
               max_iter=200, tol=1e-6):
    """CCCPPreconditioner.build with the probe block given (preconditioner.py:144-284)."""
    probes = np.asarray(probes, np.float64)
    nr = probes.shape[1]
    op_probes = apply_a(probes)
    norms = np.linalg.norm(op_probes, axis=0, keepdims=True)
    normalized = op_probes / np.maximum(norms, epsilon)
    q, r = np.linalg.qr(normalized, mode="reduced")
    shrink = adaptive_shrinkage_rho(nr, n, gamma, base_rho)
    reg = 1.0 + gamma / n
    iso = 1.0
    qbm = np.zeros((nr, nr))
    eye = np.eye(nr)
    iters = 0
    for it in range(max_iter):
        iters = it + 1
        iso_prev, qbm_prev = iso, qbm.copy()
        w, v = eigh_stable(eye * iso + qbm, eps=epsilon)
        proj = v.T @ r
        inv_m_r = proj.T @ ((1.0 / w)[:, None] * proj)
        denom = np.diag(inv_m_r) + epsilon
        weights = (n / nr) / denom
        f_gamma = ((r * weights[None, :]) @ r.T + gamma * eye) * (1.0 / reg)
        shrunk = f_gamma + shrink * (eye - f_gamma)
        shrunk_iso = (1.0 - shrink) * gamma / reg + shrink
        trace = shrunk_iso * (n - nr) + np.trace(shrunk)
        scale = n / trace
        iso = scale * shrunk_iso
        qbm = shrunk * scale
        qbm[np.diag_indices(nr)] -= iso
        iso_rel = abs(iso - iso_prev) / (abs(iso_prev) + 1e-12)
        q_rel = np.linalg.norm(qbm - qbm_prev) / (np.linalg.norm(qbm_prev) + 1e-12)
        if max(iso_rel, q_rel) < tol:
            break
    ew, ev = eigh_stable(eye * iso + qbm, eps=epsilon)
    return {
        "q_basis": q, "qr_r": r, "isotropic_coef": float(iso), "q_basis_matrix": qbm,
        "q_eigenvalues": ew, "q_eigenvectors": ev, "iterations": iters, "nr": nr,
    }


def cccp_apply(state, x):
    """preconditioner_apply_core (preconditioner.py:52-68)."""
    x = np.asarray(x, np.float64)
    inv = state["isotropic_coef"] ** (-0.5)
    coeffs = state["q_eigenvectors"].T @ (state["q_basis"].T @ x)
    scale = 1.0 / np.sqrt(state["q_eigenvalues"]) - inv
    coeffs = scale * coeffs if x.ndim == 1 else scale[:, None] * coeffs
    return inv * x + state["q_basis"] @ (state["q_eigenvectors"] @ coeffs)


# ---------------------------------------------------------------------------
# PCG  (laker/solvers.py:130-394)
# ---------------------------------------------------------------------------
class Breakdown(RuntimeError):
    pass


def pcg_solve(apply_a: Callable, apply_p: Callable, b, tol=1e-6, max_iter=None, x0=None,
              breakdown_eps=None):
    """PreconditionedConjugateGradient.solve in float64.

    Returns (x, iterations, residual_norm) where residual_norm is the final
    recurrence residual, as the reference reports it.  1-D b follows solve_1d
    (:189-295), 2-D b solve_2d (:297-394) with the global Frobenius stop test.
    """
    b = np.asarray(b, np.float64)
    if b.ndim not in (1, 2):
        raise ValueError(f"rhs must be 1-D or 2-D, got shape {b.shape}")
    n = b.shape[0]
    max_iter = n if max_iter is None else max_iter
    eps = math.sqrt(np.finfo(np.float64).eps) if breakdown_eps is None else breakdown_eps
    if x0 is None:
        x = np.zeros_like(b)
        r = b.copy()
    else:
        x = np.array(x0, np.float64)
        r = b - apply_a(x)
    z = apply_p(r)
    p = z.copy()
    bn = np.linalg.norm(b)
    if bn == 0:
        return x, 0, 0.0
    one_d = b.ndim == 1
    rz = float(r @ z) if one_d else np.sum(r * z, axis=0)
    rn = float("inf")
    for it in range(max_iter):
        ap = apply_a(p)
        if one_d:
            pap = float(p @ ap)
            bad = pap <= -eps * np.linalg.norm(p) * np.linalg.norm(ap)
        else:
            pap = np.sum(p * ap, axis=0)
            bad = np.any(pap <= -eps * np.linalg.norm(p, axis=0) * np.linalg.norm(ap, axis=0))
        if bad:
            raise Breakdown("PCG breakdown: non-positive curvature detected (p^T A p <= 0).")
        alpha = rz / pap
        x = x + (alpha * p if one_d else p * alpha[None, :])
        r = r - (alpha * ap if one_d else ap * alpha[None, :])
        rn = float(np.linalg.norm(r))
        if rn / bn <= tol:
            return x, it + 1, rn
        z = apply_p(r)
        rz_new = float(r @ z) if one_d else np.sum(r * z, axis=0)
        beta = rz_new / rz
        p = z + (beta * p if one_d else p * beta[None, :])
        rz = rz_new
    return x, max_iter, rn


# ---------------------------------------------------------------------------
# Prediction and variance  (laker/core.py:580-777)
# ---------------------------------------------------------------------------
def predict(Eq, E, alpha):
    """exp(Eq E^T) alpha (core.py:580-661)."""
    return rect_matvec(Eq, E, alpha)


def predict_variance(Eq, E, apply_a, apply_p, tol=1e-6, max_iter=1000):
    """k(q,q) - k(q,X)^T A^{-1} k(q,X), clamped at 0 (core.py:666-777)."""
    kxq = kernel_eval(E, Eq)
    v, iters, _ = pcg_solve(apply_a, apply_p, kxq, tol=tol, max_iter=max_iter)
    kdiag = np.exp(np.sum(np.asarray(Eq, np.float64) ** 2, axis=1))
    var = kdiag - np.sum(kxq * v, axis=0)
    return np.maximum(var, 0.0), iters


def relres(E, lam, x, b):
    """||b - A x|| / ||b|| with the float64 operator."""
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(b - attention_matvec(E, lam, x)) / np.linalg.norm(b))


def fit(E, y, lam=1e-2, gamma=0.1, num_probes=None, probes=None, pcg_tol=1e-6, pcg_max_iter=1000,
        cccp_max_iter=200, cccp_tol=1e-6, epsilon=1e-8, base_rho=0.05):
    """LAKERRegressor.fit after the embedding (models.py:392-455), float64."""
    E = np.asarray(E, np.float64)
    n = E.shape[0]
    if probes is None:
        raise ValueError("probes (n x N_r) must be given")
    apply_a = lambda v: attention_matvec(E, lam, v)  # noqa: E731
    state = cccp_build(apply_a, n, probes, gamma, epsilon, base_rho, cccp_max_iter, cccp_tol)
    alpha, iters, rn = pcg_solve(apply_a, lambda v: cccp_apply(state, v), y, pcg_tol, pcg_max_iter)
    return alpha, iters, state


def num_threads_env() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
