"""GPU parity of the device-resident multi-RHS PCG (solve_2d) and of the
multi-RHS CCCP apply it uses, against the float64 oracle.

The multi-RHS solve keeps X and R in FP64 and recomputes the FP64 residual
B - A X before every stop decision, so its result is held to the requested
tolerance on the float64 operator, checked here with the oracle's operator
(reference: laker/solvers.py:297-394, global Frobenius stop test; the
per-column stop is an opt-in of this package).
"""

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

APPLY_RTOL = 1e-5  # FP32 Q and W in the apply, as for the single-RHS apply
LAM = 0.1  # random embeddings: condition number ~1e4-1e5 at these sizes


def rel(a, b):
    a = a.detach().cpu().double().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = b.detach().cpu().double().numpy() if torch.is_tensor(b) else np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _problem(cuda, n, k, seed, dtype=torch.float32, nr=80):
    from laker_b200 import AttentionKernelOperator, CCCPPreconditioner

    rng = np.random.default_rng(seed)
    E = (rng.standard_normal((n, 10)) * 0.5).astype(np.float32)
    op = AttentionKernelOperator(torch.tensor(E, device=cuda).to(dtype), lambda_reg=LAM)
    pre = CCCPPreconditioner(num_probes=nr, gamma=0.1, max_iter=100, tol=1e-6, verbose=False,
                             device=cuda, dtype=dtype).build(op.matvec, n, seed=seed)
    B = rng.standard_normal((n, k))
    return E, op, pre, B


def _factors_apply(pre, R):
    """c^-1/2 R + Q W Q^T R in float64 from the fused apply's own (FP32) factors."""
    q32, w32, nr, cis = pre.apply_factors()
    Q = q32[:, :nr].double().cpu().numpy()
    W = w32.double().cpu().numpy()
    return cis * R + Q @ (W @ (Q.T @ R))


@pytest.mark.parametrize("n,k", [(700, 2), (1500, 17), (3000, 64), (2100, 300)])
def test_multi_rhs_apply_matches_factors(cuda, n, k):
    _, _, pre, B = _problem(cuda, n, k, seed=n + k)
    R = torch.tensor(B, device=cuda)
    Z = pre.apply(R)
    assert Z.shape == (n, k) and Z.dtype == torch.float64
    ref = _factors_apply(pre, B)
    col = np.linalg.norm(Z.cpu().numpy() - ref, axis=0) / np.linalg.norm(ref, axis=0)
    assert col.max() < APPLY_RTOL
    # the multi-RHS apply agrees with the single-RHS one column by column
    for c in (0, k - 1):
        assert rel(Z[:, c], pre.apply(R[:, c].contiguous())) < APPLY_RTOL
    # FP32 output
    Z32 = pre.apply(R.float())
    assert Z32.dtype == torch.float32 and rel(Z32, ref) < APPLY_RTOL


@pytest.mark.parametrize("n,k", [(900, 2), (2500, 16), (4100, 48), (2000, 300)])
def test_multi_pcg_reaches_tolerance_on_oracle_operator(cuda, n, k):
    from laker_b200 import PreconditionedConjugateGradient

    E, op, pre, B = _problem(cuda, n, k, seed=7 * n + k)
    pcg = PreconditionedConjugateGradient(tol=1e-10, max_iter=5000, verbose=False)
    X = pcg.solve(op.matvec, pre.apply, torch.tensor(B, device=cuda))
    assert X.shape == (n, k) and pcg.status == 0
    Xn = X.cpu().double().numpy()
    resid = B - O.attention_matvec(E, LAM, Xn)
    # the global Frobenius stop test of solve_2d, on the float64 operator
    assert np.linalg.norm(resid) <= 1e-10 * np.linalg.norm(B) * 1.0001
    assert abs(pcg.residual_norm - np.linalg.norm(resid)) <= 1e-3 * np.linalg.norm(resid) + 1e-14
    assert pcg.accurate_matvecs >= 1 and pcg.iterations > 0
    if n <= 2500:
        truth = np.linalg.solve(O.to_dense(E, LAM), B)
        assert rel(Xn, truth) < 1e-5
    # columns agree with single-RHS solves of the same columns
    pcg1 = PreconditionedConjugateGradient(tol=1e-10, max_iter=5000, verbose=False)
    x0 = pcg1.solve(op.matvec, pre.apply, torch.tensor(B[:, 0], device=cuda))
    assert rel(X[:, 0], x0) < 1e-6


def test_multi_pcg_deterministic_and_float64_operator(cuda):
    from laker_b200 import PreconditionedConjugateGradient

    E, op, pre, B = _problem(cuda, 1800, 12, seed=11)
    Bt = torch.tensor(B, device=cuda)
    pcg = PreconditionedConjugateGradient(tol=1e-7, max_iter=5000, verbose=False)
    X1 = pcg.solve(op.matvec, pre.apply, Bt)
    X2 = pcg.solve(op.matvec, pre.apply, Bt)
    assert torch.equal(X1, X2)
    # the float64 operator takes the same loop
    E64, op64, pre64, _ = _problem(cuda, 1800, 12, seed=11, dtype=torch.float64)
    X3 = pcg.solve(op64.matvec, pre64.apply, Bt)
    assert np.linalg.norm(B - O.attention_matvec(E64, LAM, X3.cpu().numpy())) \
        <= 1e-7 * np.linalg.norm(B) * 1.0001


def test_multi_pcg_column_stop(cuda):
    """Columns of very different scale: the global Frobenius test guarantees
    only |R|_F <= tol |B|_F; the per-column stop holds every column to
    tol |b_c| on the float64 operator."""
    from laker_b200 import PreconditionedConjugateGradient

    E, op, pre, B = _problem(cuda, 2200, 8, seed=5)
    B = B * np.logspace(-4, 2, 8)[None, :]
    Bt = torch.tensor(B, device=cuda)
    tol = 1e-7

    def col_relres(X):
        R = B - O.attention_matvec(E, LAM, X.cpu().double().numpy())
        return np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)

    glob = PreconditionedConjugateGradient(tol=tol, max_iter=5000, verbose=False)
    Xg = glob.solve(op.matvec, pre.apply, Bt)
    percol = PreconditionedConjugateGradient(tol=tol, max_iter=5000, verbose=False, column_stop=True)
    Xc = percol.solve(op.matvec, pre.apply, Bt)
    cg, cc = col_relres(Xg), col_relres(Xc)
    assert cc.max() <= tol * 1.0001
    assert percol.status == 0 and glob.status == 0
    Rg = B - O.attention_matvec(E, LAM, Xg.cpu().double().numpy())
    assert np.linalg.norm(Rg) <= tol * np.linalg.norm(B) * 1.0001
    assert cg.shape == cc.shape


def test_multi_pcg_zero_column_warm_start_and_errors(cuda):
    from laker_b200 import AttentionKernelOperator, PreconditionedConjugateGradient

    E, op, pre, B = _problem(cuda, 1300, 5, seed=3)
    B[:, 2] = 0.0
    Bt = torch.tensor(B, device=cuda)
    pcg = PreconditionedConjugateGradient(tol=1e-8, max_iter=5000, verbose=False)
    X = pcg.solve(op.matvec, pre.apply, Bt)
    assert torch.count_nonzero(X[:, 2]).item() == 0
    assert np.linalg.norm(B - O.attention_matvec(E, LAM, X.cpu().numpy())) \
        <= 1e-8 * np.linalg.norm(B) * 1.0001
    # warm start from the solution: at most a couple of iterations
    warm = PreconditionedConjugateGradient(tol=1e-8, max_iter=5000, verbose=False)
    X2 = warm.solve(op.matvec, pre.apply, Bt, x0=X)
    assert warm.iterations <= 2
    assert rel(X2, X) < 1e-7
    # all-zero right-hand side: zeros back, no iteration
    Z = pcg.solve(op.matvec, pre.apply, torch.zeros_like(Bt))
    assert torch.count_nonzero(Z).item() == 0 and pcg.iterations == 0
    # NaN in the data: a RuntimeError, not a hang or a silent result
    Bn = Bt.clone()
    Bn[5, 1] = float("nan")
    with pytest.raises(RuntimeError):
        pcg.solve(op.matvec, pre.apply, Bn)
    # an indefinite operator (negative lambda): breakdown, as in solve_2d
    bad = AttentionKernelOperator(op.embeddings, lambda_reg=-50.0)
    with pytest.raises(RuntimeError, match="breakdown"):
        pcg.solve(bad.matvec, None, Bt)
    # max_iter reached: x is returned, the status says so
    short = PreconditionedConjugateGradient(tol=1e-14, max_iter=3, verbose=False)
    short.solve(op.matvec, pre.apply, Bt)
    assert short.iterations == 3 and short.status == 4


def test_variance_uses_device_solve(cuda):
    """predict_variance (laker/core.py:666-777) on the device multi-RHS solve:
    the variances equal the oracle's direct formula to the solve tolerance."""
    from laker_b200 import LAKERRegressor, synthetic_field

    x, y, xq = synthetic_field(1500, seed=2, m=40)
    model = LAKERRegressor(num_probes=100, pcg_tol=1e-8, verbose=False, device=cuda)
    model.fit(x.to(cuda), y.to(cuda), seed=0)
    var = model.predict_variance(xq.to(cuda)).double().cpu().numpy()
    E = model.embeddings.double().cpu().numpy()
    with torch.no_grad():
        Eq = model.embedding_model(xq.to(cuda)).double().cpu().numpy()
    K = O.kernel_eval(E, Eq)
    V = np.linalg.solve(O.to_dense(E, 1e-2), K)
    ref = np.maximum(np.exp(np.sum(Eq ** 2, axis=1)) - np.sum(K * V, axis=0), 0.0)
    kq = np.exp(np.sum(Eq ** 2, axis=1))
    assert np.max(np.abs(var - ref) / kq) < 1e-6
