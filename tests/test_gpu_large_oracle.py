"""The operator kernels at the headline size, checked on row samples against
the float64 oracle.

At n = 100k (and 50k) the symmetric kernels walk thousands of block pairs
(19,306 at n = 100k); the FP64 symmetric kernel decides the solves' stop test
and the FP32 tensor-core one drives the iteration.  A full n^2 oracle product
takes seconds on the host, so each check evaluates the oracle on a random
sample of 2048 rows (exp(E[rows] E^T) x + lam x[rows], float64, OpenMP C).
The embeddings are the real ones of the configs: PositionEmbedding (seed 42)
of the synthetic field.
"""

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

LAM = 1e-2


@pytest.fixture(scope="module", params=[50000, 100000])
def config_embeddings(request, cuda):
    from laker_b200 import PositionEmbedding, synthetic_field

    n = request.param
    x, _, _ = synthetic_field(n, seed=0)
    emb = PositionEmbedding(2, 10).to(cuda)
    with torch.no_grad():
        E = emb(x.to(cuda))
    return n, E


def _sample_ref(E64, x, rows):
    return O.rect_matvec(E64[rows], E64, x) + LAM * x[rows]


def test_fp64_symmetric_kernel_rows_vs_oracle(cuda, config_embeddings):
    from laker_b200 import AttentionKernelOperator

    n, E = config_embeddings
    rng = np.random.default_rng(n)
    E64 = E.double().cpu().numpy()
    op64 = AttentionKernelOperator(E.double(), lambda_reg=LAM)
    x = rng.standard_normal(n)
    y = op64.matvec(torch.tensor(x, device=cuda)).cpu().numpy()
    rows = np.sort(rng.choice(n, 2048, replace=False))
    ref = _sample_ref(E64, x, rows)
    assert np.max(np.abs(y[rows] - ref) / np.abs(ref).max()) < 1e-12
    assert np.linalg.norm(y[rows] - ref) / np.linalg.norm(ref) < 1e-12
    # the FP64 residual b - A x the PCG stop test uses
    b = rng.standard_normal(n)
    r = op64.residual_f64(torch.tensor(x, device=cuda), torch.tensor(b, device=cuda)).cpu().numpy()
    rref = b[rows] - ref
    assert np.linalg.norm(r[rows] - rref) / np.linalg.norm(rref) < 1e-12


def test_fp32_tensor_core_symmetric_kernel_rows_vs_oracle(cuda, config_embeddings, k1t_logits):
    from laker_b200 import AttentionKernelOperator, _lib

    n, E = config_embeddings
    assert _lib.fp32_operator_kernel(n, 10) == 2
    rng = np.random.default_rng(n + 1)
    E32 = E.float()
    op32 = AttentionKernelOperator(E32, lambda_reg=LAM)
    x = rng.standard_normal(n).astype(np.float32)
    y = op32.matvec(torch.tensor(x, device=cuda)).double().cpu().numpy()
    rows = np.sort(rng.choice(n, 2048, replace=False))
    ref = _sample_ref(E32.double().cpu().numpy(), x.astype(np.float64), rows)
    # entries carry ~1e-6 relative error (split logits, ex2.approx); rows are
    # sums of n of them with mixed-sign x
    assert np.linalg.norm(y[rows] - ref) / np.linalg.norm(ref) < 3e-5
    err = np.abs(y[rows] - ref) / np.maximum(np.abs(ref), 1e-3 * np.abs(ref).max())
    assert err.max() < 3e-4
