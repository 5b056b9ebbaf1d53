"""GPU parity of the flash-style multi-RHS FP32 matvec (logits and P X on the
tensor cores, P kept in tensor memory) against the float64 oracle and the
CUDA-core-logit tensor-core kernel it replaces for unclamped operators.

The products are split TF32 (P_hi X_hi + P_hi X_lo + P_lo X_hi, ~2^-21 per
product) with split-FP16 logits, so the bar is the multi-RHS tolerance of the
other tensor-core tests: 1e-4 relative per column against the oracle
(the reference's own float32 tolerance).
"""

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

TC_RTOL = 1e-4


def colrel(Y, ref):
    Y = Y.detach().cpu().double().numpy()
    num = np.linalg.norm(Y - ref, axis=0)
    den = np.maximum(np.linalg.norm(ref, axis=0), 1e-300)
    return float((num / den).max())


def _with_flash(enabled):
    from laker_b200 import _lib
    return _lib.set_variant(_lib.VARIANT_MULTI_FLASH_K, 1024 if enabled else 0)


@pytest.fixture(autouse=True)
def flash_on(cuda):
    """Every test of this file runs with the flash kernel selected for up to
    1024 right-hand sides (the tests that compare switch it off locally)."""
    from laker_b200 import _lib
    prev = _with_flash(True)
    yield
    _lib.set_variant(_lib.VARIANT_MULTI_FLASH_K, prev)


@pytest.mark.parametrize("n,k", [(1, 2), (31, 5), (65, 16), (257, 17), (700, 64), (1500, 100),
                                 (2048, 256), (3000, 16), (4100, 512)])
def test_flash_square_matvec(cuda, n, k):
    from laker_b200 import AttentionKernelOperator, _lib

    rng = np.random.default_rng(n * 1000 + k)
    E = (rng.standard_normal((n, 10)) * 0.5).astype(np.float32)
    X = rng.standard_normal((n, k))
    op = AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=0.03)
    Xt = torch.tensor(X, device=cuda, dtype=torch.float32)
    prev = _with_flash(True)
    try:
        Y = op.matvec(Xt)
        Y2 = op.matvec(Xt)
        _with_flash(False)
        Yk2 = op.matvec(Xt)
    finally:
        _lib.set_variant(_lib.VARIANT_MULTI_FLASH_K, prev)
    assert torch.equal(Y, Y2)  # deterministic
    ref = O.attention_matvec(E, 0.03, X)
    assert colrel(Y, ref) < TC_RTOL
    assert colrel(Y, Yk2.double().cpu().numpy()) < TC_RTOL


@pytest.mark.parametrize("d", [1, 4, 7, 16])
def test_flash_rectangular_all_dims(cuda, d):
    from laker_b200 import _lib

    rng = np.random.default_rng(70 + d)
    n, m, k = 2300, 517, 40
    E = (rng.standard_normal((n, d)) * 0.7 / np.sqrt(d)).astype(np.float32)
    Eq = (rng.standard_normal((m, d)) * 0.7 / np.sqrt(d)).astype(np.float32)
    X = rng.standard_normal((n, k)).astype(np.float32)
    Et, Eqt = torch.tensor(E, device=cuda), torch.tensor(Eq, device=cuda)
    prev = _with_flash(True)
    try:
        Y = _lib.attn_matvec_f32(_lib.pack_f32(Eqt), m, _lib.pack_f32(Et), n, d, 0.0, 0,
                                 torch.tensor(X, device=cuda))
    finally:
        _lib.set_variant(_lib.VARIANT_MULTI_FLASH_K, prev)
    ref = O.rect_matvec(Eq.astype(np.float64), E.astype(np.float64), X.astype(np.float64))
    assert colrel(Y, ref) < TC_RTOL


def test_flash_clamped_operator_takes_the_other_kernel(cuda):
    """Operators that clamp their Gram entries need the clamp inside exp; the
    flash kernel's FP16 logits do not cover them, so they keep the
    CUDA-core-logit kernel (same results as the oracle with the clamp)."""
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(9)
    n, k = 600, 12
    E = rng.standard_normal((n, 4)) * 0.3
    E[:3] *= 40.0
    E32 = E.astype(np.float32)
    op = AttentionKernelOperator(torch.tensor(E32, device=cuda), lambda_reg=0.01)
    assert not op.skip_clamp
    X = rng.standard_normal((n, k))
    Y = op.matvec(torch.tensor(X, device=cuda, dtype=torch.float32))
    ref = O.attention_matvec(E32, 0.01, X, clamp=True, clamp_value=80.0)
    assert colrel(Y, ref) < TC_RTOL


def test_flash_config_embeddings_large_n_rows(cuda):
    """n = 50k with the configs' embeddings, 16 right-hand sides (the served
    variance queries' width), on a row sample of the oracle."""
    from laker_b200 import AttentionKernelOperator, PositionEmbedding, synthetic_field

    n, k = 50000, 16
    x, _, _ = synthetic_field(n, seed=0)
    with torch.no_grad():
        E = PositionEmbedding(2, 10).to(cuda)(x.to(cuda))
    op = AttentionKernelOperator(E, lambda_reg=1e-2)
    rng = np.random.default_rng(5)
    X = rng.standard_normal((n, k)).astype(np.float32)
    Xt = torch.tensor(X, device=cuda)
    Y = op.matvec(Xt).double().cpu().numpy()
    _with_flash(False)
    Yk2 = op.matvec(Xt).double().cpu().numpy()
    rows = np.sort(rng.choice(n, 1024, replace=False))
    E64 = E.double().cpu().numpy()
    ref = O.rect_matvec(E64[rows], E64, X.astype(np.float64)) + 1e-2 * X[rows]
    err = np.linalg.norm(Y[rows] - ref, axis=0) / np.linalg.norm(ref, axis=0)
    err_k2 = np.linalg.norm(Yk2[rows] - ref, axis=0) / np.linalg.norm(ref, axis=0)
    # rows are sums of 50k entries of ~1e-6 relative error against random
    # signs (|K| |x| / |K x| ~ sqrt(n)): ~1e-4 per column for either kernel
    assert err.max() < 3e-4
    assert err.max() < 2.0 * err_k2.max() + 2e-5
