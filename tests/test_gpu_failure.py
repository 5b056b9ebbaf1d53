"""Device-side failure reporting, exercised without any fault.

Every pipeline wait in the kernels is bounded; when one gives up the kernel
records LAKER_ERR_TIMEOUT in its status word, drains its copies and
tensor-core operations still in flight (always with the full limit), frees
its tensor memory and returns.  LAKER_VARIANT_WAIT_LIMIT_US = 0 makes every
pipeline wait give up at once, so these tests drive that path on purpose:
the asynchronous products write NaN and report the status through
laker_workspace_status / laker_noalloc_status, the solves stop and return
it, the Python layer raises, and a call with the normal limit on the same
stream afterwards is correct (the context stays usable).

The reference has no device code; its products raise synchronously
(laker/solvers.py:343-352 for a breakdown).
"""

import contextlib
import ctypes

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

F32_RTOL = 3e-5


def rel(a, b):
    a = a.detach().cpu().double().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@contextlib.contextmanager
def zero_wait_limit():
    from laker_b200 import _lib

    torch.cuda.synchronize()
    prev = _lib.set_variant(_lib.VARIANT_WAIT_LIMIT_US, 0)
    try:
        yield
    finally:
        torch.cuda.synchronize()
        _lib.set_variant(_lib.VARIANT_WAIT_LIMIT_US, prev)


def _embeddings(cuda, n, seed, d=10):
    rng = np.random.default_rng(seed)
    E = (rng.standard_normal((n, d)) * 0.5).astype(np.float32)
    return E, torch.tensor(E, device=cuda)


def test_wait_limit_variant_roundtrip(cuda):
    from laker_b200 import _lib

    assert _lib.get_variant(_lib.VARIANT_WAIT_LIMIT_US) == 2_000_000
    with zero_wait_limit():
        assert _lib.get_variant(_lib.VARIANT_WAIT_LIMIT_US) == 0
    assert _lib.get_variant(_lib.VARIANT_WAIT_LIMIT_US) == 2_000_000
    with pytest.raises(ValueError):
        _lib.set_variant(_lib.VARIANT_WAIT_LIMIT_US, 2_000_001)


@pytest.mark.parametrize("n,k", [(20000, 1), (2000, 1), (6000, 16), (5000, 96)])
def test_timeout_poisons_and_reports_fp32_products(cuda, n, k):
    """The symmetric tensor-core operator (n = 20000), the plain kernel
    (n = 2000) and the multi-RHS tensor-core kernel (k > 1)."""
    from laker_b200 import _lib

    lib = _lib.load()
    E, Et = _embeddings(cuda, n, seed=n + k)
    packed = _lib.pack_f32(Et)
    rng = np.random.default_rng(k)
    X = rng.standard_normal((n, k)) if k > 1 else rng.standard_normal(n)
    Xt = torch.tensor(X, device=cuda, dtype=torch.float32)
    ws = _lib.workspace(lib.laker_matvec_workspace_bytes(n, n, 10, k, 32), cuda)
    Y = torch.zeros(Xt.shape, device=cuda, dtype=torch.float32)
    stream = _lib.stream_handle(cuda)

    def call():
        st = lib.laker_attn_matvec_f32(packed.data_ptr(), n, packed.data_ptr(), n, 10,
                                       ctypes.c_float(0.01), 0, Xt.data_ptr(), k, k, Y.data_ptr(),
                                       k, ws.data_ptr(), ws.numel(), stream)
        assert st == _lib.LAKER_OK
        return _lib.workspace_status(ws)

    with zero_wait_limit():
        assert call() == _lib.LAKER_ERR_TIMEOUT
        assert torch.isnan(Y).all()
    assert call() == _lib.LAKER_OK
    ref = O.attention_matvec(E, 0.01, X)
    assert rel(Y, ref) < (F32_RTOL if k == 1 else 1e-4)


def test_timeout_fp64_symmetric_residual(cuda):
    from laker_b200 import _lib

    n = 9000
    E, Et = _embeddings(cuda, n, seed=5)
    p64 = _lib.pack_f64(Et)
    x = torch.tensor(np.random.default_rng(1).standard_normal(n), device=cuda)
    with zero_wait_limit():
        y = _lib.attn_matvec_f64(p64, n, p64, n, 10, 0.01, 0, x)
        assert torch.isnan(y).all()
        with pytest.raises(_lib.LakerError) as err:
            _lib.raise_device_status(cuda)
        assert err.value.status == _lib.LAKER_ERR_TIMEOUT
    y = _lib.attn_matvec_f64(p64, n, p64, n, 10, 0.01, 0, x)
    _lib.raise_device_status(cuda)  # cleared, and this call succeeded
    assert rel(y, O.attention_matvec(E, 0.01, x.cpu().numpy())) < 1e-12


def test_timeout_noalloc_status(cuda):
    from laker_b200 import _lib

    lib = _lib.load()
    n, m = 12000, 3000
    E, Et = _embeddings(cuda, n, seed=8)
    Q, Qt = _embeddings(cuda, m, seed=9)
    pe, pq = _lib.pack_f32(Et), _lib.pack_f32(Qt)
    a = np.random.default_rng(2).standard_normal(n)
    at = torch.tensor(a, device=cuda, dtype=torch.float32)
    y = torch.zeros(m, device=cuda, dtype=torch.float32)
    stream = _lib.stream_handle(cuda)

    def call():
        st = lib.laker_attn_matvec_f32_noalloc(pq.data_ptr(), m, pe.data_ptr(), n, 10,
                                               ctypes.c_float(0.0), 0, at.data_ptr(),
                                               y.data_ptr(), stream)
        assert st == _lib.LAKER_OK
        return _lib.noalloc_status(cuda)

    with zero_wait_limit():
        assert call() == _lib.LAKER_ERR_TIMEOUT
        assert torch.isnan(y).all()
    assert call() == _lib.LAKER_OK
    assert rel(y, O.rect_matvec(Q.astype(np.float64), E.astype(np.float64), a)) < F32_RTOL


def test_timeout_stops_solves_and_raises(cuda):
    """The fused single-RHS solve and the multi-RHS solve stop on the
    operator's status and the solver raises; the next solve is correct."""
    from laker_b200 import (AttentionKernelOperator, CCCPPreconditioner,
                            PreconditionedConjugateGradient, _lib)

    n = 8000
    E, Et = _embeddings(cuda, n, seed=12)
    lam = 0.5  # well conditioned: the solves after the failures converge quickly
    op = AttentionKernelOperator(Et, lambda_reg=lam)
    pre = CCCPPreconditioner(num_probes=64, verbose=False, device=cuda,
                             dtype=torch.float32).build(op.matvec, n, seed=0)
    rng = np.random.default_rng(4)
    b = torch.tensor(rng.standard_normal(n), device=cuda)
    B = torch.tensor(rng.standard_normal((n, 6)), device=cuda)
    pcg = PreconditionedConjugateGradient(tol=1e-7, max_iter=3000, verbose=False)
    with zero_wait_limit():
        for rhs in (b, B):
            with pytest.raises(_lib.LakerError) as err:
                pcg.solve(op.matvec, pre.apply, rhs)
            assert err.value.status == _lib.LAKER_ERR_TIMEOUT
    x = pcg.solve(op.matvec, pre.apply, b)
    assert pcg.status == _lib.LAKER_OK
    assert O.relres(E.astype(np.float64), lam, x.cpu().numpy(), b.cpu().numpy()) <= 1e-7 * 1.0001
    X = pcg.solve(op.matvec, pre.apply, B)
    assert pcg.status == _lib.LAKER_OK
    Bn = B.cpu().numpy()
    assert np.linalg.norm(Bn - O.attention_matvec(E, lam, X.cpu().numpy())) \
        <= 1e-7 * np.linalg.norm(Bn) * 1.0001
