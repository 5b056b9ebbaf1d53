"""GPU autograd through the fused operator: gradients of a loss of
(lambda I + exp(E E^T)) x with respect to the embeddings E and to x, against
torch autograd on the dense float64 product (the reference's own computation
under autograd, laker/kernels.py:121-130 with requires_grad embeddings)."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _dense_grads(E, x, gy, lam):
    E = E.detach().cpu().double().requires_grad_(True)
    x = x.detach().cpu().double().requires_grad_(True)
    y = lam * x + torch.exp(E @ E.T) @ x
    (y * gy.cpu().double()).sum().backward()
    return E.grad, x.grad, y.detach()


def rel(a, b):
    a, b = a.detach().cpu().double(), b.detach().cpu().double()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 1e-4)])
@pytest.mark.parametrize("k", [0, 3])
def test_operator_gradients(cuda, dtype, tol, k):
    from laker_b200 import AttentionKernelOperator

    g = torch.Generator().manual_seed(7 + k)
    n, d, lam = 700, 6, 0.05
    E0 = torch.randn(n, d, generator=g, dtype=torch.float64) * 0.4
    shape = (n,) if k == 0 else (n, k)
    x0 = torch.randn(*shape, generator=g, dtype=torch.float64)
    gy = torch.randn(*shape, generator=g, dtype=torch.float64)
    E = E0.to(cuda, dtype).requires_grad_(True)
    x = x0.to(cuda, dtype).requires_grad_(True)
    op = AttentionKernelOperator(E, lambda_reg=lam)
    y = op.matvec(x)
    (y * gy.to(cuda, dtype)).sum().backward()
    gE_ref, gx_ref, y_ref = _dense_grads(E0.to(dtype), x0.to(dtype), gy, lam)
    assert rel(y, y_ref) < tol
    assert rel(x.grad, gx_ref) < tol
    assert rel(E.grad, gE_ref) < tol
    # no grad requested: the plain path, same values
    with torch.no_grad():
        assert rel(op.matvec(x), y_ref) < tol


def test_clamped_operator_gradient_raises(cuda):
    from laker_b200 import AttentionKernelOperator

    E = (torch.randn(64, 4, dtype=torch.float64) * 20.0).to(cuda).requires_grad_(True)
    op = AttentionKernelOperator(E, lambda_reg=0.1)
    assert not op.skip_clamp
    y = op.matvec(torch.randn(64, dtype=torch.float64, device=cuda))
    with pytest.raises(NotImplementedError):
        y.sum().backward()
