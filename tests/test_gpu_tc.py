"""GPU parity of the tensor-core (tcgen05, split TF32) multi-RHS matvec.

The multi-RHS FP32 operator (k > 1) evaluates entries on the CUDA cores and
contracts them with X on the tensor cores as P_hi X_hi + P_hi X_lo + P_lo X_hi
(TF32 parts, FP32 accumulation).  Each product carries ~2^-21 relative error
(the dropped P_lo X_lo term and the TF32 rounding of the lo parts), and a
column of K X with mixed-sign X cancels, so the bar is the reference's own
float32 tolerance: 1e-4 relative per column against the float64 oracle on the
FP32-rounded embeddings (measured 1e-6 .. 5e-5).
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


@pytest.mark.parametrize("n,k", [(1, 2), (31, 5), (33, 16), (257, 17), (700, 64), (1500, 256),
                                 (1029, 300), (2048, 512)])
def test_tc_square_matvec(cuda, n, k):
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(n * 1000 + k)
    E = (rng.standard_normal((n, 10)) * 0.5).astype(np.float32)
    X = rng.standard_normal((n, k))
    op = AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=0.03)
    Y = op.matvec(torch.tensor(X, device=cuda, dtype=torch.float32))
    assert Y.shape == (n, k)
    assert colrel(Y, O.attention_matvec(E, 0.03, X)) < TC_RTOL


@pytest.mark.parametrize("d", [1, 4, 7, 16])
def test_tc_dims_and_rectangular(cuda, d):
    from laker_b200 import _lib

    rng = np.random.default_rng(40 + d)
    n, m, k = 900, 333, 48
    E = (rng.standard_normal((n, d)) * 0.7 / np.sqrt(d)).astype(np.float32)
    Eq = (rng.standard_normal((m, d)) * 0.7 / np.sqrt(d)).astype(np.float32)
    X = rng.standard_normal((n, k)).astype(np.float32)
    Et, Eqt = torch.tensor(E, device=cuda), torch.tensor(Eq, device=cuda)
    Y = _lib.attn_matvec_f32(_lib.pack_f32(Eqt), m, _lib.pack_f32(Et), n, d, 0.0, 0,
                             torch.tensor(X, device=cuda))
    ref = O.rect_matvec(Eq.astype(np.float64), E.astype(np.float64), X.astype(np.float64))
    assert colrel(Y, ref) < TC_RTOL


def test_tc_linearity_and_repeatability(cuda):
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(3)
    n, k = 1200, 40
    E = torch.tensor((rng.standard_normal((n, 10)) * 0.5).astype(np.float32), device=cuda)
    op = AttentionKernelOperator(E, lambda_reg=0.01)
    A = torch.randn(n, k, device=cuda)
    B = torch.randn(n, k, device=cuda)
    lhs = op.matvec(2.0 * A - 0.5 * B)
    rhs = 2.0 * op.matvec(A) - 0.5 * op.matvec(B)
    assert (torch.linalg.norm(lhs - rhs) / torch.linalg.norm(rhs)).item() < 1e-5
    # deterministic: the same call twice gives the same bits
    assert torch.equal(op.matvec(A), op.matvec(A))
    # columns agree with the single-RHS operator
    y0 = op.matvec(A[:, 7].contiguous())
    assert (torch.linalg.norm(op.matvec(A)[:, 7] - y0) / torch.linalg.norm(y0)).item() < TC_RTOL


_LOGITS_TC_CHILD = r"""
import numpy as np, torch
from oracle import laker_oracle as O
from laker_b200 import AttentionKernelOperator, _lib
cuda = torch.device("cuda", 0)
def colrel(Y, ref):
    Y = Y.detach().cpu().double().numpy()
    return float((np.linalg.norm(Y - ref, axis=0) / np.maximum(np.linalg.norm(ref, axis=0), 1e-300)).max())
worst = 0.0
for n, k in ((257, 17), (1500, 256), (2048, 512), (3000, 16)):
    rng = np.random.default_rng(n * 1000 + k)
    E = (rng.standard_normal((n, 10)) * 0.5).astype(np.float32)
    X = rng.standard_normal((n, k))
    op = AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=0.03)
    worst = max(worst, colrel(op.matvec(torch.tensor(X, device=cuda, dtype=torch.float32)),
                              O.attention_matvec(E, 0.03, X)))
rng = np.random.default_rng(47)
n, m, k, d = 900, 333, 48, 7
E = (rng.standard_normal((n, d)) * 0.7 / np.sqrt(d)).astype(np.float32)
Eq = (rng.standard_normal((m, d)) * 0.7 / np.sqrt(d)).astype(np.float32)
X = rng.standard_normal((n, k)).astype(np.float32)
Et, Eqt = torch.tensor(E, device=cuda), torch.tensor(Eq, device=cuda)
Y = _lib.attn_matvec_f32(_lib.pack_f32(Eqt), m, _lib.pack_f32(Et), n, d, 0.0, 0, torch.tensor(X, device=cuda))
worst = max(worst, colrel(Y, O.rect_matvec(Eq.astype(np.float64), E.astype(np.float64), X.astype(np.float64))))
print("WORST", worst)
"""


def test_tc_logits_on_tensor_cores_variant(cuda):
    """The opt-in variant with the logits on the tensor cores too
    (LAKER_K2_LOGITS_TC=1, read once per process, hence a child process):
    square and rectangular products to the same per-column tolerance."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, LAKER_K2_LOGITS_TC="1", PYTHONPATH=str(root))
    out = subprocess.run([sys.executable, "-c", _LOGITS_TC_CHILD], cwd=root, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    worst = float(out.stdout.split("WORST")[-1])
    assert worst < TC_RTOL
