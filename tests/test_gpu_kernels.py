"""GPU parity of the fused kernels against the float64 oracle and the goldens.

Tolerances: the FP32 operator carries FP32 entries (ex2.approx, FP32 logits),
so it is held to 3e-5 relative per output; its multi-RHS form contracts on the
tensor cores in split TF32 (~2^-21 per product) and is held to the reference's
own float32 test tolerance, 1e-4; FP64 kernels are held to 1e-12.
"""

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

F32_RTOL = 3e-5
F32_MULTI_RTOL = 1e-4
F64_RTOL = 1e-12


def rel(a, b):
    a = a.detach().cpu().double().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = b.detach().cpu().double().numpy() if torch.is_tensor(b) else np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("key", ["n30_d4", "n100_d6", "n257_d10", "n1000_d10"])
def test_matvec_golden(cuda, golden, key):
    from laker_b200 import AttentionKernelOperator

    g = golden("kernels")
    E = torch.tensor(g[f"{key}_E"], device=cuda)
    for dtype, tol in ((torch.float32, F32_RTOL), (torch.float64, F64_RTOL)):
        op = AttentionKernelOperator(E.to(dtype), lambda_reg=0.05)
        x = torch.tensor(g[f"{key}_x"], device=cuda, dtype=dtype)
        X = torch.tensor(g[f"{key}_X"], device=cuda, dtype=dtype)
        assert rel(op.matvec(x), g[f"{key}_matvec"]) < tol
        assert rel(op.matvec(X), g[f"{key}_matvec2d"]) < (F32_MULTI_RTOL if dtype == torch.float32 else tol)
        assert rel(op.diagonal(), g[f"{key}_diag"]) < max(tol, 1e-6 if dtype == torch.float32 else 0)
        q = torch.tensor(g[f"{key}_q"], device=cuda, dtype=dtype)
        assert rel(op.kernel_eval(q), g[f"{key}_keval"]) < max(tol, 1e-6 if dtype == torch.float32 else 0)


@pytest.fixture(params=["default", "symmetric", "symmetric-f16"])
def sym_route(request):
    """Run with the default routing (small square operators on the plain
    kernel), with the symmetric kernels forced down to one block, and the
    same with the tensor-core kernel's split-FP16 logits."""
    from laker_b200 import _lib

    if request.param == "default":
        yield request.param
        return
    prev = _lib.set_variant(_lib.VARIANT_SYM_MIN_BLOCKS, 0)
    prev_f = _lib.set_variant(_lib.VARIANT_K1T_LOGITS, 1 if request.param.endswith("f16") else 0)
    try:
        yield request.param
    finally:
        _lib.set_variant(_lib.VARIANT_SYM_MIN_BLOCKS, prev)
        _lib.set_variant(_lib.VARIANT_K1T_LOGITS, prev_f)



@pytest.mark.parametrize("n", [1, 2, 3, 255, 256, 257, 511, 513, 1029, 4097])
def test_matvec_ragged_sizes(cuda, n, sym_route):
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(n)
    E = rng.standard_normal((n, 10)) * 0.5
    x = rng.standard_normal(n)
    ref = O.attention_matvec(E, 0.01, x)
    Et = torch.tensor(E, device=cuda)
    op64 = AttentionKernelOperator(Et, lambda_reg=0.01)
    op32 = AttentionKernelOperator(Et.float(), lambda_reg=0.01)
    assert rel(op64.matvec(torch.tensor(x, device=cuda)), ref) < F64_RTOL
    # FP32 operator on FP32-rounded embeddings, compared with the FP64 oracle of the same
    ref32 = O.attention_matvec(E.astype(np.float32), 0.01, x)
    assert rel(op32.matvec(torch.tensor(x, device=cuda, dtype=torch.float32)), ref32) < F32_RTOL


@pytest.mark.parametrize("n", [20000, 36100])
def test_symmetric_operator_many_pairs_per_cta(cuda, n, k1t_logits):
    """The operator at sizes where every CTA of the persistent symmetric kernel
    walks several block pairs (row-block changes, operand-stage reuse,
    accumulator-buffer wrap-around; n = 20000: 820 pairs, 36100: 2485 pairs
    over 148 CTAs), a partial last block, and repeated calls bit for bit."""
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(n)
    E = (rng.standard_normal((n, 10)) * 0.5).astype(np.float32)
    x = rng.standard_normal(n)
    ref = O.attention_matvec(E, 0.01, x)
    op32 = AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=0.01)
    xd = torch.tensor(x, device=cuda, dtype=torch.float32)
    y1 = op32.matvec(xd)
    y2 = op32.matvec(xd)
    assert torch.equal(y1, y2)
    assert rel(y1, ref) < F32_RTOL
    # per-row agreement, not only in norm: entries carry ~1e-6 relative error,
    # which a row whose sum cancels down to 1e-3 of the largest row amplifies
    # by up to ~|K||x| / |y_i|; measured worst rows 8e-5 (split TF32) and
    # 1.6e-4 (split FP16) at n = 20000, 7e-5 and 1.7e-5 at n = 36100
    err = np.abs(y1.cpu().double().numpy() - ref) / np.maximum(np.abs(ref), 1e-3 * np.abs(ref).max())
    assert err.max() < 3e-4
    assert np.quantile(err, 0.999) < 1e-4


@pytest.mark.parametrize("d", [1, 2, 3, 5, 8, 11, 16])
def test_matvec_all_dims(cuda, d, sym_route):
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(100 + d)
    n = 700
    E = (rng.standard_normal((n, d)) * 0.6 / np.sqrt(d) * 2).astype(np.float32)
    x = rng.standard_normal(n)
    X = rng.standard_normal((n, 5))
    Et = torch.tensor(E, device=cuda)
    op32 = AttentionKernelOperator(Et, lambda_reg=0.02)
    op64 = AttentionKernelOperator(Et.double(), lambda_reg=0.02)
    assert rel(op32.matvec(torch.tensor(x, device=cuda, dtype=torch.float32)),
               O.attention_matvec(E, 0.02, x)) < F32_RTOL
    assert rel(op64.matvec(torch.tensor(x, device=cuda)), O.attention_matvec(E, 0.02, x)) < F64_RTOL
    assert rel(op32.matvec(torch.tensor(X, device=cuda, dtype=torch.float32)),
               O.attention_matvec(E, 0.02, X)) < F32_MULTI_RTOL
    assert rel(op64.matvec(torch.tensor(X, device=cuda)), O.attention_matvec(E, 0.02, X)) < F64_RTOL


def test_matvec_multi_rhs_wide(cuda):
    """k = 256 right-hand sides (the CCCP probe block), ragged n."""
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(5)
    n, k = 1500, 256
    E = (rng.standard_normal((n, 10)) * 0.5).astype(np.float32)
    X = rng.standard_normal((n, k))
    ref = O.attention_matvec(E, 0.01, X)
    op32 = AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=0.01)
    Y = op32.matvec(torch.tensor(X, device=cuda, dtype=torch.float32))
    col = [rel(Y[:, c], ref[:, c]) for c in range(k)]
    assert max(col) < F32_MULTI_RTOL
    op64 = AttentionKernelOperator(torch.tensor(E, device=cuda).double(), lambda_reg=0.01)
    assert rel(op64.matvec(torch.tensor(X, device=cuda)), ref) < F64_RTOL


def test_clamp_path(cuda):
    """max ||e||^2 >= the dtype's limit: Gram entries clamped before exp."""
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(9)
    n = 300
    E = rng.standard_normal((n, 4)) * 0.3
    E[:3] *= 40.0  # a few points with ||e||^2 ~ 100-1000
    x = rng.standard_normal(n)
    E32 = E.astype(np.float32)
    op32 = AttentionKernelOperator(torch.tensor(E32, device=cuda), lambda_reg=0.01)
    assert not op32.skip_clamp
    ref32 = O.attention_matvec(E32, 0.01, x, clamp=True, clamp_value=80.0)
    assert rel(op32.matvec(torch.tensor(x, device=cuda, dtype=torch.float32)), ref32) < F32_RTOL
    E64 = E.copy()
    E64[0] *= 2.0  # ||e||^2 > 700 as well
    op64 = AttentionKernelOperator(torch.tensor(E64, device=cuda), lambda_reg=0.01)
    assert not op64.skip_clamp
    ref64 = O.attention_matvec(E64, 0.01, x, clamp=True, clamp_value=700.0)
    assert rel(op64.matvec(torch.tensor(x, device=cuda)), ref64) < 1e-11


def test_rectangular_prediction_kernel(cuda):
    from laker_b200 import _lib

    rng = np.random.default_rng(4)
    n, m = 3000, 77
    E = rng.standard_normal((n, 10)) * 0.5
    Eq = rng.standard_normal((m, 10)) * 0.5
    a = rng.standard_normal(n)
    Et = torch.tensor(E, device=cuda)
    Eqt = torch.tensor(Eq, device=cuda)
    out = _lib.attn_matvec_f64(_lib.pack_f64(Eqt), m, _lib.pack_f64(Et), n, 10, 0.0, 0,
                               torch.tensor(a, device=cuda))
    assert rel(out, O.rect_matvec(Eq, E, a)) < F64_RTOL
    # m == n rectangular product: lam must not be applied when passed as 0
    out2 = _lib.attn_matvec_f64(_lib.pack_f64(Et), n, _lib.pack_f64(Et), n, 10, 0.0, 0,
                                torch.tensor(a, device=cuda))
    assert rel(out2, O.rect_matvec(E, E, a)) < F64_RTOL


def test_precond_apply_golden(cuda, golden):
    from laker_b200 import AttentionKernelOperator, CCCPPreconditioner

    g = golden("solver_n400")
    E = torch.tensor(g["E"], device=cuda)
    op = AttentionKernelOperator(E, lambda_reg=float(g["lam"]))
    # probes from a CPU generator: the golden comes from the reference run on the CPU
    pre = CCCPPreconditioner(num_probes=60, gamma=0.1, max_iter=50, tol=1e-6, verbose=False,
                             device=cuda, dtype=torch.float64, probe_device="cpu")
    pre.build(op.matvec, E.shape[0], seed=3)
    assert abs(pre.isotropic_coef - float(g["iso"])) < 1e-8 * float(g["iso"])
    assert rel(pre.q_eigenvalues, g["q_eigenvalues"]) < 1e-8
    v = torch.tensor(g["apply_v"], device=cuda)
    assert rel(pre.apply(v), g["apply_out"]) < 1e-5  # FP32 Q and W in the fused apply
    # linearity (reference tests/test_math_correctness.py:554-584)
    u = torch.randn_like(v)
    lhs = pre.apply(2.5 * u - 1.3 * v)
    rhs = 2.5 * pre.apply(u) - 1.3 * pre.apply(v)
    assert rel(lhs, rhs) < 1e-5
    # 2-D apply agrees with 1-D columns
    V = torch.stack([u, v], dim=1)
    assert rel(pre.apply(V)[:, 1], pre.apply(v)) < 1e-5


def test_pcg_fused_solves_to_tolerance(cuda, golden, sym_route):
    from laker_b200 import AttentionKernelOperator, CCCPPreconditioner, PreconditionedConjugateGradient

    g = golden("solver_n400")
    E = torch.tensor(g["E"], device=cuda)
    b = torch.tensor(g["b"], device=cuda)
    for dtype in (torch.float32, torch.float64):
        op = AttentionKernelOperator(E.to(dtype), lambda_reg=float(g["lam"]))
        pre = CCCPPreconditioner(num_probes=60, gamma=0.1, max_iter=50, tol=1e-6, verbose=False,
                                 device=cuda, dtype=dtype).build(op.matvec, E.shape[0], seed=3)
        pcg = PreconditionedConjugateGradient(tol=1e-10, max_iter=2000, verbose=False)
        x = pcg.solve(op.matvec, pre.apply, b.to(torch.float64))
        E_used = op.embeddings.double().cpu().numpy()
        assert O.relres(E_used, float(g["lam"]), x.cpu().numpy(), g["b"]) <= 1e-10
        assert pcg.residual_norm / np.linalg.norm(g["b"]) <= 1e-10
        assert pcg.accurate_matvecs >= 1
        if dtype == torch.float64:
            assert rel(x, g["x"]) < 1e-6


def test_pcg_edge_cases(cuda):
    from laker_b200 import AttentionKernelOperator, PreconditionedConjugateGradient

    rng = np.random.default_rng(1)
    E = torch.tensor(rng.standard_normal((200, 5)) * 0.4, device=cuda, dtype=torch.float32)
    op = AttentionKernelOperator(E, lambda_reg=0.1)
    pcg = PreconditionedConjugateGradient(tol=1e-8, max_iter=300, verbose=False)
    # zero rhs -> zeros, 0 iterations
    z = pcg.solve(op.matvec, None, torch.zeros(200, device=cuda, dtype=torch.float64))
    assert torch.count_nonzero(z).item() == 0
    # rhs must be 1-D or 2-D
    with pytest.raises(ValueError):
        pcg.solve(op.matvec, None, torch.zeros(2, 100, 1, device=cuda))
    # NaN in the rhs -> RuntimeError, no hang
    b = torch.randn(200, device=cuda, dtype=torch.float64)
    b[7] = float("nan")
    with pytest.raises(RuntimeError):
        pcg.solve(op.matvec, None, b)
    # negative lambda large enough to make A indefinite -> breakdown
    bad = AttentionKernelOperator(E, lambda_reg=-1e4)
    with pytest.raises(RuntimeError, match="breakdown"):
        pcg.solve(bad.matvec, None, torch.randn(200, device=cuda, dtype=torch.float64))
    # warm start from the solution converges immediately
    b = torch.randn(200, device=cuda, dtype=torch.float64)
    x = pcg.solve(op.matvec, None, b)
    cold = pcg.iterations
    x2 = pcg.solve(op.matvec, None, b, x0=x)
    # at least one iteration runs (laker/solvers.py:224-295 tests convergence
    # after the update); from the solution the FP32 recurrence needs only a few
    assert 1 <= pcg.iterations <= max(10, cold // 5)
    assert rel(x2, x) < 1e-7
    # max_iter reached: warning path, x returned
    short = PreconditionedConjugateGradient(tol=1e-14, max_iter=3, verbose=False)
    short.solve(op.matvec, None, b)
    assert short.iterations == 3


@pytest.mark.parametrize("k", [2, 5, 16])
def test_narrow_multi_rhs_fp64_vs_oracle(cuda, k):
    """FP64 multi-RHS products of at most 16 right-hand sides (64 x 16 tiles),
    with and without a right-hand side B (the residual B - A X)."""
    from laker_b200 import _lib

    rng = np.random.default_rng(300 + k)
    n = 2100
    E = rng.standard_normal((n, 10)) * 0.5
    X = rng.standard_normal((n, k))
    B = rng.standard_normal((n, k))
    p64 = _lib.pack_f64(torch.tensor(E, device=cuda))
    Xt, Bt = torch.tensor(X, device=cuda), torch.tensor(B, device=cuda)
    ref = O.attention_matvec(E, 0.07, X)
    assert rel(_lib.attn_matvec_f64(p64, n, p64, n, 10, 0.07, 0, Xt), ref) < F64_RTOL
    assert rel(_lib.attn_matvec_f64(p64, n, p64, n, 10, 0.07, 0, Xt, B=Bt), B - ref) < F64_RTOL


_NARROW_CHILD = r"""
import numpy as np, torch
from oracle import laker_oracle as O
from laker_b200 import _lib
cuda = torch.device("cuda", 0)
out = []
for k in (2, 5, 16):
    rng = np.random.default_rng(400 + k)
    n = 1900
    E = (rng.standard_normal((n, 10)) * 0.5).astype(np.float32)
    X = rng.standard_normal((n, k))
    p32 = _lib.pack_f32(torch.tensor(E, device=cuda))
    p64 = _lib.pack_f64(torch.tensor(E, device=cuda))
    Y = _lib.attn_matvec_f32(p32, n, p32, n, 10, 0.07, 0, torch.tensor(X, device=cuda, dtype=torch.float32))
    Y64 = _lib.attn_matvec_f64(p64, n, p64, n, 10, 0.07, 0, torch.tensor(X, device=cuda))
    ref = O.attention_matvec(E, 0.07, X)
    out.append(np.linalg.norm(Y.double().cpu().numpy() - ref) / np.linalg.norm(ref))
    np.save(f"_narrow_{k}.npy", Y64.cpu().numpy())
print("WORST", max(out))
"""


def test_narrow_multi_rhs_cuda_core_paths(cuda, tmp_path):
    """The CUDA-core FP32 multi-RHS kernel (LAKER_K2_TENSOR_CORES=0; the
    switches are read once per process, hence child processes) against the
    oracle, and the narrow 64 x 16 tiles against the wide ones
    (LAKER_MULTI_NARROW=0): the same FP64 products."""
    import os
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    results = {}
    for narrow in ("1", "0"):
        d = tmp_path / narrow
        d.mkdir()
        env = dict(os.environ, LAKER_K2_TENSOR_CORES="0", LAKER_MULTI_NARROW=narrow,
                   PYTHONPATH=str(root))
        out = subprocess.run([sys.executable, "-c", _NARROW_CHILD], cwd=d, env=env,
                             capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, out.stderr[-2000:]
        assert float(out.stdout.split("WORST")[-1]) < F32_RTOL
        results[narrow] = {k: np.load(d / f"_narrow_{k}.npy") for k in (2, 5, 16)}
    for k in (2, 5, 16):
        assert np.linalg.norm(results["1"][k] - results["0"][k]) <= F64_RTOL * np.linalg.norm(results["0"][k])
