"""The custom ops on the GPU: torch.library.opcheck (schema: no input is
mutated, outputs do not alias inputs; fake implementation: same shapes,
dtypes and devices as the real run) and the ops' results against the float64
oracle, including the fused PCG solve called as an op."""

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

CHECKS = ("test_schema", "test_faketensor")


def rel(a, b):
    a = a.detach().cpu().double().numpy()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_opcheck_and_oracle(cuda):
    ops = torch.ops.laker_b200
    n, d, lam = 700, 10, 0.02
    rng = np.random.default_rng(3)
    E = rng.standard_normal((n, d)) * 0.5
    x = rng.standard_normal(n)
    X = rng.standard_normal((n, 5))
    Et = torch.tensor(E, device=cuda)
    xt, Xt = torch.tensor(x, device=cuda), torch.tensor(X, device=cuda)
    torch.library.opcheck(ops.pack.default, (Et.float(), 32), test_utils=CHECKS)
    torch.library.opcheck(ops.pack.default, (Et, 64), test_utils=CHECKS)
    p32, p64 = ops.pack(Et.float(), 32), ops.pack(Et, 64)
    for args in ((p32, n, p32, n, d, lam, False, xt), (p64, n, p64, n, d, lam, False, Xt),
                 (p64, 300, p64, n, d, 0.0, False, xt)):
        torch.library.opcheck(ops.attn_matvec.default, args, test_utils=CHECKS)
    E32 = E.astype(np.float32).astype(np.float64)
    assert rel(ops.attn_matvec(p32, n, p32, n, d, lam, False, xt), O.attention_matvec(E32, lam, x)) < 3e-5
    assert rel(ops.attn_matvec(p64, n, p64, n, d, lam, False, Xt), O.attention_matvec(E, lam, X)) < 1e-12
    bt = torch.tensor(x[::-1].copy(), device=cuda)
    args = (p64, n, p64, n, d, lam, False, xt, bt)
    torch.library.opcheck(ops.attn_residual.default, args, test_utils=CHECKS)
    assert rel(ops.attn_residual(*args), x[::-1] - O.attention_matvec(E, lam, x)) < 1e-10
    torch.library.opcheck(ops.attn_diagonal.default, (p64, n, d, lam), test_utils=CHECKS)
    assert rel(ops.attn_diagonal(p64, n, d, lam), O.diagonal(E, lam)) < 1e-14
    torch.library.opcheck(ops.kernel_eval.default, (p64, n, p64, 9, d, False, True), test_utils=CHECKS)
    assert rel(ops.kernel_eval(p64, n, p64, 9, d, False, True), O.kernel_eval(E, E[:9])) < 1e-14


def test_solve_and_precond_ops(cuda):
    from laker_b200 import AttentionKernelOperator, CCCPPreconditioner
    from laker_b200 import ops as L_ops

    ops = torch.ops.laker_b200
    n, lam = 2500, 1e-2
    rng = np.random.default_rng(9)
    E = rng.standard_normal((n, 10)) * 0.5
    b = rng.standard_normal(n)
    op = AttentionKernelOperator(torch.tensor(E, device=cuda).float(), lambda_reg=lam)
    pc = CCCPPreconditioner(num_probes=100, verbose=False, device=cuda,
                            dtype=torch.float32).build(op.matvec, n, seed=2)
    bt = torch.tensor(b, device=cuda)
    cis = pc.isotropic_coef ** -0.5
    q32, w32, nr, cis = pc.apply_factors()
    pargs = (q32, w32, n, nr, cis, bt, True)
    torch.library.opcheck(ops.precond_apply.default, pargs, test_utils=CHECKS)
    assert torch.equal(ops.precond_apply(*pargs), pc.apply(bt))
    p = op.packed
    sargs = (p.packed32, p.packed64, n, 10, lam, False, q32, w32, nr, cis, bt, None,
             1e-8, 2000, 0.03, 1e-8, 0, False)
    torch.library.opcheck(ops.pcg_solve.default, sargs, test_utils=CHECKS)
    x, stats = ops.pcg_solve(*sargs)
    res = L_ops.result_from_stats(stats)
    assert res.status == 0 and res.iterations > 0 and res.accurate_matvecs >= 1
    E32 = E.astype(np.float32).astype(np.float64)
    assert O.relres(E32, lam, x.cpu().numpy(), b) <= 1e-8
    assert abs(res.residual_norm / res.rhs_norm - O.relres(E32, lam, x.cpu().numpy(), b)) < 1e-9
