"""GPU tests of the batched solve (laker_pcg_solve_batched) and the batched
CCCP build.

Each instance of a batch is an independent regression (its own n, lambda,
embeddings and preconditioner).  The batch is held to the single solve's bar:
true float64 relative residual <= tol per instance, checked with the float64
oracle.  Row and column partial sums of the symmetric matvec are stored per
block pair and summed in a fixed order, so an instance's result must be
bitwise identical whether it is solved alone or inside any batch.
"""

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu


def make_ops(cuda, ns, d=6, seed=0, lams=None):
    from laker_b200 import AttentionKernelOperator

    rng = np.random.default_rng(seed)
    ops, Es, bs = [], [], []
    for k, n in enumerate(ns):
        E = (rng.standard_normal((n, d)) * 0.5).astype(np.float32)
        lam = lams[k] if lams is not None else float(10 ** rng.uniform(-3, -1))
        ops.append(AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=lam))
        Es.append(E.astype(np.float64))
        bs.append(rng.standard_normal(n))
    return ops, Es, bs


def solve_batch(cuda, ops, bs, pres=None, tol=1e-8, max_iter=2000):
    from laker_b200 import BatchedPCG

    pcg = BatchedPCG(tol=tol, max_iter=max_iter)
    xs = pcg.solve(ops, pres, [torch.tensor(b, device=cuda) for b in bs])
    return pcg, xs


@pytest.mark.parametrize("with_pc", [False, True])
def test_batched_solves_each_instance(cuda, with_pc):
    from laker_b200 import build_cccp_batched

    ns = [1, 300, 513, 1200, 2049, 777]
    ops, Es, bs = make_ops(cuda, ns, seed=1)
    pres = build_cccp_batched(ops, num_probes=40, max_iter=50, seeds=list(range(len(ns)))) if with_pc else None
    # without a preconditioner these systems (condition numbers up to 2e5)
    # need up to ~1500 float64 CG iterations
    tol = 1e-8
    pcg, xs = solve_batch(cuda, ops, bs, pres, tol=tol, max_iter=2000 if with_pc else 8000)
    for k, op in enumerate(ops):
        assert pcg.statuses[k] == 0, (k, pcg.statuses)
        x = xs[k].cpu().numpy()
        assert x.shape == (ns[k],)
        assert O.relres(Es[k], op.lambda_reg, x, bs[k]) <= tol
        assert pcg.residual_norms[k] <= tol * pcg.rhs_norms[k]
        assert pcg.accurate_matvecs[k] >= 1
    assert pcg.kernel_launches > 0


def test_batched_alone_equals_mix(cuda):
    from laker_b200 import build_cccp_batched

    ns = [640, 1500, 90, 1025, 2300]
    ops, Es, bs = make_ops(cuda, ns, seed=2)
    pres = build_cccp_batched(ops, num_probes=50, max_iter=50, seeds=[11, 12, 13, 14, 15])
    _, mixed = solve_batch(cuda, ops, bs, pres)
    for k in (0, 3, 4):
        pcg1, alone = solve_batch(cuda, [ops[k]], [bs[k]], [pres[k]])
        assert torch.equal(alone[0], mixed[k]), k
    # a different batch composition and order
    order = [4, 1, 0]
    _, mixed2 = solve_batch(cuda, [ops[k] for k in order], [bs[k] for k in order],
                            [pres[k] for k in order])
    for j, k in enumerate(order):
        assert torch.equal(mixed2[j], mixed[k]), k


def test_batched_matches_single_solver(cuda):
    from laker_b200 import CCCPPreconditioner, PreconditionedConjugateGradient

    ns = [700, 1800]
    ops, Es, bs = make_ops(cuda, ns, seed=3, lams=[0.01, 0.05])
    pres = [CCCPPreconditioner(num_probes=60, max_iter=60, tol=1e-6, verbose=False, device=cuda,
                               dtype=torch.float32).build(op.matvec, op.n, seed=5) for op in ops]
    pcg_b, xs = solve_batch(cuda, ops, bs, pres, tol=1e-9)
    for k, op in enumerate(ops):
        single = PreconditionedConjugateGradient(tol=1e-9, max_iter=2000, verbose=False)
        x1 = single.solve(op.matvec, pres[k].apply, torch.tensor(bs[k], device=cuda))
        # both solve to 1e-9; the solutions agree to the conditioning of A
        diff = torch.linalg.norm(x1 - xs[k]) / torch.linalg.norm(x1)
        assert diff.item() < 1e-5
        assert abs(pcg_b.iterations[k] - single.iterations) <= max(10, 0.2 * single.iterations)


def test_batched_edge_statuses(cuda):
    ns = [400, 300, 500, 256]
    ops, Es, bs = make_ops(cuda, ns, seed=4)
    bs[1] = np.zeros(ns[1])
    bs[2] = bs[2].copy()
    bs[2][17] = np.nan
    pcg, xs = solve_batch(cuda, ops, bs, tol=1e-8)
    assert pcg.statuses[1] == 0 and pcg.iterations[1] == 0
    assert torch.count_nonzero(xs[1]).item() == 0
    assert pcg.statuses[2] == 5  # LAKER_ERR_NONFINITE
    for k in (0, 3):
        assert pcg.statuses[k] == 0
        assert O.relres(Es[k], ops[k].lambda_reg, xs[k].cpu().numpy(), bs[k]) <= 1e-8
    # max_iter reached: NOT_CONVERGED, iterations capped
    pcg2, _ = solve_batch(cuda, ops[:1], bs[:1], tol=1e-14, max_iter=5)
    assert pcg2.statuses[0] == 4 and pcg2.iterations[0] == 5
    # indefinite operator (large negative lambda) -> breakdown for that instance only
    from laker_b200 import AttentionKernelOperator

    bad = AttentionKernelOperator(ops[0].embeddings, lambda_reg=-1e4)
    pcg3, _ = solve_batch(cuda, [bad, ops[3]], [bs[0], bs[3]])
    assert pcg3.statuses[0] == 3 and pcg3.statuses[1] == 0


def test_build_cccp_batched_matches_single(cuda):
    from laker_b200 import CCCPPreconditioner, build_cccp_batched

    ns = [300, 900, 1300]
    ops, _, _ = make_ops(cuda, ns, seed=6)
    seeds = [3, 4, 5]
    batched = build_cccp_batched(ops, num_probes=None, max_iter=80, tol=1e-7, seeds=seeds)
    for k, op in enumerate(ops):
        single = CCCPPreconditioner(num_probes=None, max_iter=80, tol=1e-7, verbose=False,
                                    device=cuda, dtype=torch.float32).build(op.matvec, op.n,
                                                                            seed=seeds[k])
        pb = batched[k]
        assert pb.nr == single.nr
        assert abs(pb.isotropic_coef - single.isotropic_coef) <= 1e-8 * abs(single.isotropic_coef)
        ev_b, ev_s = pb.q_eigenvalues.double(), single.q_eigenvalues.double()
        assert (torch.linalg.norm(ev_b - ev_s) / torch.linalg.norm(ev_s)).item() < 1e-8
        assert abs(pb.cccp_iterations - single.cccp_iterations) <= 1
        v = torch.randn(op.n, device=cuda, dtype=torch.float32)
        assert (torch.linalg.norm(pb.apply(v) - single.apply(v)) / torch.linalg.norm(single.apply(v))).item() < 1e-5

