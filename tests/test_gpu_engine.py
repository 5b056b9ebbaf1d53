"""GPU tests of the continuous-batching solve engine (laker_engine_*).

An instance admitted while others are iterating, or moved down when the
arenas are compacted, must give the same bits as the same instance solved
alone; every result is held to the single solve's bar (true float64 relative
residual <= tol, checked with the float64 oracle).
"""

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu


def make_problem(cuda, n, seed, lam=None, d=6, with_pc=True):
    from laker_b200 import AttentionKernelOperator, CCCPPreconditioner

    rng = np.random.default_rng(seed)
    E = (rng.standard_normal((n, d)) * 0.5).astype(np.float32)
    lam = lam if lam is not None else float(10 ** rng.uniform(-1.7, -1))
    op = AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=lam)
    pre = None
    if with_pc:
        pre = CCCPPreconditioner(num_probes=min(60, n), max_iter=40, verbose=False, device=cuda,
                                 dtype=torch.float32).build(op.matvec, n, seed=seed)
    b = torch.tensor(rng.standard_normal(n), device=cuda)
    return op, pre, b, E.astype(np.float64)


def solo(cuda, op, pre, b, tol=1e-7):
    from laker_b200 import SolveEngine

    eng = SolveEngine(max_slots=1, max_points=op.n, d=op.embedding_dim, max_nr=pre.nr if pre else 0,
                      tol=tol, max_iter=3000, device=cuda)
    slot = eng.admit(op, pre, b)
    out = eng.solve_all()
    eng.release()
    return out[slot]


def test_engine_solves_and_matches_solo(cuda, k1t_logits):
    from laker_b200 import SolveEngine

    probs = [make_problem(cuda, n, s) for s, n in enumerate([300, 1100, 77, 2049])]
    eng = SolveEngine(max_slots=8, max_points=8192, d=6, max_nr=60, tol=1e-7, max_iter=3000, device=cuda)
    slots = [eng.admit(op, pre, b) for op, pre, b, _ in probs]
    out = eng.solve_all()
    for slot, (op, pre, b, E) in zip(slots, probs):
        x, res = out[slot]
        assert res.status == 0
        assert O.relres(E, op.lambda_reg, x.cpu().numpy(), b.cpu().numpy()) <= 1e-7
        x1, res1 = solo(cuda, op, pre, b)
        assert torch.equal(x, x1)
        assert res.iterations == res1.iterations


def test_engine_admits_while_running(cuda):
    from laker_b200 import SolveEngine

    a = make_problem(cuda, 1500, 10)
    b_ = make_problem(cuda, 700, 11)
    c = make_problem(cuda, 2500, 12)
    eng = SolveEngine(max_slots=4, max_points=8192, d=6, max_nr=60, tol=1e-7, max_iter=3000, chunk=4, device=cuda)
    sa = eng.admit(*a[:3])
    eng.step()
    eng.step()
    sb = eng.admit(*b_[:3])  # joins while a is iterating
    eng.step()
    sc = eng.admit(*c[:3])
    got = eng.solve_all()
    for slot, prob in ((sa, a), (sb, b_), (sc, c)):
        x1, _ = solo(cuda, *prob[:3])
        assert torch.equal(got[slot][0], x1)


def test_engine_capacity_and_compaction(cuda):
    from laker_b200 import EngineCapacityError, SolveEngine

    a = make_problem(cuda, 600, 20)    # 2 blocks
    bb = make_problem(cuda, 900, 21)   # 2 blocks
    c = make_problem(cuda, 1000, 22)   # 2 blocks
    eng = SolveEngine(max_slots=2, max_points=4 * 512, max_pairs=6, d=6, max_nr=60, tol=1e-7,
                      max_iter=3000, device=cuda)
    sa = eng.admit(*a[:3])
    sb = eng.admit(*bb[:3])
    with pytest.raises(EngineCapacityError):
        eng.admit(*c[:3])  # no slot left
    while sa not in eng.finished():
        eng.step()
    xa, _ = eng.collect(sa)  # leaves a hole below b
    sc = eng.admit(*c[:3])   # fits only after b is moved down
    got = eng.solve_all()
    for x, prob in ((xa, a), (got[sb][0], bb), (got[sc][0], c)):
        x1, _ = solo(cuda, *prob[:3])
        assert torch.equal(x, x1)


def test_engine_edge_statuses(cuda):
    from laker_b200 import SolveEngine

    op, pre, b, E = make_problem(cuda, 400, 30, with_pc=False)
    eng = SolveEngine(max_slots=3, max_points=4096, d=6, tol=1e-8, max_iter=6, device=cuda)
    s0 = eng.admit(op, None, torch.zeros_like(b))
    bn = b.clone()
    bn[5] = float("nan")
    s1 = eng.admit(op, None, bn)
    s2 = eng.admit(op, None, b)  # 6 iterations are not enough without a preconditioner
    out = eng.solve_all()
    assert out[s0][1].status == 0 and torch.count_nonzero(out[s0][0]).item() == 0
    assert out[s1][1].status == 5  # LAKER_ERR_NONFINITE
    assert out[s2][1].status == 4 and out[s2][1].iterations == 6
