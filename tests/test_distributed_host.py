"""Row-sharded solve on the CPU: gloo process groups of 2 and 3 ranks.

The exchange (RowExchange), the sharded preconditioner and the solve loop
(sharded_pcg_solve) run as they do on GPUs; only the rows of the operator come
from a test shard over the float64 oracle instead of the CUDA kernels (the
FP32 product is rounded to float32, as the kernel's output is).  Results are
checked against a dense float64 solve, across ranks (every rank must return
the same bits) and against the reference's split of the rows
(laker/distributed_kernels.py:140-182).
"""

import math
import os
import socket
import sys
import tempfile
from datetime import timedelta
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

from oracle import laker_oracle as O  # noqa: E402


class OracleShard:
    """Rows [r0, r1) of lam I + exp(E E^T) from the float64 oracle."""

    def __init__(self, E, lam, r0, r1):
        self.E, self.lam, self.r0, self.r1 = E, float(lam), r0, r1

    def apply32(self, xf, lam):
        xs = xf.double().numpy()
        y = O.rect_matvec(self.E[self.r0:self.r1], self.E, xs) + lam * xs[self.r0:self.r1]
        return torch.tensor(y, dtype=torch.float32)

    def residual64(self, xf, b_loc):
        xs = xf.double().numpy()
        y = O.rect_matvec(self.E[self.r0:self.r1], self.E, xs) + self.lam * xs[self.r0:self.r1]
        return b_loc.double() - torch.tensor(y)


def _problem(n, d=6, seed=0, scale=0.4):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, d)) * scale, rng.standard_normal(n)


def _cccp_factors(E, lam, nr, seed=1):
    """The oracle's CCCP state folded into (Q, W, c^-1/2) as the apply uses it."""
    n = E.shape[0]
    probes = np.random.default_rng(seed).standard_normal((n, nr))
    st = O.cccp_build(lambda X: O.attention_matvec(E, lam, X), n, probes, gamma=0.1, max_iter=50)
    cis = st["isotropic_coef"] ** -0.5
    v = st["q_eigenvectors"]
    w = (v * (st["q_eigenvalues"] ** -0.5 - cis)[None, :]) @ v.T
    return st["q_basis"], w, cis


def _solve_case(rank, world, n, lam, nr, tol, **kw):
    from laker_b200.distributed import RowExchange, ShardedPreconditioner, sharded_pcg_solve

    E, b = _problem(n)
    exch = RowExchange(n)
    pre = None
    if nr:
        q, w, cis = _cccp_factors(E, lam, nr)
        pre = ShardedPreconditioner(torch.tensor(q[exch.r0:exch.r1]), torch.tensor(w), cis)
    shard = OracleShard(E, lam, exch.r0, exch.r1)
    x, info = sharded_pcg_solve(shard, exch, torch.tensor(b), precond=pre, tol=tol, **kw)
    return {"x": x, "iterations": info.iterations, "status": info.status,
            "accurate": info.accurate_matvecs, "residual": info.residual_norm,
            "bounds": exch.bounds}


def _edge_case(rank, world):
    from laker_b200 import _lib
    from laker_b200.distributed import RowExchange, ShardedSolveInfo, sharded_pcg_solve

    n, lam = 40, 0.1
    E, b = _problem(n, seed=3)
    exch = RowExchange(n)
    shard = OracleShard(E, lam, exch.r0, exch.r1)
    out = {}
    # gather of 1-D and 2-D rows
    rows = torch.arange(exch.r0, exch.r1, dtype=torch.float64)
    out["gather1"] = exch.gather(rows)
    out["gather2"] = exch.gather(torch.stack([rows, -rows], dim=1))
    # zero rhs: zeros, no iteration
    x, info = sharded_pcg_solve(shard, exch, torch.zeros(n))
    out["zero"] = (float(x.abs().sum()), info.iterations, info.status)
    # NaN in the rhs: the same RuntimeError on every rank
    bad = torch.tensor(b)
    bad[5] = float("nan")
    try:
        sharded_pcg_solve(shard, exch, bad)
        out["nan"] = "no error"
    except RuntimeError as e:
        out["nan"] = str(e)
    # indefinite operator: breakdown on every rank
    neg = OracleShard(E, -1e4, exch.r0, exch.r1)
    info = ShardedSolveInfo()
    try:
        sharded_pcg_solve(neg, exch, torch.tensor(b), info=info)
        out["breakdown"] = "no error"
    except RuntimeError as e:
        out["breakdown"] = (str(e), info.status)
    # max_iter: not converged, x returned
    x, info = sharded_pcg_solve(shard, exch, torch.tensor(b), tol=1e-14, max_iter=3)
    out["short"] = (info.iterations, info.status, info.accurate_matvecs)
    # warm start from the solution
    x, info = sharded_pcg_solve(shard, exch, torch.tensor(b), tol=1e-12, max_iter=300)
    x2, info2 = sharded_pcg_solve(shard, exch, torch.tensor(b), tol=1e-10, max_iter=300, x0=x)
    out["warm"] = (info.iterations, info2.iterations, float((x2 - x).norm() / x.norm()))
    out["ok"] = _lib.LAKER_OK
    return out


CASES = {
    "cccp": lambda rank, world: _solve_case(rank, world, 301, 0.05, 40, 1e-10),
    # max_iter above n: the FP32 recurrence needs a few restarts to 1e-12
    "identity": lambda rank, world: _solve_case(rank, world, 7, 0.5, 0, 1e-12, max_iter=200),
    "tiny": lambda rank, world: _solve_case(rank, world, 2, 0.5, 0, 1e-12, max_iter=200),
    "edge": _edge_case,
}


def _worker(rank, world, port, case, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.set_num_threads(1)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        torch.save(CASES[case](rank, world), os.path.join(out_dir, f"{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(case, world):
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), case, d), nprocs=world,
                           join=True, start_method="spawn")
        return [torch.load(os.path.join(d, f"{r}.pt"), weights_only=False) for r in range(world)]


def _dense_solution(n, lam):
    E, b = _problem(n)
    return np.linalg.solve(O.to_dense(E, lam), b), E, b


def test_shard_bounds_match_reference_split():
    from laker_b200.distributed import shard_bounds

    # n // G each, the first n % G one more (distributed_kernels.py:160-166)
    assert shard_bounds(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert shard_bounds(2, 3) == [(0, 1), (1, 2), (2, 2)]
    assert shard_bounds(0, 2) == [(0, 0), (0, 0)]
    for n in (1, 7, 100, 100001):
        for g in (1, 2, 3, 8):
            b = shard_bounds(n, g)
            sizes = [e - s for s, e in b]
            assert b[0][0] == 0 and b[-1][1] == n and sum(sizes) == n
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        shard_bounds(5, 0)


def test_single_process_solve_without_group():
    """No process group: one shard holds every row."""
    res = _solve_case(0, 1, 301, 0.05, 40, 1e-10)
    ref, E, b = _dense_solution(301, 0.05)
    assert res["bounds"] == [(0, 301)]
    assert res["status"] == 0
    assert O.relres(E, 0.05, res["x"].numpy(), b) <= 1e-10
    assert np.linalg.norm(res["x"].numpy() - ref) / np.linalg.norm(ref) < 1e-8


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_cccp_solve(world):
    outs = run_ranks("cccp", world)
    ref, E, b = _dense_solution(301, 0.05)
    single = _solve_case(0, 1, 301, 0.05, 40, 1e-10)
    for o in outs:
        assert o["status"] == 0
        assert torch.equal(o["x"], outs[0]["x"])  # the same bits on every rank
        assert o["iterations"] == outs[0]["iterations"]
    x = outs[0]["x"].numpy()
    assert O.relres(E, 0.05, x, b) <= 1e-10
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-8
    # the sharded recurrence is the single-shard one up to summation order
    assert abs(outs[0]["iterations"] - single["iterations"]) <= 2
    assert outs[0]["bounds"] == [tuple(t) for t in outs[0]["bounds"]]


@pytest.mark.parametrize("case,world", [("identity", 3), ("tiny", 3), ("identity", 2)])
def test_sharded_uneven_and_empty_shards(case, world):
    """Shards of unequal size, and a rank that holds no row at all (n = 2)."""
    n = 7 if case == "identity" else 2
    outs = run_ranks(case, world)
    ref, E, b = _dense_solution(n, 0.5)
    for o in outs:
        assert o["status"] == 0
        assert torch.equal(o["x"], outs[0]["x"])
        assert np.linalg.norm(o["x"].numpy() - ref) / np.linalg.norm(ref) < 1e-10
    if case == "tiny":
        assert outs[0]["bounds"][2] == (2, 2)


def test_sharded_edge_cases():
    outs = run_ranks("edge", 2)
    n = 40
    for o in outs:
        assert torch.equal(o["gather1"], torch.arange(n, dtype=torch.float64))
        assert torch.equal(o["gather2"][:, 1], -torch.arange(n, dtype=torch.float64))
        assert o["zero"] == (0.0, 0, o["ok"])
        assert "non-finite" in o["nan"]
        msg, status = o["breakdown"]
        assert "breakdown" in msg
        its, status, accurate = o["short"]
        assert its == 3 and status != o["ok"] and accurate >= 1
        cold, warm, rel = o["warm"]
        # at least one iteration runs; from the solution only a few are needed
        assert 1 <= warm <= max(10, cold // 5)
        assert rel < 1e-8
    assert outs[0]["breakdown"] == outs[1]["breakdown"]


def test_exchange_without_group_is_identity():
    from laker_b200.distributed import RowExchange

    e = RowExchange(5)
    assert (e.world, e.rank, e.r0, e.r1) == (1, 0, 0, 5)
    v = torch.arange(5.0)
    assert torch.equal(e.gather(v), v)
    t = torch.ones(3)
    assert torch.equal(e.sum_(t), torch.ones(3))
    with pytest.raises(ValueError):
        e.gather(torch.zeros(4))
    assert not math.isnan(float(e.sum_(torch.zeros(1))[0]))
