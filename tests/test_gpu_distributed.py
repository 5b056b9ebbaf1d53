"""Row-sharded operator and solve on the GPU kernels.

* RowShard products over every shard of 2 and 3-way splits (uneven, ragged
  row counts) assembled in one process and compared with the float64 oracle.
* sharded_pcg_solve on one shard holding every row, with the real kernels
  and the CCCP factors, against the oracle's residual.
* Two ranks of a gloo process group on one GPU running
  LAKERRegressor(distributed=True): fit (sharded solve), predict and
  predict_variance (the 2-D solve over the sharded products) against a
  single-process fit.  The ranks exchange on the host only (gloo), so none of
  their kernels waits on the other's.
"""

import os
import socket
import tempfile
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

F32_RTOL = 3e-5
F64_RTOL = 1e-12


def rel(a, b):
    a = a.detach().cpu().double().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = b.detach().cpu().double().numpy() if torch.is_tensor(b) else np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("n,world", [(1029, 3), (4097, 2), (5, 3), (2, 3)])
def test_row_shards_assemble_the_operator(cuda, n, world):
    from laker_b200 import AttentionKernelOperator
    from laker_b200.distributed import RowShard, shard_bounds

    rng = np.random.default_rng(n)
    E = rng.standard_normal((n, 10)) * 0.5
    x = rng.standard_normal(n)
    X = rng.standard_normal((n, 3))
    b = rng.standard_normal(n)
    lam = 0.02
    op32 = AttentionKernelOperator(torch.tensor(E, device=cuda).float(), lambda_reg=lam)
    op64 = AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=lam)
    E32 = E.astype(np.float32).astype(np.float64)
    xt = torch.tensor(x, device=cuda)
    Xt = torch.tensor(X, device=cuda)
    y32, y64, Y64, res = [], [], [], []
    for r0, r1 in shard_bounds(n, world):
        s32, s64 = RowShard(op32, r0, r1), RowShard(op64, r0, r1)
        y32.append(s32.apply32(xt, lam))
        y64.append(s64.apply64(xt, lam))
        Y64.append(s64.apply64(Xt, lam))
        res.append(s64.residual64(xt, torch.tensor(b[r0:r1], device=cuda)))
    assert rel(torch.cat(y32), O.attention_matvec(E32, lam, x)) < F32_RTOL
    assert rel(torch.cat(y64), O.attention_matvec(E, lam, x)) < F64_RTOL
    assert rel(torch.cat(Y64), O.attention_matvec(E, lam, X)) < F64_RTOL
    assert rel(torch.cat(res), b - O.attention_matvec(E, lam, x)) < 1e-10


def test_sharded_loop_on_one_shard(cuda):
    from laker_b200 import AttentionKernelOperator, CCCPPreconditioner
    from laker_b200.distributed import (RowExchange, RowShard, ShardedPreconditioner,
                                        sharded_pcg_solve)

    n, lam = 3000, 1e-2
    rng = np.random.default_rng(7)
    E = rng.standard_normal((n, 10)) * 0.5
    b = rng.standard_normal(n)
    op = AttentionKernelOperator(torch.tensor(E, device=cuda).float(), lambda_reg=lam)
    pc = CCCPPreconditioner(num_probes=120, verbose=False, device=cuda,
                            dtype=torch.float32).build(op.matvec, n, seed=1)
    exch = RowExchange(n)
    x, info = sharded_pcg_solve(RowShard(op, 0, n), exch, torch.tensor(b, device=cuda),
                                precond=ShardedPreconditioner.from_cccp(pc, 0, n), tol=1e-8,
                                max_iter=2000)
    assert info.status == 0 and info.accurate_matvecs >= 1
    E32 = E.astype(np.float32).astype(np.float64)
    assert O.relres(E32, lam, x.cpu().numpy(), b) <= 1e-8
    # the fused single-GPU solve reaches the same solution
    from laker_b200 import PreconditionedConjugateGradient

    pcg = PreconditionedConjugateGradient(tol=1e-8, max_iter=2000, verbose=False)
    xf = pcg.solve(op.matvec, pc.apply, torch.tensor(b, device=cuda))
    assert rel(x, xf) < 1e-6
    assert abs(info.iterations - pcg.iterations) <= max(3, pcg.iterations // 10)


def _fit_worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from laker_b200 import LAKERRegressor
        from laker_b200.data import synthetic_field

        x, y, _ = synthetic_field(3500, 3)
        dev = torch.device("cuda", 0)
        reg = LAKERRegressor(device=dev, verbose=False, distributed=True).fit(x, y, seed=3)
        op = reg.kernel_operator
        xq = torch.rand(64, 2, generator=torch.Generator().manual_seed(5)) * 100.0
        out = {"pred": reg.predict(xq).cpu(), "var": reg.predict_variance(xq[:16]).cpu(),
               "iters": reg.pcg_iterations_, "alpha": reg.alpha.cpu(),
               "single": op.single_device, "chunks": op.chunk_sizes,
               "devices": [str(d) for d in op.devices], "type": type(op).__name__}
        torch.save(out, os.path.join(out_dir, f"{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_fit_matches_single_process(cuda):
    from laker_b200 import LAKERRegressor
    from laker_b200.data import synthetic_field

    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_fit_worker, args=(2, _free_port(), d), nprocs=2, join=True,
                           start_method="spawn")
        outs = [torch.load(os.path.join(d, f"{r}.pt"), weights_only=False) for r in range(2)]
    x, y, _ = synthetic_field(3500, 3)
    reg = LAKERRegressor(device=cuda, verbose=False).fit(x, y, seed=3)
    xq = torch.rand(64, 2, generator=torch.Generator().manual_seed(5)) * 100.0
    pred, var = reg.predict(xq).cpu(), reg.predict_variance(xq[:16]).cpu()
    for o in outs:
        assert o["type"] == "DistributedAttentionKernelOperator" and not o["single"]
        assert o["chunks"] == [1750, 1750] and o["devices"] == ["cuda:0", "cuda:0"]
        assert torch.equal(o["pred"], outs[0]["pred"]) and torch.equal(o["var"], outs[0]["var"])
        # both solves stop at a float64 residual of 1e-6: the solutions and
        # predictions agree to that order
        assert rel(o["alpha"], reg.alpha) < 1e-4
        assert rel(o["pred"], pred) < 1e-5
        # the variance k(x,x) - k^T A^-1 k is a difference of terms of order
        # exp(|e_q|^2) (1..25 here) leaving ~1e-3: two solves at a 1e-6
        # residual agree to ~1e-6 of the terms, absolutely
        assert float((o["var"] - var).abs().max()) < 2e-5
        assert abs(o["iters"] - reg.pcg_iterations_) <= max(5, reg.pcg_iterations_ // 10)
