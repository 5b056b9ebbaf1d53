"""Generate tests/golden/*.npz by running the LAKER reference package itself.

Run where the reference source is available, passing its path:

    python tests/golden/make_golden.py /path/to/reference

The fixtures pin the float64 oracle (oracle/laker_oracle.py) and the GPU
path.  Inputs come from laker_b200.data.synthetic_field (CPU torch draws) and
from fixed seeds; every output is produced by the reference's own classes on
the CPU in float64 (embeddings in float32, cast to float64, as the reference
does with embedding_dtype=float32).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if len(sys.argv) < 2:
    sys.exit(f"usage: python {Path(__file__).name} <path of the reference checkout>")
REF = Path(sys.argv[1])
sys.path.insert(0, str(REF))
sys.path.insert(0, str(REPO))

from laker.embeddings import PositionEmbedding  # noqa: E402
from laker.kernels import AttentionKernelOperator  # noqa: E402
from laker.models import LAKERRegressor  # noqa: E402
from laker.preconditioner import CCCPPreconditioner  # noqa: E402
from laker.solvers import PreconditionedConjugateGradient  # noqa: E402

import laker_b200.data as data  # noqa: E402

torch.set_num_threads(8)


def kernel_cases():
    """Matvec / diagonal / kernel_eval / chunking of the exact operator."""
    out = {}
    g = torch.Generator().manual_seed(7)
    for n, de in [(30, 4), (100, 6), (257, 10), (1000, 10)]:
        e = torch.randn(n, de, generator=g, dtype=torch.float64) * 0.5
        x = torch.randn(n, generator=g, dtype=torch.float64)
        X = torch.randn(n, 3, generator=g, dtype=torch.float64)
        op = AttentionKernelOperator(e, lambda_reg=0.05)
        op_chunk = AttentionKernelOperator(e, lambda_reg=0.05, chunk_size=16)
        q = torch.randn(9, de, generator=g, dtype=torch.float64) * 0.5
        key = f"n{n}_d{de}"
        out[f"{key}_E"] = e.numpy()
        out[f"{key}_x"] = x.numpy()
        out[f"{key}_X"] = X.numpy()
        out[f"{key}_q"] = q.numpy()
        out[f"{key}_matvec"] = op.matvec(x).numpy()
        out[f"{key}_matvec_chunked"] = op_chunk.matvec(x).numpy()
        out[f"{key}_matvec2d"] = op.matvec(X).numpy()
        out[f"{key}_diag"] = op.diagonal().numpy()
        out[f"{key}_keval"] = op.kernel_eval(q).numpy()
    np.savez_compressed(HERE / "kernels.npz", **out)


def paper_case():
    """The n=3 worked example (tests/test_models.py:37-88 of the reference)."""
    e = torch.tensor([[0.241, 0.444], [-0.336, 0.112], [-0.220, 0.353]], dtype=torch.float64)
    y = torch.tensor([-66.14, -65.77, -77.30], dtype=torch.float64)
    a = torch.exp(e @ e.T) + 0.1 * torch.eye(3, dtype=torch.float64)
    alpha = torch.linalg.solve(a, y)
    e_star = torch.tensor([[0.051, 0.452]], dtype=torch.float64)
    pred = (torch.exp(e_star @ e.T) @ alpha).numpy()
    np.savez_compressed(HERE / "paper_n3.npz", E=e.numpy(), y=y.numpy(), alpha=alpha.numpy(),
                        e_star=e_star.numpy(), pred=pred, lam=0.1)


def solver_case():
    """CCCP build + PCG on a seeded small attention system (float64)."""
    g = torch.Generator().manual_seed(11)
    n, de = 400, 6
    e = torch.randn(n, de, generator=g, dtype=torch.float64) * 0.6
    b = torch.randn(n, generator=g, dtype=torch.float64)
    op = AttentionKernelOperator(e, lambda_reg=1e-2)
    pre = CCCPPreconditioner(num_probes=60, gamma=0.1, max_iter=50, tol=1e-6, verbose=False,
                             device=torch.device("cpu"), dtype=torch.float64)
    pre.build(op.matvec, n, seed=3)
    probes = torch.randn(n, 60, generator=torch.Generator().manual_seed(3), dtype=torch.float64)
    pcg = PreconditionedConjugateGradient(tol=1e-10, max_iter=1000, verbose=False)
    x = pcg.solve(op.matvec, pre.apply, b)
    v = torch.randn(n, generator=g, dtype=torch.float64)
    np.savez_compressed(
        HERE / "solver_n400.npz", E=e.numpy(), b=b.numpy(), probes=probes.numpy(), x=x.numpy(),
        iterations=pcg.iterations, iso=float(pre.isotropic_coef),
        q_eigenvalues=pre.q_eigenvalues.numpy(), apply_v=v.numpy(), apply_out=pre.apply(v).numpy(),
        lam=1e-2,
    )


def fit_case(n: int, m_pred: int, m_var: int, name: str):
    """Config-1 style fit on the synthetic field: float64 reference, f32 embeddings."""
    x, y, xq = data.synthetic_field(n, seed=0, m=m_pred)
    model = LAKERRegressor(embedding_dim=10, lambda_reg=1e-2, gamma=0.1, pcg_tol=1e-6,
                           pcg_max_iter=1000, dtype=torch.float64, embedding_dtype=torch.float32,
                           verbose=False)
    model.fit(x.double(), y.double(), seed=0)
    pred = model.predict(xq.double())
    var = model.predict_variance(xq[:m_var].double())
    E = model.embeddings
    # high-accuracy truth: direct solve
    a = torch.exp(E @ E.T)
    a.diagonal().add_(1e-2)
    alpha_true = torch.linalg.solve(a, y.double())
    with torch.no_grad():
        eq = model.embedding_model(xq.float()).double()
    pe = PositionEmbedding(2, 10, dtype=torch.float32)
    np.savez_compressed(
        HERE / f"{name}.npz", x=x.numpy(), y=y.numpy(), xq=xq.numpy(), E=E.numpy(),
        Eq=eq.numpy(), alpha=model.alpha.numpy(), alpha_true=alpha_true.numpy(),
        pred=pred.numpy(), var=var.numpy(), iterations=model.pcg_iterations_,
        iso=float(model.preconditioner.isotropic_coef),
        q_eigenvalues=model.preconditioner.q_eigenvalues.numpy(), nr=model.preconditioner.nr,
        freq=pe.freq.numpy(), phase=pe.phase.numpy(), w1=pe.mlp[0].weight.detach().numpy(),
        b1=pe.mlp[0].bias.detach().numpy(), w2=pe.mlp[2].weight.detach().numpy(),
        b2=pe.mlp[2].bias.detach().numpy(),
    )


if __name__ == "__main__":
    kernel_cases()
    paper_case()
    solver_case()
    fit_case(2000, 2000, 64, "fit_n2000")
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)
