"""Write tests/golden/ref_model_n300.pt with the LAKER reference package's own
LAKERRegressor.save (laker/persistence.py:74-137): a float64 fit on CPU at
n = 300 (synthetic field, seed 0).  The persistence tests load it to check
that a file written by the reference restores here.

    python tests/golden/make_golden_model.py /path/to/reference
"""

from __future__ import annotations

import sys
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if len(sys.argv) < 2:
    sys.exit(f"usage: python {Path(__file__).name} <path of the reference checkout>")
REF = Path(sys.argv[1])
sys.path.insert(0, str(REF))
sys.path.insert(0, str(REPO))

from laker.models import LAKERRegressor  # noqa: E402

import laker_b200.data as data  # noqa: E402


def main() -> None:
    x, y, _ = data.synthetic_field(300, 0)
    reg = LAKERRegressor(embedding_dim=10, lambda_reg=1e-2, pcg_tol=1e-10, pcg_max_iter=2000,
                         device="cpu", dtype=torch.float64, embedding_dtype=torch.float32,
                         verbose=False)
    reg.fit(x, y.double(), seed=0)
    reg.save(str(HERE / "ref_model_n300.pt"))
    print("wrote", HERE / "ref_model_n300.pt", "alpha norm", float(reg.alpha.norm()))


if __name__ == "__main__":
    main()
