"""GPU round trip of model persistence: a model fitted here, saved and
loaded, predicts and answers variance queries with the same bits (the CCCP
factors are restored, not rebuilt); a model file written by the reference
package loads onto the GPU and predicts what the float64 oracle computes from
the stored embeddings and alpha."""

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_model_n300.pt"


def test_save_load_same_bits(cuda, tmp_path):
    from laker_b200 import LAKERRegressor
    from laker_b200.data import synthetic_field

    x, y, _ = synthetic_field(900, 3)
    reg = LAKERRegressor(device=cuda, verbose=False).fit(x, y, seed=3)
    xq = torch.rand(64, 2, generator=torch.Generator().manual_seed(5)) * 100.0
    p0, v0 = reg.predict(xq), reg.predict_variance(xq[:24])
    path = tmp_path / "model.pt"
    reg.save(str(path))
    back = LAKERRegressor.load(str(path))
    assert back.preconditioner is not None and back.pcg_iterations_ == reg.pcg_iterations_
    assert back.get_params()["lambda_reg"] == reg.lambda_reg
    assert torch.equal(back.predict(xq), p0)
    assert torch.equal(back.predict_variance(xq[:24]), v0)


def test_reference_written_model_loads(cuda):
    from laker_b200 import LAKERRegressor

    reg = LAKERRegressor.load(str(GOLDEN), device=cuda)
    assert reg.alpha.device.type == "cuda" and reg.preconditioner is None
    xq = torch.rand(50, 2, generator=torch.Generator().manual_seed(11)) * 100.0
    pred = reg.predict(xq.to(cuda)).cpu().numpy()
    with torch.no_grad():
        Eq = reg.embedding_model(xq.to(cuda).float()).double().cpu().numpy()
    ref = O.rect_matvec(Eq, reg.embeddings.double().cpu().numpy(), reg.alpha.double().cpu().numpy())
    assert np.linalg.norm(pred - ref) / np.linalg.norm(ref) < 1e-10
    var = reg.predict_variance(xq[:8].to(cuda))  # builds the CCCP factors on first use
    assert reg.preconditioner is not None
    assert torch.isfinite(var).all() and (var >= 0).all()
