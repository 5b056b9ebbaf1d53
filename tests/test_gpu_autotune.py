"""GPU test of the measuring autotuner: it times the kernel variants, keeps
the fastest, and the operator still matches the float64 oracle afterwards
(and with every variant, since the tuner checks that they agree)."""

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu


def test_autotune_picks_variants_and_keeps_results(cuda):
    import laker_b200 as L
    from laker_b200 import _lib

    before = {w: _lib.get_variant(w) for w in range(6)}
    try:
        # n = 4000: above the plain-kernel threshold, so the tensor-core
        # symmetric operator's variants are timed too
        res = L.autotune(n=4000, d=10, ks=(16, 100, 256), reps=2, device=cuda)
        assert set(res) >= {"k1t_logits", "k2_logits_n32", "k2_logits_n128", "k2_logits_wide"}
        assert _lib.get_variant(_lib.VARIANT_K1T_LOGITS) == res["k1t_logits"]["choice"]
        for name, r in res.items():
            assert r["choice"] in r["ms"] and all(t > 0 for t in r["ms"].values())
        assert _lib.get_variant(_lib.VARIANT_K2_LOGITS_WIDE) == res["k2_logits_wide"]["choice"]
        rng = np.random.default_rng(1)
        n = 1500
        E = (rng.standard_normal((n, 10)) * 0.5).astype(np.float32)
        X = rng.standard_normal((n, 40))
        op = L.AttentionKernelOperator(torch.tensor(E, device=cuda), lambda_reg=0.01)
        Y = op.matvec(torch.tensor(X, device=cuda, dtype=torch.float32)).double().cpu().numpy()
        ref = O.attention_matvec(E, 0.01, X)
        assert (np.linalg.norm(Y - ref, axis=0) / np.linalg.norm(ref, axis=0)).max() < 1e-4
        y = op.matvec(torch.tensor(X[:, 0], device=cuda, dtype=torch.float32)).double().cpu().numpy()
        assert np.linalg.norm(y - ref[:, 0]) / np.linalg.norm(ref[:, 0]) < 3e-5
    finally:
        for w, v in before.items():
            _lib.set_variant(w, v)
