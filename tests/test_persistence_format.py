"""Model file format (no GPU): a file written by the reference's
LAKERRegressor.save (tests/golden/ref_model_n300.pt, made by
tests/golden/make_golden_model.py) is read with weights_only=True, its
embedding network loads into this package's PositionEmbedding and reproduces
the stored embeddings, and this package writes every key the reference
writes."""

from pathlib import Path

import torch

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_model_n300.pt"


def test_reference_model_file_restores_embedding_net():
    from laker_b200 import PositionEmbedding
    from laker_b200.data import synthetic_field

    state = torch.load(GOLDEN, map_location="cpu", weights_only=True)
    assert state["embedding_model_class"] == "PositionEmbedding"
    emb = PositionEmbedding(input_dim=int(state["input_dim"]), embedding_dim=state["embedding_dim"],
                            device=torch.device("cpu"), dtype=torch.float32)
    emb.load_state_dict(state["embedding_model_state"])  # strict: same parameter names
    x, _, _ = synthetic_field(300, 0)
    with torch.no_grad():
        E = emb(x.float()).double()
    ref = state["embeddings"]
    assert E.shape == ref.shape
    assert float((E - ref).abs().max() / ref.abs().max()) < 1e-6


def test_saved_keys_cover_the_reference_format():
    from laker_b200 import persistence

    ref_keys = set(torch.load(GOLDEN, map_location="cpu", weights_only=True).keys())
    ours = set(persistence._HYPER) | {"device", "dtype", "embedding_dtype", "embeddings", "alpha",
                                      "embedding_model_state", "embedding_model_class",
                                      "embedding_model_module", "input_dim"}
    assert ref_keys <= ours, ref_keys - ours
