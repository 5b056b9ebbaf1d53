"""Model persistence: save a fitted LAKERRegressor and load it back.

Drop-in for laker.persistence.ModelPersistence (laker/persistence.py:74-137
save, :139-230 load): one dictionary written with torch.save, with the
reference's keys (hyperparameters, `embeddings`, `alpha`, the embedding
network's `embedding_model_state` / `_class` / `_module`, `input_dim`), so a
file written here loads in the reference and one written by the reference
loads here.  Added for the device path: `cccp_state`, the CCCP
preconditioner's factors exactly as the fused apply uses them (Q, the folded
FP32 core W, c, the fixed-point state), so a reloaded model answers variance
queries without rebuilding its preconditioner and gives the same bits as
before saving.  A file without `cccp_state` (the reference's) reloads with the
preconditioner rebuilt on the first variance query.  The file holds tensors and
plain values only and is read with weights_only=True.
"""

from __future__ import annotations

import importlib
import logging
from typing import TYPE_CHECKING, Any, Dict

import torch

if TYPE_CHECKING:  # pragma: no cover
    from .models import LAKERRegressor

logger = logging.getLogger(__name__)

_HYPER = ("embedding_dim", "lambda_reg", "gamma", "num_probes", "epsilon", "base_rho",
          "cccp_max_iter", "cccp_tol", "pcg_tol", "pcg_max_iter", "chunk_size", "kernel_approx",
          "num_landmarks", "num_features", "k_neighbors", "grid_size", "distributed", "verbose")


def _cpu(t):
    return t.detach().to("cpu") if torch.is_tensor(t) else t


class ModelPersistence:
    """Serialisation of fitted LAKERRegressor models (laker/persistence.py:51)."""

    @staticmethod
    def save(regressor: "LAKERRegressor", path: str) -> None:
        """Write the fitted model to `path` (overwrites).

        Raises:
            RuntimeError: if the regressor has not been fitted.
        """
        if regressor.alpha is None:
            raise RuntimeError("Model has not been fitted. Call fit() before saving.")
        state: Dict[str, Any] = {k: getattr(regressor, k) for k in _HYPER}
        state["device"] = str(regressor.device)
        state["dtype"] = str(regressor.dtype)
        state["embedding_dtype"] = str(regressor.embedding_dtype) if regressor.embedding_dtype else None
        state["embeddings"] = _cpu(regressor.embeddings)
        state["alpha"] = _cpu(regressor.alpha)
        model = regressor.embedding_model
        if model is not None:
            state["embedding_model_state"] = {k: _cpu(v) for k, v in model.state_dict().items()}
            state["embedding_model_class"] = model.__class__.__name__
            state["embedding_model_module"] = model.__class__.__module__
            if hasattr(model, "input_dim"):
                state["input_dim"] = model.input_dim
        if regressor.preconditioner is not None and regressor.preconditioner.q_basis is not None:
            state["cccp_state"] = regressor.preconditioner.state_dict()
        if getattr(regressor, "pcg_iterations_", None) is not None:
            state["pcg_iterations"] = int(regressor.pcg_iterations_)
        torch.save(state, path)

    @staticmethod
    def load(path: str, device=None) -> "LAKERRegressor":
        """Rebuild a LAKERRegressor from a file written by save (here or by
        the reference): operator and, when stored, CCCP factors on the device,
        ready for predict and predict_variance.  `device` overrides the stored
        device (a file saved on a CPU host)."""
        from .embeddings import PositionEmbedding
        from .models import LAKERRegressor
        from .preconditioner import CCCPPreconditioner

        state = torch.load(path, map_location="cpu", weights_only=True)
        dtype = torch.float32 if "float32" in state["dtype"] else torch.float64
        edt = state.get("embedding_dtype")
        embedding_dtype = None if not edt else (torch.float32 if "float32" in edt else torch.float64)
        kwargs = {k: state[k] for k in _HYPER if k in state}
        reg = LAKERRegressor(dtype=dtype, embedding_dtype=embedding_dtype,
                             device=device if device is not None else state["device"], **kwargs)
        dev = reg.device
        reg.embeddings = state["embeddings"].to(dev)
        reg.alpha = state["alpha"].to(dev)
        if "embedding_model_state" in state:
            cls = PositionEmbedding
            name = state.get("embedding_model_class", "PositionEmbedding")
            module = state.get("embedding_model_module", "")
            if name != "PositionEmbedding":
                try:
                    cls = getattr(importlib.import_module(module), name)
                except (ImportError, AttributeError):
                    logger.warning("Could not import %s.%s for loading; falling back to "
                                   "PositionEmbedding.", module, name)
            input_dim = int(state.get("input_dim", 2))
            if cls is PositionEmbedding:
                model = PositionEmbedding(input_dim=input_dim, embedding_dim=reg.embedding_dim,
                                          device=dev, dtype=reg.embedding_dtype)
            else:
                model = cls(input_dim, reg.embedding_dim)
            model.load_state_dict({k: v.to(dev) for k, v in state["embedding_model_state"].items()})
            reg.embedding_model = model.to(dev)
        reg.kernel_operator = reg.core.build_kernel_operator(reg.embeddings)
        if "cccp_state" in state:
            reg.preconditioner = CCCPPreconditioner.from_state(state["cccp_state"], device=dev,
                                                               dtype=reg.dtype)
        if "pcg_iterations" in state:
            reg.pcg_iterations_ = state["pcg_iterations"]
        return reg
