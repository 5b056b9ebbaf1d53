"""LAKERRegressor: sklearn-style estimator over the B200 solve path.

Drop-in for the solve-path surface of laker.models.LAKERRegressor
(laker/models.py:58-537, 715-850): same constructor and validation
(ValueError messages of models.py:242-288), hyperparameter delegation to the
core, fit / predict / predict_variance / score / score_r2 / get_params /
set_params, and the fitted attributes (embeddings, alpha, kernel_operator,
preconditioner, embedding_model, pcg_iterations_, x_train, y_train).
save / load round-trip a fitted model (persistence.py; the CCCP factors
included).  Training, search and streaming helpers are outside the solve path
and raise NotImplementedError.
"""

from __future__ import annotations

import logging
from typing import Any, Optional, Union

import torch
import torch.nn as nn

from .backend import to_tensor
from .core import LAKERCore

logger = logging.getLogger(__name__)

_OUT_OF_SCOPE = (
    "fit_with_search", "fit_with_bo", "partial_fit", "fit_path", "fit_continuation",
    "fit_learned_embeddings", "fit_residual_corrector", "fit_bilevel", "fit_uncertainty_aware",
    "condition_number",
)


class LAKERRegressor:
    """Learning-based Attention Kernel Regression estimator (B200 solve path)."""

    HYPERPARAMS = (
        "embedding_dim", "lambda_reg", "gamma", "num_probes", "epsilon", "base_rho",
        "cccp_max_iter", "cccp_tol", "pcg_tol", "pcg_max_iter", "chunk_size", "kernel_approx",
        "num_landmarks", "num_features", "k_neighbors", "grid_size", "distributed",
        "twoscale_alpha", "landmark_method", "landmark_pilot_size", "spectral_knots",
        "preconditioner_strategy", "embedding_dtype", "device", "dtype", "verbose",
        "embedding_module",
    )

    def __init__(
        self,
        embedding_dim: int = 10,
        lambda_reg: float = 1e-2,
        gamma: float = 1e-1,
        num_probes: Optional[int] = None,
        epsilon: float = 1e-8,
        base_rho: float = 0.05,
        cccp_max_iter: int = 200,
        cccp_tol: float = 1e-6,
        pcg_tol: float = 1e-6,
        pcg_max_iter: int = 1000,
        chunk_size: Optional[int] = None,
        embedding_module: Optional[nn.Module] = None,
        kernel_approx: Optional[str] = None,
        num_landmarks: Optional[int] = None,
        num_features: Optional[int] = None,
        k_neighbors: Optional[int] = None,
        grid_size: Optional[int] = None,
        distributed: bool = False,
        twoscale_alpha: float = 0.5,
        landmark_method: str = "greedy",
        landmark_pilot_size: int = 1000,
        spectral_knots: int = 5,
        preconditioner: str = "cccp",
        embedding_dtype: Optional[torch.dtype] = None,
        device: Optional[Union[str, torch.device]] = None,
        dtype: Optional[torch.dtype] = None,
        verbose: bool = True,
        residual_corrector: Optional[nn.Module] = None,
    ) -> None:
        if embedding_dim <= 0:
            raise ValueError(f"embedding_dim must be positive, got {embedding_dim}")
        if lambda_reg <= 0:
            raise ValueError(f"lambda_reg must be positive, got {lambda_reg}")
        if gamma < 0:
            raise ValueError(f"gamma must be non-negative, got {gamma}")
        if epsilon <= 0:
            raise ValueError(f"epsilon must be positive, got {epsilon}")
        if not 0 <= base_rho <= 1:
            raise ValueError(f"base_rho must be in [0, 1], got {base_rho}")
        if cccp_max_iter <= 0:
            raise ValueError(f"cccp_max_iter must be positive, got {cccp_max_iter}")
        if cccp_tol <= 0:
            raise ValueError(f"cccp_tol must be positive, got {cccp_tol}")
        if pcg_tol <= 0:
            raise ValueError(f"pcg_tol must be positive, got {pcg_tol}")
        if pcg_max_iter <= 0:
            raise ValueError(f"pcg_max_iter must be positive, got {pcg_max_iter}")
        if kernel_approx not in (None, "nystrom", "rff", "knn", "ski", "twoscale", "spectral"):
            raise ValueError(
                "kernel_approx must be None, 'nystrom', 'rff', 'knn', 'ski', "
                f"'twoscale', or 'spectral', got {kernel_approx}"
            )
        if k_neighbors is not None and k_neighbors <= 0:
            raise ValueError(f"k_neighbors must be positive, got {k_neighbors}")
        if grid_size is not None and grid_size < 2:
            raise ValueError(f"grid_size must be at least 2, got {grid_size}")
        if not 0.0 <= twoscale_alpha <= 1.0:
            raise ValueError(f"twoscale_alpha must be in [0, 1], got {twoscale_alpha}")
        if landmark_method not in ("greedy", "leverage"):
            raise ValueError(
                f"landmark_method must be 'greedy' or 'leverage', got {landmark_method}"
            )
        if landmark_pilot_size <= 0:
            raise ValueError(f"landmark_pilot_size must be positive, got {landmark_pilot_size}")
        if preconditioner not in ("cccp", "adaptive"):
            raise ValueError(f"preconditioner must be 'cccp' or 'adaptive', got {preconditioner}")
        if spectral_knots <= 0:
            raise ValueError(f"spectral_knots must be positive, got {spectral_knots}")

        object.__setattr__(
            self,
            "core",
            LAKERCore(
                embedding_dim=embedding_dim, lambda_reg=lambda_reg, gamma=gamma,
                num_probes=num_probes, epsilon=epsilon, base_rho=base_rho,
                cccp_max_iter=cccp_max_iter, cccp_tol=cccp_tol, pcg_tol=pcg_tol,
                pcg_max_iter=pcg_max_iter, chunk_size=chunk_size,
                embedding_module=embedding_module, kernel_approx=kernel_approx,
                num_landmarks=num_landmarks, num_features=num_features, k_neighbors=k_neighbors,
                grid_size=grid_size, distributed=distributed, twoscale_alpha=twoscale_alpha,
                landmark_method=landmark_method, landmark_pilot_size=landmark_pilot_size,
                spectral_knots=spectral_knots, preconditioner_strategy=preconditioner,
                embedding_dtype=embedding_dtype, device=device, dtype=dtype, verbose=verbose,
            ),
        )
        self.embeddings: Optional[torch.Tensor] = None
        self.alpha: Optional[torch.Tensor] = None
        self.kernel_operator = None
        self.preconditioner = None
        self.embedding_model: Optional[nn.Module] = None
        self.residual_corrector = residual_corrector
        self.x_train: Optional[torch.Tensor] = None
        self.y_train: Optional[torch.Tensor] = None
        self.partial_fit_count: int = 0

    # ------------------------------------------------------------------
    def __getattr__(self, name: str) -> Any:
        if name in LAKERRegressor.HYPERPARAMS:
            return getattr(self.__dict__["core"], name)
        if name in _OUT_OF_SCOPE:
            def _unavailable(*args, **kwargs):
                raise NotImplementedError(f"LAKERRegressor.{name} is outside the B200 solve path")
            return _unavailable
        raise AttributeError(f"'{type(self).__name__}' has no attribute '{name}'")

    def __setattr__(self, name: str, value: Any) -> None:
        if name in self.HYPERPARAMS and "core" in self.__dict__:
            if name == "device" and isinstance(value, str):
                value = torch.device(value)
            if name in ("dtype", "embedding_dtype") and isinstance(value, str):
                value = torch.float32 if "float32" in value else torch.float64
            setattr(self.core, name, value)
        else:
            super().__setattr__(name, value)

    # ------------------------------------------------------------------
    def fit(self, x, y, x0: Optional[torch.Tensor] = None, seed: Optional[int] = None):
        """Embed, build the operator and the CCCP preconditioner, solve (models.py:392-455)."""
        x = to_tensor(x, device=self.device, dtype=self.dtype)
        y = to_tensor(y, device=self.device, dtype=self.dtype).squeeze()
        if x.dim() != 2:
            raise ValueError(f"x must be 2-D, got shape {x.shape}")
        if y.dim() != 1:
            raise ValueError(f"y must be 1-D, got shape {y.shape}")
        self.x_train = x
        self.y_train = y
        self.embeddings, self.embedding_model = self.core.compute_embeddings(x)
        op = self.core.build_kernel_operator(self.embeddings)
        self.kernel_operator = op
        self.preconditioner = self.core.build_preconditioner(
            op.matvec, self.embeddings.shape[0], seed=seed, diagonal=None
        )
        self.alpha, self.pcg_iterations_ = self.core.solve_pcg(op, self.preconditioner, y, x0=x0)
        return self

    def predict(self, x) -> torch.Tensor:
        """Kernel interpolation at query locations (models.py:457-495)."""
        if self.alpha is None or self.embeddings is None:
            raise RuntimeError("Model has not been fitted. Call fit() first.")
        x = to_tensor(x, device=self.device, dtype=self.dtype)
        if x.dim() != 2:
            raise ValueError(f"x must be 2-D, got shape {x.shape}")
        return self.core.predict(x, self.embedding_model, self.embeddings, self.kernel_operator,
                                 self.alpha, self.residual_corrector)

    def predict_variance(self, x) -> torch.Tensor:
        """Posterior variance at query locations (models.py:497-537)."""
        if self.alpha is None or self.embeddings is None:
            raise RuntimeError("Model has not been fitted. Call fit() first.")
        x = to_tensor(x, device=self.device, dtype=self.dtype)
        if x.dim() != 2:
            raise ValueError(f"x must be 2-D, got shape {x.shape}")
        if self.preconditioner is None:  # e.g. loaded from a file without CCCP factors
            self.preconditioner = self.core.build_preconditioner(
                self.kernel_operator.matvec, self.embeddings.shape[0], diagonal=None)
        return self.core.predict_variance(x, self.embedding_model, self.embeddings,
                                          self.kernel_operator, self.preconditioner, self.alpha,
                                          self.lambda_reg)

    def score(self, x, y) -> float:
        """Negative RMSE (models.py:715-736)."""
        y_pred = self.predict(x)
        y_true = to_tensor(y, device=self.device, dtype=self.dtype).squeeze()
        return -torch.sqrt(torch.mean((y_pred - y_true) ** 2)).item()

    def score_r2(self, x, y) -> float:
        """Coefficient of determination (models.py:738-767)."""
        y_pred = self.predict(x)
        y_true = to_tensor(y, device=self.device, dtype=self.dtype).squeeze()
        ss_res = torch.sum((y_true - y_pred) ** 2)
        ss_tot = torch.sum((y_true - y_true.mean()) ** 2)
        if ss_tot.item() == 0.0:
            return 1.0 if ss_res.item() == 0.0 else 0.0
        return (1.0 - ss_res / ss_tot).item()

    def save(self, path: str) -> None:
        """Serialise the fitted model (models.py:851-864; persistence.py)."""
        from .persistence import ModelPersistence

        ModelPersistence.save(self, path)

    @classmethod
    def load(cls, path: str, device=None) -> "LAKERRegressor":
        """Rebuild a model written by save (models.py:866-882; persistence.py);
        `device` overrides the stored one (a file saved on a CPU host)."""
        from .persistence import ModelPersistence

        return ModelPersistence.load(path, device=device)

    def get_params(self, deep: bool = True) -> dict:
        """Constructor parameters (models.py:778-824)."""
        del deep
        return {
            "embedding_dim": self.embedding_dim,
            "lambda_reg": self.lambda_reg,
            "gamma": self.gamma,
            "num_probes": self.num_probes,
            "epsilon": self.epsilon,
            "base_rho": self.base_rho,
            "cccp_max_iter": self.cccp_max_iter,
            "cccp_tol": self.cccp_tol,
            "pcg_tol": self.pcg_tol,
            "pcg_max_iter": self.pcg_max_iter,
            "chunk_size": self.chunk_size,
            "embedding_module": self.embedding_module,
            "kernel_approx": self.kernel_approx,
            "num_landmarks": self.num_landmarks,
            "num_features": self.num_features,
            "k_neighbors": self.k_neighbors,
            "grid_size": self.grid_size,
            "distributed": self.distributed,
            "twoscale_alpha": self.twoscale_alpha,
            "landmark_method": self.landmark_method,
            "landmark_pilot_size": self.landmark_pilot_size,
            "preconditioner": self.preconditioner_strategy,
            "embedding_dtype": (
                str(self.embedding_dtype).replace("torch.", "") if self.embedding_dtype else None
            ),
            "device": str(self.device),
            "dtype": str(self.dtype).replace("torch.", ""),
            "verbose": self.verbose,
            "residual_corrector": self.residual_corrector,
        }

    def set_params(self, **params) -> "LAKERRegressor":
        """Update hyperparameters by name (models.py:826-849)."""
        for key, value in params.items():
            if key == "preconditioner":
                self.core.preconditioner_strategy = value
                continue
            if key not in self.HYPERPARAMS and key not in self.__dict__:
                raise ValueError(f"Invalid parameter {key!r} for LAKERRegressor")
            setattr(self, key, value)
        return self
