"""laker_b200: the LAKER exact-kernel solve path on NVIDIA B200 (sm_100a).

Public API (drop-in for the solve path of the `laker` package):

    AttentionKernelOperator   laker.kernels.AttentionKernelOperator
    PreconditionedConjugateGradient  laker.solvers.PreconditionedConjugateGradient
    CCCPPreconditioner        laker.preconditioner.CCCPPreconditioner
    PositionEmbedding         laker.embeddings.PositionEmbedding
    LAKERCore / LAKERRegressor  laker.core / laker.models

The heavy lifting is in liblaker_b200.so (C ABI: include/laker_b200.h), built
in-tree by `laker_b200.build()`; its entry points are registered as torch
custom ops (`torch.ops.laker_b200.*`, module `laker_b200.ops`), which the
classes above call.  Every operator requires CUDA tensors; there
is no CPU implementation to fall back on.
"""

from __future__ import annotations

from . import _lib, ops
from ._build import LIB_PATH
from ._build import build as _build_lib
from .backend import get_default_device, get_default_dtype, set_default_device, set_default_dtype
from .core import LAKERCore
from .data import batch_instances, synthetic_field
from .embeddings import PositionEmbedding
from .kernels import AttentionKernelOperator, KernelOperator
from .distributed import DistributedAttentionKernelOperator, sharded_pcg_solve
from .models import LAKERRegressor
from .preconditioner import CCCPPreconditioner, adaptive_shrinkage_rho, eigh_stable
from .solvers import PreconditionedConjugateGradient
from .batched import BatchedPCG, build_cccp_batched
from .autotune import autotune
from .engine import EngineCapacityError, SolveEngine, engine_bytes_per_instance

__version__ = "0.1.0"


def build(force: bool = False, verbose: bool = False):
    """Compile liblaker_b200.so for sm_100a (in-tree) and load it."""
    path = _build_lib(force=force, verbose=verbose)
    _lib.load()
    return path


__all__ = [
    "autotune",
    "AttentionKernelOperator",
    "BatchedPCG",
    "build_cccp_batched",
    "CCCPPreconditioner",
    "DistributedAttentionKernelOperator",
    "EngineCapacityError",
    "SolveEngine",
    "engine_bytes_per_instance",
    "KernelOperator",
    "LAKERCore",
    "LAKERRegressor",
    "LIB_PATH",
    "PositionEmbedding",
    "PreconditionedConjugateGradient",
    "adaptive_shrinkage_rho",
    "batch_instances",
    "build",
    "sharded_pcg_solve",
    "eigh_stable",
    "get_default_device",
    "get_default_dtype",
    "set_default_device",
    "set_default_dtype",
    "synthetic_field",
]
