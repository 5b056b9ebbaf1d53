"""Default device / dtype registry (mirrors laker/backend.py:41-87, 211-244).

The default device is the current CUDA device: the B200 path has no CPU
implementation, so constructing an operator on a CPU tensor raises instead of
silently falling back.  The LAKER_DEVICE / LAKER_DTYPE environment variables
are honoured as in the reference.
"""

from __future__ import annotations

import os
from typing import Optional, Union

import torch

_DEFAULT_DEVICE: Optional[torch.device] = None
_DEFAULT_DTYPE: torch.dtype = torch.float32
_ENV_DONE = False


def _init_from_env() -> None:
    global _ENV_DONE, _DEFAULT_DEVICE, _DEFAULT_DTYPE
    if _ENV_DONE:
        return
    _ENV_DONE = True
    dev = os.environ.get("LAKER_DEVICE")
    if dev:
        _DEFAULT_DEVICE = torch.device(dev)
    dt = os.environ.get("LAKER_DTYPE")
    if dt == "float32":
        _DEFAULT_DTYPE = torch.float32
    elif dt == "float64":
        _DEFAULT_DTYPE = torch.float64


def get_default_device() -> torch.device:
    _init_from_env()
    if _DEFAULT_DEVICE is not None:
        return _DEFAULT_DEVICE
    if torch.cuda.is_available():
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cuda")


def set_default_device(device: Union[str, torch.device]) -> None:
    global _DEFAULT_DEVICE
    _init_from_env()
    _DEFAULT_DEVICE = torch.device(device)


def get_default_dtype() -> torch.dtype:
    _init_from_env()
    return _DEFAULT_DTYPE


def set_default_dtype(dtype: torch.dtype) -> None:
    global _DEFAULT_DTYPE
    _init_from_env()
    if dtype not in (torch.float32, torch.float64):
        raise ValueError(f"dtype must be float32 or float64, got {dtype}")
    _DEFAULT_DTYPE = dtype


def to_tensor(data, device: Optional[torch.device] = None, dtype: Optional[torch.dtype] = None):
    """Array-like -> tensor on the requested device/dtype (laker/backend.py:211-244)."""
    if device is None:
        device = get_default_device()
    if dtype is None:
        dtype = get_default_dtype()
    if isinstance(data, torch.Tensor):
        return data.to(device=device, dtype=dtype)
    return torch.as_tensor(data, device=device, dtype=dtype)
