"""PositionEmbedding: the input producer of the solve path.

Same module as laker/embeddings.py:42-242 (random Fourier features
cos(2*pi*x@F + phi) followed by Linear-Tanh-Linear), with the same
parameter draws in the same order from a generator seeded with `seed`:
freq ~ N(0,1)/sigma (input_dim x num_fourier), phase ~ U(0, 2*pi), then for
each Linear the weight and the bias ~ U(-b, b) with b = sqrt(1/fan_in).

One deliberate difference: the draws always come from a CPU generator and
are then moved to the target device.  The reference draws from a generator on
the target device, so on CUDA it would get different weights than on CPU;
drawing on the CPU keeps a seeded model identical across devices and equal to
the CPU float64 oracle's.  The forward pass is plain torch and stays on the
device (about 600 flops per point, negligible next to the solve).
"""

from __future__ import annotations

import math
from typing import Optional

import torch
import torch.nn as nn

from .backend import get_default_device, get_default_dtype


class PositionEmbedding(nn.Module):
    """Position-driven embedding (laker/embeddings.py:42-242)."""

    def __init__(
        self,
        input_dim: int,
        embedding_dim: int,
        num_fourier: Optional[int] = None,
        sigma: float = 10.0,
        seed: int = 42,
        device: Optional[torch.device] = None,
        dtype: Optional[torch.dtype] = None,
    ) -> None:
        super().__init__()
        self.input_dim = input_dim
        self.embedding_dim = embedding_dim
        self.sigma = sigma
        if num_fourier is None:
            num_fourier = embedding_dim * 2
        self.num_fourier = num_fourier
        if device is None:
            device = get_default_device()
        if dtype is None:
            dtype = get_default_dtype()

        gen = torch.Generator(device="cpu").manual_seed(seed)
        freq = torch.randn(input_dim, num_fourier, generator=gen, dtype=dtype) / sigma
        phase = torch.rand(num_fourier, generator=gen, dtype=dtype) * 2.0 * math.pi
        self.register_buffer("freq", freq)
        self.register_buffer("phase", phase)

        mlp_hidden = max(embedding_dim, num_fourier // 2)
        self.mlp = nn.Sequential(
            nn.Linear(num_fourier, mlp_hidden, dtype=dtype),
            nn.Tanh(),
            nn.Linear(mlp_hidden, embedding_dim, dtype=dtype),
        )
        with torch.no_grad():
            for layer in self.mlp:
                if isinstance(layer, nn.Linear):
                    bound = math.sqrt(1.0 / layer.weight.shape[1])
                    layer.weight.copy_(
                        torch.rand(layer.weight.shape, generator=gen, dtype=dtype) * (2 * bound)
                        - bound
                    )
                    if layer.bias is not None:
                        layer.bias.copy_(
                            torch.rand(layer.bias.shape, generator=gen, dtype=dtype) * (2 * bound)
                            - bound
                        )
        self.to(device=device, dtype=dtype)

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        if x.dim() == 1:
            x = x.unsqueeze(0)
        features = torch.cos(2.0 * math.pi * (x @ self.freq) + self.phase)
        return self.mlp(features)

    def extra_repr(self) -> str:
        return (
            f"input_dim={self.input_dim}, embedding_dim={self.embedding_dim}, "
            f"num_fourier={self.num_fourier}, sigma={self.sigma}"
        )
