"""Seeded synthetic path-loss fields (the workload generator).

A radio map of 5 transmitters at uniform positions in [0, 100]^2 with
log-distance path loss -20 log10(d + 1) dB each (the field of
examples/basic.py:160-185 without its constant offset, which standardisation
removes), plus N(0, 2^2) shadowing, standardised to zero mean and unit
variance.  All draws come from one CPU torch.Generator seeded with `seed`, in
this order: n locations, 5 transmitters, n shadowing values, then m query
locations.  Everything is float32.
"""

from __future__ import annotations

import math
from typing import Optional, Tuple

import torch

NUM_SOURCES = 5
SHADOW_STD = 2.0
EXTENT = 100.0


def synthetic_field(
    n: int, seed: int, m: int = 0
) -> Tuple[torch.Tensor, torch.Tensor, Optional[torch.Tensor]]:
    """Return (x (n,2), y (n,), x_query (m,2) or None) on the CPU, float32."""
    g = torch.Generator().manual_seed(int(seed))
    x = torch.rand(n, 2, generator=g) * EXTENT
    tx = torch.rand(NUM_SOURCES, 2, generator=g) * EXTENT
    y = torch.zeros(n)
    for t in tx:
        y += -20.0 * torch.log10(torch.norm(x - t, dim=1) + 1.0)
    y = y + SHADOW_STD * torch.randn(n, generator=g)
    y = (y - y.mean()) / y.std()
    xq = torch.rand(m, 2, generator=g) * EXTENT if m > 0 else None
    return x, y, xq


def batch_instances(count: int, meta_seed: int = 1234, n_min: int = 500, n_max: int = 20000,
                    lam_min: float = 1e-3, lam_max: float = 1e-1):
    """(n_i, lambda_i) for `count` independent regressions: n log-uniform in
    [n_min, n_max], lambda log-uniform in [lam_min, lam_max], drawn from a
    meta-seed generator; instance i uses field seed i."""
    g = torch.Generator().manual_seed(int(meta_seed))
    u = torch.rand(count, 2, generator=g, dtype=torch.float64)
    ns = torch.floor(torch.exp(math.log(n_min) + u[:, 0] * (math.log(n_max) - math.log(n_min))))
    lams = torch.exp(math.log(lam_min) + u[:, 1] * (math.log(lam_max) - math.log(lam_min)))
    return [int(v) for v in ns.tolist()], [float(v) for v in lams.tolist()]
