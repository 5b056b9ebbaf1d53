"""Shared pytest configuration.

`gpu` marks tests that need a CUDA device (a B200); everything else runs on
the CPU.  The repository root is put on sys.path so that `laker_b200` (the
package shim) and `oracle` (the float64 checker) import without installation.
"""

import sys
from pathlib import Path

import numpy as np
import pytest
import torch

REPO = Path(__file__).resolve().parent.parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / f"{name}.npz"))
    return load


@pytest.fixture(scope="session")
def cuda():
    import laker_b200  # noqa: F401  (loads the library, fails loudly if missing)
    from laker_b200 import _lib
    _lib.load()
    return torch.device("cuda", 0)


@pytest.fixture(params=["tf32", "f16"])
def k1t_logits(request):
    """The tensor-core symmetric kernel with split-TF32 and split-FP16 logits
    (LAKER_VARIANT_K1T_LOGITS; an engine keeps the format of its creation)."""
    from laker_b200 import _lib

    prev = _lib.set_variant(_lib.VARIANT_K1T_LOGITS, 1 if request.param == "f16" else 0)
    try:
        yield request.param
    finally:
        _lib.set_variant(_lib.VARIANT_K1T_LOGITS, prev)
