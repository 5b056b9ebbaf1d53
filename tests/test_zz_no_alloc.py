"""The allocation-free FP32 matvec entry point, called through the C ABI.

laker_attn_matvec_f32_noalloc serves callers that can hand over input and
output device buffers but cannot allocate device memory themselves (their
buffers come from another framework's allocator, or their loop may not call
cudaMalloc).  Its scratch is a fixed array inside the library, shared by all
calls.  This file is collected last so that a run stopping at the first
failure has already run every other test; it passes alone in a fresh process
and after the rest of the suite.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

F32_RTOL = 3e-5  # the FP32 operator tolerance used by the other GPU tests


def rel(a, b):
    a, b = a.double(), b.double()
    return float((a - b).norm() / b.norm())


def _free_bytes_settled(cuda, expect):
    """Device free memory, read again once if it differs (another context on
    the GPU can change it between two reads)."""
    free = torch.cuda.mem_get_info(cuda)[0]
    if free != expect:
        torch.cuda.synchronize()
        free = torch.cuda.mem_get_info(cuda)[0]
    return free


def test_noalloc_matches_workspace_entry_point_twice(cuda):
    """Two calls in a row, of different sizes (so the segment split of the
    scratch differs between them), each against the workspace entry point
    and the float64 oracle."""
    from laker_b200 import _lib
    from oracle import laker_oracle as O

    lib = _lib.load()
    rng = np.random.default_rng(21)
    d = 10
    stream = _lib.stream_handle(cuda)
    for call, (n, lam) in enumerate(((3001, 0.01), (9000, 0.3))):
        E_np = (rng.standard_normal((n, d)) * 0.5).astype(np.float32)
        packed = _lib.pack_f32(torch.tensor(E_np, device=cuda))
        x_np = rng.standard_normal(n).astype(np.float32)
        x = torch.tensor(x_np, device=cuda)
        ref = _lib.attn_matvec_f32(packed, n, packed, n, d, lam, 0, x)
        y = torch.full((n,), float("nan"), device=cuda, dtype=torch.float32)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(cuda)[0]
        st = lib.laker_attn_matvec_f32_noalloc(packed.data_ptr(), n, packed.data_ptr(), n, d,
                                               ctypes.c_float(lam), 0, x.data_ptr(),
                                               y.data_ptr(), stream)
        assert st == _lib.LAKER_OK, _lib.status_string(st)
        assert _lib.noalloc_status(cuda) == _lib.LAKER_OK
        if call == 1:
            # after the first call set the scratch up, calls allocate nothing
            assert _free_bytes_settled(cuda, free_before) == free_before
        assert torch.isfinite(y).all()
        assert rel(y, ref) < F32_RTOL
        oracle = torch.tensor(O.attention_matvec(E_np, lam, x_np.astype(np.float64)))
        assert rel(y.cpu(), oracle) < F32_RTOL


def test_noalloc_rectangular_and_limit(cuda):
    from laker_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(22)
    n, m, d = 2000, 333, 10
    E = torch.tensor(rng.standard_normal((n, d)) * 0.5, device=cuda, dtype=torch.float32)
    Q = torch.tensor(rng.standard_normal((m, d)) * 0.5, device=cuda, dtype=torch.float32)
    pe, pq = _lib.pack_f32(E), _lib.pack_f32(Q)
    a = torch.tensor(rng.standard_normal(n), device=cuda, dtype=torch.float32)
    ref = _lib.attn_matvec_f32(pq, m, pe, n, d, 0.0, 0, a)
    y = torch.empty(m, device=cuda, dtype=torch.float32)
    st = lib.laker_attn_matvec_f32_noalloc(pq.data_ptr(), m, pe.data_ptr(), n, d,
                                           ctypes.c_float(0.0), 0, a.data_ptr(), y.data_ptr(),
                                           _lib.stream_handle(cuda))
    assert st == _lib.LAKER_OK
    torch.cuda.synchronize()
    assert rel(y, ref) < F32_RTOL
    # beyond the fixed scratch: a clear error, nothing launched
    too_many = 2_000_001
    st = lib.laker_attn_matvec_f32_noalloc(pq.data_ptr(), too_many, pe.data_ptr(), n, d,
                                           ctypes.c_float(0.0), 0, a.data_ptr(), y.data_ptr(),
                                           _lib.stream_handle(cuda))
    assert st == _lib.LAKER_ERR_SCRATCH_LIMIT
    assert "fixed scratch" in _lib.status_string(st)
