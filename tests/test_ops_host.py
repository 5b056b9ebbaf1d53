"""The C-ABI entry points registered as torch custom ops: every op exists in
the `laker_b200` namespace with its schema, and its fake implementation
propagates shapes, dtypes and devices without a GPU (FakeTensor CUDA
tensors), including the packed layouts' sizes from the library's queries."""

import pytest
import torch
from torch._subclasses.fake_tensor import FakeTensorMode


def test_ops_registered_with_schemas():
    import laker_b200 as L

    for name in L.ops.OPS:
        op = getattr(torch.ops.laker_b200, name)
        schema = str(op.default._schema)
        assert schema.startswith(f"laker_b200::{name}(")
    s = str(torch.ops.laker_b200.attn_matvec.default._schema)
    assert "Tensor rows, SymInt m, Tensor cols, SymInt n, SymInt d, float lam, bool clamp, Tensor x" in s
    assert "Tensor? q32" in str(torch.ops.laker_b200.pcg_solve.default._schema)


@pytest.mark.parametrize("n,d,k", [(1, 1, 1), (1000, 10, 1), (1001, 16, 7)])
def test_fake_shapes(n, d, k):
    import laker_b200 as L
    from laker_b200 import _lib

    lib = _lib.load()
    ops = torch.ops.laker_b200
    with FakeTensorMode():
        E = torch.empty(n, d, device="cuda", dtype=torch.float32)
        p32, p64 = ops.pack(E, 32), ops.pack(E, 64)
        assert p32.shape == (lib.laker_packed32_floats(n, d),) and p32.dtype == torch.float32
        assert p64.shape == (lib.laker_packed64_doubles(n, d),) and p64.dtype == torch.float64
        x = torch.empty((n,) if k == 1 else (n, k), device="cuda", dtype=torch.float64)
        y = ops.attn_matvec(p32, n, p32, n, d, 0.01, False, x)
        assert y.shape == x.shape and y.dtype == torch.float32 and y.device.type == "cuda"
        assert ops.attn_matvec(p64, n, p64, n, d, 0.01, True, x).dtype == torch.float64
        r = ops.attn_residual(p64, 3 if n > 3 else n, p64, n, d, 0.0, False, x, x[:3])
        assert r.shape[0] == min(3, n) and r.dtype == torch.float64
        assert ops.attn_diagonal(p64, n, d, 0.1).shape == (n,)
        assert ops.kernel_eval(p64, n, p64, 5, d, False, False).shape == (n, 5)
        q32 = torch.empty(n, 8, device="cuda")
        w32 = torch.empty(5, 5, device="cuda")
        z = ops.precond_apply(q32, w32, n, 5, 0.5, x, True)
        assert z.shape == x.shape and z.dtype == torch.float64
        b = torch.empty(n, device="cuda", dtype=torch.float64)
        xs, st = ops.pcg_solve(p32, p64, n, d, 0.01, False, q32, w32, 5, 0.5, b, None, 1e-6, 10,
                               0.03, 1e-8, 0, False)
        assert xs.shape == (n,) and xs.dtype == torch.float64
        assert st.shape == (len(L.ops.STATS_FIELDS),) and st.device.type == "cpu"
        v = ops.variance_finalize(p64, 4, d, torch.empty(n, 4, device="cuda", dtype=torch.float64),
                                  torch.empty(n, 4, device="cuda", dtype=torch.float64))
        assert v.shape == (4,)


def test_result_from_stats_roundtrip():
    from laker_b200 import _lib, ops

    vals = [4.0, 17.0, 3.0, 1.5e-7, 2.0, 3e-7, 120.0, 1.25, 0.5, 17.0, 3.0]
    res = ops.result_from_stats(torch.tensor(vals, dtype=torch.float64))
    assert res.status == 4 and res.iterations == 17 and res.accurate_matvecs == 3
    assert res.residual_norm == 1.5e-7 and res.kernel_launches == 120
    assert [name for name, _ in _lib.laker_pcg_result._fields_] == list(ops.STATS_FIELDS)


def test_ops_reject_cpu_tensors():
    from laker_b200 import _lib

    with pytest.raises((RuntimeError, ValueError, _lib.LakerError)):
        torch.ops.laker_b200.pack(torch.zeros(4, 3), 32)
