"""CPU tests: the C ABI loads and validates, host-side logic mirrors the reference."""

import ctypes

import numpy as np
import pytest
import torch


def test_library_exports_every_header_symbol():
    from laker_b200 import _lib

    lib = _lib.load()
    names = _lib.header_symbols()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    # every declared entry point has a ctypes signature in the binding
    assert set(names) <= set(_lib._SIGNATURES)


def test_status_strings_and_version():
    from laker_b200 import _lib

    lib = _lib.load()
    assert lib.laker_version() >= 100
    assert "breakdown" in _lib.status_string(_lib.LAKER_ERR_BREAKDOWN)
    assert _lib.status_string(12345) == "unknown status"


def test_argument_validation_without_gpu():
    """Invalid arguments are rejected before any CUDA call."""
    from laker_b200 import _lib

    lib = _lib.load()
    assert lib.laker_pack_f32(None, 0, 10, 0, 0, None, None) == _lib.LAKER_ERR_INVALID_ARG
    assert lib.laker_pack_f64(None, 0, 10, 17, 17, None, None) == _lib.LAKER_ERR_INVALID_ARG
    assert lib.laker_attn_matvec_f32(None, -1, None, 5, 10, 0.0, 0, None, 1, 1, None, 1, None, 0,
                                     None) == _lib.LAKER_ERR_INVALID_ARG
    assert lib.laker_attn_matvec_f64(None, 4, None, 4, 10, 0.0, 0, None, 2, 1, None, 0, None, 2,
                                     None, 0, None) == _lib.LAKER_ERR_INVALID_ARG
    res = _lib.laker_pcg_result()
    prm = _lib.laker_pcg_params(1e-6, 10, 0.1, 1e-8, 1, 0, 0)
    assert lib.laker_pcg_solve(None, None, None, 1, None, ctypes.byref(prm), None, 0,
                               ctypes.byref(res), None) == _lib.LAKER_ERR_INVALID_ARG
    # zero-size problems are no-ops
    assert lib.laker_attn_matvec_f32(None, 0, None, 0, 10, 0.0, 0, None, 1, 1, None, 1, None, 0,
                                     None) == _lib.LAKER_OK


def test_operator_kernel_query():
    from laker_b200 import _lib

    lib = _lib.load()
    assert lib.laker_fp32_operator_kernel(100000, 10) in (1, 2)
    assert lib.laker_fp32_operator_kernel(100000, 16) == lib.laker_fp32_operator_kernel(100000, 10)
    assert lib.laker_fp32_operator_kernel(2000, 10) == 0  # small: the plain kernel
    assert lib.laker_fp32_operator_kernel(100000, 0) == -1
    assert lib.laker_fp32_operator_kernel(100000, 17) == -1
    assert lib.laker_fp32_operator_kernel(-1, 10) == -1


def test_variant_switches_without_gpu():
    from laker_b200 import _lib

    lib = _lib.load()
    unit = lib.laker_get_variant(_lib.VARIANT_K1T_UNIT)
    assert unit in (2, 4)
    assert lib.laker_set_variant(_lib.VARIANT_K1T_UNIT, 3) == -1  # invalid: unchanged
    assert lib.laker_get_variant(_lib.VARIANT_K1T_UNIT) == unit
    assert lib.laker_set_variant(_lib.VARIANT_K1T_UNIT, 2) == unit
    assert lib.laker_set_variant(_lib.VARIANT_K1T_UNIT, unit) == 2
    for slot in (_lib.VARIANT_K2_LOGITS_N32, _lib.VARIANT_K2_LOGITS_N128, _lib.VARIANT_K2_LOGITS_WIDE):
        v = lib.laker_get_variant(slot)
        assert v in (0, 1)
        assert lib.laker_set_variant(slot, 2) == -1
        assert lib.laker_set_variant(slot, 1 - v) == v
        assert lib.laker_set_variant(slot, v) == 1 - v
    mb = lib.laker_get_variant(_lib.VARIANT_SYM_MIN_BLOCKS)
    assert 0 <= mb <= 64
    assert lib.laker_set_variant(_lib.VARIANT_SYM_MIN_BLOCKS, 65) == -1
    assert lib.laker_set_variant(_lib.VARIANT_SYM_MIN_BLOCKS, 0) == mb
    if lib.laker_fp32_operator_kernel(100000, 10) != 0:
        assert lib.laker_fp32_operator_kernel(2000, 10) != 0  # forced symmetric
        assert lib.laker_fp32_operator_kernel(0, 10) == 0
    assert lib.laker_set_variant(_lib.VARIANT_SYM_MIN_BLOCKS, mb) == 0
    lg = lib.laker_get_variant(_lib.VARIANT_K1T_LOGITS)
    assert lg in (0, 1)
    assert lib.laker_set_variant(_lib.VARIANT_K1T_LOGITS, 2) == -1
    assert lib.laker_set_variant(_lib.VARIANT_K1T_LOGITS, 1 - lg) == lg
    assert lib.laker_set_variant(_lib.VARIANT_K1T_LOGITS, lg) == 1 - lg
    assert lib.laker_get_variant(9) == -1 and lib.laker_set_variant(9, 0) == -1


def test_workspace_and_layout_queries():
    from laker_b200 import _lib

    lib = _lib.load()
    # packed32: pairs padded to 128-pair tiles, dimension padded to even
    assert lib.laker_packed32_floats(1, 10) == 128 * 10 * 2
    assert lib.laker_packed32_floats(257, 3) == 256 * 4 * 2
    assert lib.laker_packed64_doubles(129, 10) == 256 * 10
    assert lib.laker_packed32_floats(10, 17) == 0
    assert lib.laker_pcg_workspace_bytes(100000, 10, 256, 1) > 100000 * 8
    assert lib.laker_pcg_workspace_bytes(0, 10, 256, 1) == 0
    assert lib.laker_precond_workspace_bytes(1000, 2000, 1) == 0  # nr > 1024
    # batched layout: instances at 256-point aligned offsets
    ns = (ctypes.c_int64 * 3)(1, 256, 257)
    offs = (ctypes.c_int64 * 4)()
    assert lib.laker_batch_layout(3, ns, offs) == 1024
    assert list(offs) == [0, 256, 512, 1024]
    assert lib.laker_pcg_batched_workspace_bytes(3, ns, 6, 256) > 1024 * 8
    assert lib.laker_pcg_batched_workspace_bytes(3, ns, 6, 0) > 1024 * 8
    assert lib.laker_pcg_batched_workspace_bytes(3, ns, 6, 2000) == 0
    assert lib.laker_pcg_batched_workspace_bytes(3, ns, 17, 0) == 0
    assert lib.laker_pcg_batched_workspace_bytes(0, ns, 6, 0) == 0
    res = (_lib.laker_pcg_result * 3)()
    prm = _lib.laker_pcg_params(1e-6, 10, 0.1, 1e-8, 1, 0, 0)
    assert lib.laker_pcg_solve_batched(None, None, None, ctypes.byref(prm), None, 0, res,
                                       None) == _lib.LAKER_ERR_INVALID_ARG


def test_estimator_validation_messages():
    from laker_b200 import LAKERRegressor

    for kwargs, msg in [
        ({"embedding_dim": 0}, "embedding_dim must be positive"),
        ({"lambda_reg": 0.0}, "lambda_reg must be positive"),
        ({"gamma": -1.0}, "gamma must be non-negative"),
        ({"pcg_tol": 0.0}, "pcg_tol must be positive"),
        ({"kernel_approx": "bogus"}, "kernel_approx must be None"),
        ({"preconditioner": "jacobi"}, "preconditioner must be 'cccp' or 'adaptive'"),
        ({"base_rho": 2.0}, "base_rho must be in"),
    ]:
        with pytest.raises(ValueError, match=msg):
            LAKERRegressor(**kwargs)


def test_estimator_params_and_delegation():
    from laker_b200 import LAKERRegressor

    m = LAKERRegressor(lambda_reg=0.05, pcg_tol=1e-7, verbose=False, device="cpu")
    assert m.lambda_reg == 0.05 and m.core.lambda_reg == 0.05
    m.lambda_reg = 0.2
    assert m.core.lambda_reg == 0.2
    p = m.get_params()
    assert p["pcg_tol"] == 1e-7 and p["preconditioner"] == "cccp" and p["dtype"] == "float32"
    m.set_params(pcg_max_iter=77)
    assert m.pcg_max_iter == 77
    with pytest.raises(ValueError):
        m.set_params(no_such_param=1)
    with pytest.raises(RuntimeError, match="not been fitted"):
        m.predict(np.zeros((2, 2)))
    with pytest.raises(NotImplementedError):
        m.partial_fit(None, None)


def test_cpu_tensors_fail_loudly():
    """No CPU fallback: the operator refuses CPU embeddings."""
    from laker_b200 import AttentionKernelOperator

    with pytest.raises(RuntimeError, match="CUDA"):
        AttentionKernelOperator(torch.randn(10, 4), lambda_reg=0.1)
    with pytest.raises(ValueError):
        AttentionKernelOperator(torch.randn(10), lambda_reg=0.1)


def test_embedding_matches_reference_weights(golden):
    """Seeded PositionEmbedding parameters equal the reference's (CPU)."""
    from laker_b200 import PositionEmbedding

    g = golden("fit_n2000")
    pe = PositionEmbedding(2, 10, device=torch.device("cpu"), dtype=torch.float32)
    np.testing.assert_array_equal(pe.freq.numpy(), g["freq"])
    np.testing.assert_array_equal(pe.phase.numpy(), g["phase"])
    np.testing.assert_array_equal(pe.mlp[0].weight.detach().numpy(), g["w1"])
    np.testing.assert_array_equal(pe.mlp[2].bias.detach().numpy(), g["b2"])
    with torch.no_grad():
        E = pe(torch.tensor(g["x"]))
    np.testing.assert_array_equal(E.numpy(), g["E"].astype(np.float32))


def test_synthetic_field_deterministic():
    from laker_b200 import batch_instances, synthetic_field

    x1, y1, q1 = synthetic_field(500, seed=4, m=7)
    x2, y2, q2 = synthetic_field(500, seed=4, m=7)
    assert torch.equal(x1, x2) and torch.equal(y1, y2) and torch.equal(q1, q2)
    assert abs(float(y1.mean())) < 1e-5 and abs(float(y1.std()) - 1.0) < 1e-5
    assert x1.min() >= 0 and x1.max() <= 100
    ns, lams = batch_instances(64)
    assert min(ns) >= 500 and max(ns) <= 20000
    assert min(lams) >= 1e-3 and max(lams) <= 1e-1
    assert batch_instances(64) == (ns, lams)


def test_shrinkage_matches_oracle():
    from laker_b200 import adaptive_shrinkage_rho
    from oracle import laker_oracle as O

    for nr, n, g in [(200, 2000, 0.1), (256, 100000, 0.1), (50, 40, 0.1), (30, 3000, 0.01)]:
        assert adaptive_shrinkage_rho(nr, n, g) == O.adaptive_shrinkage_rho(nr, n, g)
