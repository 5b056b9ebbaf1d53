"""ctypes binding of liblaker_b200.so (the C ABI declared in include/laker_b200.h).

This module is the only place that touches the shared library.  It loads it
once, declares every entry point's signature, and offers thin tensor-level
wrappers that pass raw device pointers plus the current CUDA stream.  There
is no fallback: if the library has not been built, or a tensor is not on a
CUDA device, the wrappers raise.
"""

from __future__ import annotations

import ctypes
import re
import threading
from ctypes import POINTER, c_double, c_float, c_int, c_int64, c_size_t, c_void_p
from pathlib import Path
from typing import Optional

import torch

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "liblaker_b200.so"
HEADER_PATH = PKG_DIR.parent / "include" / "laker_b200.h"

# Status codes (enum laker_status).
LAKER_OK = 0
LAKER_ERR_INVALID_ARG = 1
LAKER_ERR_CUDA = 2
LAKER_ERR_BREAKDOWN = 3
LAKER_ERR_NOT_CONVERGED = 4
LAKER_ERR_NONFINITE = 5
LAKER_ERR_TIMEOUT = 6
LAKER_ERR_WORKSPACE = 7
LAKER_ERR_UNSUPPORTED = 8
LAKER_ERR_SCRATCH_LIMIT = 9
LAKER_ERR_CAPACITY = 10


class LakerError(RuntimeError):
    """A non-OK status returned by liblaker_b200."""

    def __init__(self, status: int, where: str, message: str) -> None:
        super().__init__(f"{where}: {message} (status {status})")
        self.status = status


class laker_precond(ctypes.Structure):
    _fields_ = [
        ("q_basis", c_void_p),
        ("w_core", c_void_p),
        ("n", c_int64),
        ("nr", c_int),
        ("ldq", c_int),
        ("inv_sqrt_iso", c_double),
    ]


class laker_operator(ctypes.Structure):
    _fields_ = [
        ("packed32", c_void_p),
        ("packed64", c_void_p),
        ("n", c_int64),
        ("d", c_int),
        ("lambda_reg", c_double),
        ("clamp", c_int),
    ]


class laker_pcg_params(ctypes.Structure):
    _fields_ = [
        ("tol", c_double),
        ("max_iter", c_int),
        ("reliable_delta", c_double),
        ("breakdown_eps", c_double),
        ("check_every", c_int),
        ("has_x0", c_int),
        ("profile", c_int),
        ("column_stop", c_int),
    ]


class laker_pcg_result(ctypes.Structure):
    _fields_ = [
        ("status", c_int),
        ("iterations", c_int),
        ("accurate_matvecs", c_int),
        ("residual_norm", c_double),
        ("rhs_norm", c_double),
        ("recurrence_norm", c_double),
        ("kernel_launches", c_int),
        ("fp32_matvec_ms", c_double),
        ("fp64_matvec_ms", c_double),
        ("fp32_matvec_launches", c_int),
        ("fp64_matvec_launches", c_int),
    ]


class laker_batch(ctypes.Structure):
    _fields_ = [
        ("count", c_int),
        ("d", c_int),
        ("clamp", c_int),
        ("n", POINTER(c_int64)),
        ("lambda_reg", POINTER(c_double)),
        ("packed32", c_void_p),
        ("packed64", c_void_p),
        ("precond", POINTER(laker_precond)),
    ]


class laker_engine_config(ctypes.Structure):
    _fields_ = [
        ("max_slots", c_int),
        ("max_points", c_int64),
        ("max_pairs", c_int64),
        ("d", c_int),
        ("max_nr", c_int),
        ("clamp", c_int),
        ("chunk", c_int),
    ]


_P = c_void_p
_SIGNATURES = {
    "laker_engine_host_bytes": (c_size_t, [POINTER(laker_engine_config)]),
    "laker_engine_workspace_bytes": (c_size_t, [POINTER(laker_engine_config)]),
    "laker_engine_init": (
        c_int,
        [_P, c_size_t, _P, c_size_t, POINTER(laker_engine_config), POINTER(laker_pcg_params), _P],
    ),
    "laker_engine_admit": (
        c_int, [_P, c_int64, c_double, _P, _P, POINTER(laker_precond), _P, POINTER(c_int)],
    ),
    "laker_engine_step": (c_int, [_P, POINTER(c_int)]),
    "laker_engine_launch": (c_int, [_P]),
    "laker_engine_sync": (c_int, [_P, POINTER(c_int)]),
    "laker_engine_finished": (c_int, [_P, POINTER(c_int), c_int, POINTER(c_int)]),
    "laker_engine_collect": (c_int, [_P, c_int, _P, POINTER(laker_pcg_result)]),
    "laker_engine_release": (c_int, [_P]),
    "laker_batch_layout": (c_int64, [c_int, POINTER(c_int64), POINTER(c_int64)]),
    "laker_pcg_batched_workspace_bytes": (c_size_t, [c_int, POINTER(c_int64), c_int, c_int]),
    "laker_pcg_solve_batched": (
        c_int,
        [POINTER(laker_batch), _P, _P, POINTER(laker_pcg_params), _P, c_size_t,
         POINTER(laker_pcg_result), _P],
    ),
    "laker_version": (c_int, []),
    "laker_status_string": (ctypes.c_char_p, [c_int]),
    "laker_last_cuda_error": (c_int, []),
    "laker_packed32_floats": (c_size_t, [c_int64, c_int]),
    "laker_packed64_doubles": (c_size_t, [c_int64, c_int]),
    "laker_pack_f32": (c_int, [_P, c_int, c_int64, c_int, c_int64, _P, _P]),
    "laker_pack_f64": (c_int, [_P, c_int, c_int64, c_int, c_int64, _P, _P]),
    "laker_matvec_workspace_bytes": (c_size_t, [c_int64, c_int64, c_int, c_int, c_int]),
    "laker_attn_matvec_f32": (
        c_int,
        [_P, c_int64, _P, c_int64, c_int, c_float, c_int, _P, c_int, c_int64, _P, c_int64, _P,
         c_size_t, _P],
    ),
    "laker_attn_matvec_f32_noalloc": (
        c_int,
        [_P, c_int64, _P, c_int64, c_int, c_float, c_int, _P, _P, _P],
    ),
    "laker_noalloc_status": (c_int, [POINTER(c_int), _P]),
    "laker_workspace_status": (c_int, [_P, POINTER(c_int), _P]),
    "laker_attn_matvec_f64": (
        c_int,
        [_P, c_int64, _P, c_int64, c_int, c_double, c_int, _P, c_int, c_int64, _P, c_int64, _P,
         c_int64, _P, c_size_t, _P],
    ),
    "laker_attn_diagonal": (c_int, [_P, c_int64, c_int, c_double, _P, _P]),
    "laker_kernel_eval": (c_int, [_P, c_int64, _P, c_int64, c_int, c_int, _P, c_int, c_int64, _P]),
    "laker_precond_workspace_bytes": (c_size_t, [c_int64, c_int, c_int]),
    "laker_precond_apply": (
        c_int,
        [POINTER(laker_precond), _P, c_int, c_int64, _P, c_int, c_int64, _P, c_size_t, _P],
    ),
    "laker_pcg_workspace_bytes": (c_size_t, [c_int64, c_int, c_int, c_int]),
    "laker_pcg_solve": (
        c_int,
        [POINTER(laker_operator), POINTER(laker_precond), _P, c_int, _P,
         POINTER(laker_pcg_params), _P, c_size_t, POINTER(laker_pcg_result), _P],
    ),
    "laker_variance_finalize": (
        c_int,
        [_P, c_int64, c_int, _P, _P, c_int64, c_int64, _P, _P],
    ),
    "laker_fp32_matvec_work": (
        c_int,
        [c_int64, c_int, POINTER(c_double), POINTER(c_double), POINTER(c_double)],
    ),
    "laker_peaks_scratch_bytes": (c_size_t, []),
    "laker_fp32_operator_kernel": (c_int, [c_int64, c_int]),
    "laker_set_variant": (c_int, [c_int, c_int]),
    "laker_get_variant": (c_int, [c_int]),
    "laker_measure_peaks": (
        c_int,
        [_P, POINTER(c_double), POINTER(c_double), POINTER(c_double), _P],
    ),
}

_lib: Optional[ctypes.CDLL] = None
_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Load liblaker_b200.so once and declare its signatures.

    Raises:
        RuntimeError: if the shared library has not been built.
    """
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run __graft_entry__.build() "
                "(or python -m laker_b200.build) first"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def header_symbols() -> list[str]:
    """Function names declared in include/laker_b200.h."""
    text = HEADER_PATH.read_text()
    return sorted(set(re.findall(r"\b(laker_[a-z0-9_]+)\s*\(", text)))


def status_string(status: int) -> str:
    return load().laker_status_string(status).decode()


def check(status: int, where: str) -> None:
    if status == LAKER_OK:
        return
    msg = status_string(status)
    if status == LAKER_ERR_CUDA:
        msg += f" (cudaError {load().laker_last_cuda_error()})"
    raise LakerError(status, where, msg)


def stream_handle(device: torch.device) -> int:
    """Raw cudaStream_t of torch's current stream on `device`."""
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise RuntimeError(
            f"{name} must be a CUDA tensor: the LAKER B200 path runs only on the GPU "
            f"(got device {t.device})"
        )


def ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


# Device status words of the asynchronous products, folded per (device,
# stream) into one int32 on the device without a host synchronisation; the
# synchronising layers (solvers, predictions, the CCCP build) read it through
# raise_device_status.  A failed product (a bounded wait that expired on the
# device) has also written NaN to its output.
_pending_status: dict = {}


def note_status(ws: torch.Tensor) -> None:
    """Fold the status word at the start of a product's workspace into the
    pending status of the current stream (asynchronous)."""
    key = (ws.device.index, torch.cuda.current_stream(ws.device).cuda_stream)
    acc = _pending_status.get(key)
    if acc is None:
        acc = torch.zeros(1, dtype=torch.int32, device=ws.device)
        _pending_status[key] = acc
    torch.maximum(acc, ws[:4].view(torch.int32), out=acc)


def raise_device_status(device: torch.device) -> None:
    """Raise LakerError if a product enqueued on the current stream since the
    last check recorded a device-side failure (synchronises that stream)."""
    device = torch.device(device)
    if device.type != "cuda":
        return
    idx = device.index if device.index is not None else torch.cuda.current_device()
    key = (idx, torch.cuda.current_stream(device).cuda_stream)
    acc = _pending_status.get(key)
    if acc is None:
        return
    v = int(acc.item())
    if v != LAKER_OK:
        acc.zero_()
        raise LakerError(v, "device", status_string(v) + " (a bounded wait on the GPU expired; "
                         "the product's outputs were written as NaN)")


def workspace_status(ws: torch.Tensor) -> int:
    """Status word of the last product that used `ws` (synchronises the stream)."""
    st = c_int(0)
    check(load().laker_workspace_status(ptr(ws), ctypes.byref(st), stream_handle(ws.device)),
          "laker_workspace_status")
    return int(st.value)


def noalloc_status(device: torch.device) -> int:
    """Status word of the last allocation-free matvec on `device`'s current
    stream (synchronises it)."""
    st = c_int(0)
    check(load().laker_noalloc_status(ctypes.byref(st), stream_handle(device)),
          "laker_noalloc_status")
    return int(st.value)


# ---------------------------------------------------------------------------
# Tensor-level wrappers
# ---------------------------------------------------------------------------
def pack_f32(E: torch.Tensor) -> torch.Tensor:
    """Pair-interleaved FP32 layout of an (n, d) embedding matrix."""
    require_cuda(E, "embeddings")
    lib = load()
    E = E.contiguous()
    n, d = E.shape
    out = torch.empty(lib.laker_packed32_floats(n, d), dtype=torch.float32, device=E.device)
    check(
        lib.laker_pack_f32(ptr(E), int(E.dtype == torch.float64), n, d, d, ptr(out),
                           stream_handle(E.device)),
        "laker_pack_f32",
    )
    return out


def pack_f64(E: torch.Tensor) -> torch.Tensor:
    """Row-padded FP64 layout of an (n, d) embedding matrix."""
    require_cuda(E, "embeddings")
    lib = load()
    E = E.contiguous()
    n, d = E.shape
    out = torch.empty(lib.laker_packed64_doubles(n, d), dtype=torch.float64, device=E.device)
    check(
        lib.laker_pack_f64(ptr(E), int(E.dtype == torch.float64), n, d, d, ptr(out),
                           stream_handle(E.device)),
        "laker_pack_f64",
    )
    return out


def attn_matvec_f32(rows32, m, cols32, n, d, lam, clamp, X) -> torch.Tensor:
    lib = load()
    X = X.contiguous()
    k = 1 if X.dim() == 1 else X.shape[1]
    Y = torch.empty((m,) if X.dim() == 1 else (m, k), dtype=torch.float32, device=X.device)
    ws = workspace(lib.laker_matvec_workspace_bytes(m, n, d, k, 32), X.device)
    check(
        lib.laker_attn_matvec_f32(ptr(rows32), m, ptr(cols32), n, d, float(lam), int(clamp),
                                  ptr(X), k, k, ptr(Y), k, ptr(ws), ws.numel(),
                                  stream_handle(X.device)),
        "laker_attn_matvec_f32",
    )
    note_status(ws)
    return Y


def attn_matvec_f64(rows64, m, cols64, n, d, lam, clamp, X, B=None) -> torch.Tensor:
    lib = load()
    X = X.contiguous()
    k = 1 if X.dim() == 1 else X.shape[1]
    if B is not None:
        B = B.contiguous()
    Y = torch.empty((m,) if X.dim() == 1 else (m, k), dtype=torch.float64, device=X.device)
    ws = workspace(lib.laker_matvec_workspace_bytes(m, n, d, k, 64), X.device)
    check(
        lib.laker_attn_matvec_f64(ptr(rows64), m, ptr(cols64), n, d, float(lam), int(clamp),
                                  ptr(X), k, k, ptr(B), k, ptr(Y), k, ptr(ws), ws.numel(),
                                  stream_handle(X.device)),
        "laker_attn_matvec_f64",
    )
    note_status(ws)
    return Y


def attn_diagonal(packed64, n, d, lam, device) -> torch.Tensor:
    lib = load()
    out = torch.empty(n, dtype=torch.float64, device=device)
    check(lib.laker_attn_diagonal(ptr(packed64), n, d, float(lam), ptr(out), stream_handle(device)),
          "laker_attn_diagonal")
    return out


def kernel_eval(rows64, m, cols64, p, d, clamp, out_dtype, device) -> torch.Tensor:
    lib = load()
    out = torch.empty((m, p), dtype=out_dtype, device=device)
    check(
        lib.laker_kernel_eval(ptr(rows64), m, ptr(cols64), p, d, int(clamp), ptr(out),
                              int(out_dtype == torch.float64), p, stream_handle(device)),
        "laker_kernel_eval",
    )
    return out


def padded_q(q: torch.Tensor) -> torch.Tensor:
    """FP32 copy of Q (n x nr) with rows padded to a multiple of 4 columns (zeros)."""
    n, nr = q.shape
    ldq = (nr + 3) // 4 * 4
    out = torch.zeros((n, ldq), dtype=torch.float32, device=q.device)
    out[:, :nr] = q
    return out


def precond_struct(q32, w32, n, nr, cis) -> laker_precond:
    """Descriptor of the fused apply's factors; q32 from padded_q()."""
    return laker_precond(ptr(q32), ptr(w32), n, nr, int(q32.shape[1]), float(cis))


def precond_apply(pc: laker_precond, R: torch.Tensor, out_dtype) -> torch.Tensor:
    lib = load()
    R = R.to(torch.float64).contiguous()
    k = 1 if R.dim() == 1 else R.shape[1]
    if R.dim() == 2 and k == 1:
        return precond_apply(pc, R[:, 0], out_dtype).unsqueeze(1)
    Z = torch.empty(R.shape, dtype=out_dtype, device=R.device)
    ws = workspace(lib.laker_precond_workspace_bytes(pc.n, pc.nr, k), R.device)
    check(
        lib.laker_precond_apply(ctypes.byref(pc), ptr(R), k, k, ptr(Z),
                                int(out_dtype == torch.float64), k, ptr(ws), ws.numel(),
                                stream_handle(R.device)),
        "laker_precond_apply",
    )
    return Z


def pcg_solve(op: laker_operator, pc: Optional[laker_precond], B: torch.Tensor, X: torch.Tensor,
              params: laker_pcg_params) -> laker_pcg_result:
    """Run laker_pcg_solve; returns the result struct (status not raised)."""
    lib = load()
    k = 1 if B.dim() == 1 else B.shape[1]
    nr = pc.nr if pc is not None else 0
    nbytes = lib.laker_pcg_workspace_bytes(op.n, op.d, nr, k)
    if nbytes == 0:
        raise LakerError(LAKER_ERR_UNSUPPORTED, "laker_pcg_workspace_bytes",
                         f"unsupported solve shape (n={op.n}, d={op.d}, nr={nr}, k={k})")
    ws = workspace(nbytes, B.device)
    res = laker_pcg_result()
    status = lib.laker_pcg_solve(
        ctypes.byref(op), ctypes.byref(pc) if pc is not None else None, ptr(B), k, ptr(X),
        ctypes.byref(params), ptr(ws), ws.numel(), ctypes.byref(res), stream_handle(B.device),
    )
    if status not in (LAKER_OK, LAKER_ERR_BREAKDOWN, LAKER_ERR_NOT_CONVERGED, LAKER_ERR_NONFINITE):
        check(status, "laker_pcg_solve")
    return res


def variance_finalize(q64, m, d, Kxq, V) -> torch.Tensor:
    lib = load()
    n = Kxq.shape[0]
    Kxq = Kxq.contiguous()
    V = V.contiguous()
    var = torch.empty(m, dtype=torch.float64, device=Kxq.device)
    check(
        lib.laker_variance_finalize(ptr(q64), m, d, ptr(Kxq), ptr(V), n, m, ptr(var),
                                    stream_handle(Kxq.device)),
        "laker_variance_finalize",
    )
    return var


def fp32_matvec_work(n: int, d: int) -> dict:
    """Entries evaluated, FP32 flops and exp2s of one square FP32 operator application."""
    e, f, x = c_double(), c_double(), c_double()
    check(load().laker_fp32_matvec_work(n, d, ctypes.byref(e), ctypes.byref(f), ctypes.byref(x)),
          "laker_fp32_matvec_work")
    return {"entries": e.value, "flops": f.value, "exps": x.value}


# kernel variant slots (include/laker_b200.h, LAKER_VARIANT_*)
VARIANT_K1T_UNIT = 0
VARIANT_K2_LOGITS_N32 = 1
VARIANT_K2_LOGITS_N128 = 2
VARIANT_K2_LOGITS_WIDE = 3
VARIANT_SYM_MIN_BLOCKS = 4
VARIANT_K1T_LOGITS = 5
VARIANT_WAIT_LIMIT_US = 6
VARIANT_MULTI_FLASH_K = 7


def set_variant(which: int, value: int) -> int:
    """Set a kernel variant choice; returns the previous value."""
    prev = int(load().laker_set_variant(which, value))
    if prev < 0:
        raise ValueError(f"invalid kernel variant {which} = {value}")
    return prev


def get_variant(which: int) -> int:
    v = int(load().laker_get_variant(which))
    if v < 0:
        raise ValueError(f"unknown kernel variant {which}")
    return v


def fp32_operator_kernel(n: int, d: int) -> int:
    """0 plain, 1 symmetric (CUDA-core logits), 2 symmetric (tensor-core logits)."""
    return int(load().laker_fp32_operator_kernel(n, d))


def measure_peaks(device: torch.device) -> dict:
    """FP32 FMA (TFLOP/s), MUFU exp2 (Tops/s) and FP64 FMA (TFLOP/s) rates."""
    lib = load()
    scratch = workspace(lib.laker_peaks_scratch_bytes(), device)
    f, mu, dd = c_double(), c_double(), c_double()
    check(lib.laker_measure_peaks(ptr(scratch), ctypes.byref(f), ctypes.byref(mu),
                                  ctypes.byref(dd), stream_handle(device)),
          "laker_measure_peaks")
    return {"ffma_tflops": f.value, "mufu_tops": mu.value, "dfma_tflops": dd.value}
