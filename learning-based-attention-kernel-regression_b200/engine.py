"""Continuous-batching solve engine (laker_engine_* of liblaker_b200).

`SolveEngine` keeps many independent PCG solves resident on one GPU and
iterates all of them in one device loop (the iteration is a CUDA graph
replayed by `step`).  Instances are admitted and collected between steps, so
new work joins while other work is in flight; each instance's result is the
same bits whatever else is in the engine.  Per instance the engine stores a
copy of its packed embeddings and right-hand side plus its Krylov state; the
preconditioner factors stay with the caller's CCCPPreconditioner, which the
engine keeps referenced until the instance is collected.

The reference solves each problem with its own PreconditionedConjugateGradient
call (laker/solvers.py:130-295); it has no engine.
"""

from __future__ import annotations

import ctypes
import math
from typing import Dict, List, Optional, Tuple

import torch

from . import _lib
from .kernels import AttentionKernelOperator
from .preconditioner import CCCPPreconditioner

BLOCK = 512  # points per block of the engine's arenas


class EngineCapacityError(RuntimeError):
    """The engine has no free slot, points or block pairs for an instance."""


def instance_blocks(n: int) -> Tuple[int, int]:
    """(blocks, block pairs) an instance of n points occupies in an engine."""
    nb = max(1, math.ceil(n / BLOCK))
    return nb, nb * (nb + 1) // 2


def engine_bytes_per_instance(n: int, d: int, nr: int = 0) -> int:
    """Device bytes an instance needs inside an engine sized for it alone
    (packed embeddings, vectors, the tensor-core operand image of 256 bytes
    per point, pair partials, block partials)."""
    nb, npairs = instance_blocks(n)
    dp = (d + 1) // 2 * 2
    pts = nb * BLOCK
    ldq = max(4, (nr + 3) // 4 * 4)
    return (pts * (12 * dp + 36 + 256) + npairs * BLOCK * 28 + nb * (32 + 4 * ldq + 4) + 4 * ldq + 512)


class SolveEngine:
    """A persistent device loop over resident solves.

    Args:
        max_slots: instances resident at once.
        max_points: sum over resident instances of round_up(n, 512).
        max_pairs: sum over resident instances of nb (nb + 1) / 2 with
            nb = ceil(n / 512) (default: what max_points allows in one instance).
        d: embedding dimension of every instance.
        max_nr: largest preconditioner N_r (0: no preconditioner).
        clamp: clamp Gram entries (needed when an instance's operator does not
            skip the clamp).
        chunk: iterations per step (graph replay).
        tol, max_iter, reliable_delta: PCG parameters (as PreconditionedConjugateGradient).
        device: CUDA device; stream: torch stream the engine enqueues on.
    """

    def __init__(self, max_slots: int, max_points: int, max_pairs: Optional[int] = None,
                 d: int = 10, max_nr: int = 0, clamp: bool = False, chunk: int = 8,
                 tol: float = 1e-6, max_iter: int = 1000, reliable_delta: float = 0.03,
                 device: Optional[torch.device] = None,
                 stream: Optional[torch.cuda.Stream] = None) -> None:
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if self.device.type != "cuda":
            raise RuntimeError("SolveEngine requires a CUDA device")
        lib = _lib.load()
        if max_pairs is None:
            _, max_pairs = instance_blocks(max_points)
        self.cfg = _lib.laker_engine_config(int(max_slots), int(max_points), int(max_pairs), int(d),
                                            int(max_nr), int(bool(clamp)), int(chunk))
        self.params = _lib.laker_pcg_params(float(tol), int(max_iter), float(reliable_delta),
                                            torch.finfo(torch.float32).eps ** 0.5, int(chunk), 0, 0)
        hbytes = lib.laker_engine_host_bytes(ctypes.byref(self.cfg))
        wbytes = lib.laker_engine_workspace_bytes(ctypes.byref(self.cfg))
        if hbytes == 0 or wbytes == 0:
            raise ValueError("invalid engine configuration")
        self.stream = stream if stream is not None else torch.cuda.Stream(device=self.device)
        # pinned, so that launch() returns before the replay completes
        self._host_buf = torch.empty(hbytes, dtype=torch.uint8, pin_memory=True)
        self._host = ctypes.c_void_p(self._host_buf.data_ptr())
        self.workspace = torch.empty(wbytes, dtype=torch.uint8, device=self.device)
        self.workspace_bytes = wbytes
        self._lib = lib
        self._keep: Dict[int, tuple] = {}
        self.running = 0
        _lib.check(lib.laker_engine_init(self._host, hbytes, self.workspace.data_ptr(), wbytes,
                                         ctypes.byref(self.cfg), ctypes.byref(self.params),
                                         ctypes.c_void_p(self.stream.cuda_stream)),
                   "laker_engine_init")
        self._live = True

    # ------------------------------------------------------------------
    def admit(self, op: AttentionKernelOperator, pre: Optional[CCCPPreconditioner],
              b: torch.Tensor) -> int:
        """Admit the solve (lambda I + K) x = b; returns its slot."""
        if op.embedding_dim != self.cfg.d:
            raise ValueError(f"embedding_dim {op.embedding_dim} != engine d {self.cfg.d}")
        if not op.skip_clamp and not self.cfg.clamp:
            raise ValueError("this operator needs clamped entries; create the engine with clamp=True")
        if b.dim() != 1 or b.shape[0] != op.n:
            raise ValueError(f"b must have shape ({op.n},), got {tuple(b.shape)}")
        b64 = b.to(device=self.device, dtype=torch.float64).contiguous()
        pc = pre.c_precond() if pre is not None else None
        slot = ctypes.c_int(-1)
        # the copies run on the engine's stream: order them after b's producer
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        st = self._lib.laker_engine_admit(self._host, op.n, float(op.lambda_reg),
                                          op.packed.packed32.data_ptr(), op.packed.packed64.data_ptr(),
                                          ctypes.byref(pc) if pc is not None else None,
                                          b64.data_ptr(), ctypes.byref(slot))
        if st == _lib.LAKER_ERR_CAPACITY:
            raise EngineCapacityError("engine capacity exhausted (slots, points or block pairs)")
        _lib.check(st, "laker_engine_admit")
        self._keep[slot.value] = (op, pre, b64)
        self.running += 1
        return slot.value

    def step(self) -> int:
        """One graph replay (chunk iterations of every running instance)."""
        running = ctypes.c_int(0)
        _lib.check(self._lib.laker_engine_step(self._host, ctypes.byref(running)), "laker_engine_step")
        self.running = running.value
        return self.running

    def launch(self) -> None:
        """Start one graph replay without waiting (admit/collect wait for sync)."""
        _lib.check(self._lib.laker_engine_launch(self._host), "laker_engine_launch")

    def sync(self) -> int:
        """Wait for the replay started by launch(); running instances after it."""
        running = ctypes.c_int(0)
        _lib.check(self._lib.laker_engine_sync(self._host, ctypes.byref(running)), "laker_engine_sync")
        self.running = running.value
        return self.running

    def finished(self) -> List[int]:
        """Slots that have stopped and are not collected yet."""
        n = self.cfg.max_slots
        arr = (ctypes.c_int * n)()
        cnt = ctypes.c_int(0)
        _lib.check(self._lib.laker_engine_finished(self._host, arr, n, ctypes.byref(cnt)),
                   "laker_engine_finished")
        return [arr[i] for i in range(cnt.value)]

    def collect(self, slot: int) -> Tuple[torch.Tensor, _lib.laker_pcg_result]:
        """Solution (float64, on the device) and PCG result of a stopped slot;
        frees the slot."""
        op = self._keep[slot][0]
        x = torch.empty(op.n, dtype=torch.float64, device=self.device)
        res = _lib.laker_pcg_result()
        with torch.cuda.stream(self.stream):
            _lib.check(self._lib.laker_engine_collect(self._host, slot, x.data_ptr(), ctypes.byref(res)),
                       "laker_engine_collect")
        torch.cuda.current_stream(self.device).wait_stream(self.stream)
        del self._keep[slot]
        return x, res

    def solve_all(self) -> Dict[int, Tuple[torch.Tensor, _lib.laker_pcg_result]]:
        """Step until nothing runs; collect every stopped slot."""
        while self.running > 0:
            self.step()
        return {k: self.collect(k) for k in self.finished()}

    def release(self) -> None:
        if self._live:
            self._lib.laker_engine_release(self._host)
            self._live = False

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
