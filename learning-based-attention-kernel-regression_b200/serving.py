"""Serving loop: fit and predictive-variance requests with continuous batching.

A `Server` keeps fitted models (embeddings, CCCP factors, alpha) resident on
the GPU and serves a stream of requests:

* fit(n, lambda, seed): synthetic locations and field (data.synthetic_field),
  PositionEmbedding, operator and CCCP build (laker/models.py:392-455) on a
  build stream, then the PCG solve as an instance of the shared SolveEngine;
* variance(model, m, seed): sigma^2 at m query points of a resident model
  (laker/core.py:666-777): query embeddings, k(X, x*), the m-RHS mixed
  precision PCG on the tensor-core operator and the finish, on a variance
  stream driven by a worker thread.

Continuous batching: the main thread launches an engine replay, prepares the
next fit on the build stream while the replay runs, then admits prepared fits
and collects finished ones between replays; variance solves run concurrently
on their own stream.  Admission is by an HBM budget: a fit is prepared only
when its footprint fits next to the resident models and the engine, evicting
the least recently used models that no queued request needs.  Every result is
the same alone and in any mix (the engine's arithmetic is placement- and
batch-invariant; builds and variance solves are deterministic).

`run_plain` serves the same trace one request at a time through the
single-instance APIs, the baseline the server is compared with.
"""

from __future__ import annotations

import collections
import math
import queue
import statistics
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import torch

from . import _lib
from .core import LAKERCore
from .data import synthetic_field
from .embeddings import PositionEmbedding
from .engine import EngineCapacityError, SolveEngine, engine_bytes_per_instance, instance_blocks
from .kernels import AttentionKernelOperator
from .preconditioner import CCCPPreconditioner
from .solvers import PreconditionedConjugateGradient


@dataclass
class Request:
    rid: int
    kind: str          # "fit" or "variance"
    arrival: float     # seconds after the start of the trace
    seed: int
    n: int = 0         # fit: training points
    lam: float = 1e-2  # fit: lambda_reg
    m: int = 0         # variance: query points
    target: int = -1   # variance: rid of the fit whose model it queries
    refit: bool = False  # internal: rebuild an evicted model for a variance query


@dataclass
class Record:
    rid: int
    kind: str
    arrival: float
    start: float = math.nan
    finish: float = math.nan
    iterations: int = 0
    relres: float = math.nan
    status: int = 0

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


def make_trace(count: int, rate: float, seed: int = 0, n_range=(1000, 50000), m_range=(16, 256),
               fit_fraction: float = 0.7, lam: float = 1e-2) -> List[Request]:
    """Poisson arrivals at `rate` per second: fits (n log-uniform in n_range)
    and variance queries (m uniform in m_range) against a uniformly chosen
    earlier fit; request i uses seed i.  The first request is a fit."""
    g = torch.Generator().manual_seed(int(seed))
    t = 0.0
    out: List[Request] = []
    fits: List[int] = []
    lo, hi = math.log(n_range[0]), math.log(n_range[1])
    for i in range(count):
        u = torch.rand(4, generator=g, dtype=torch.float64).tolist()
        t += -math.log(max(u[0], 1e-300)) / rate
        if not fits or u[1] < fit_fraction:
            n = int(math.floor(math.exp(lo + u[2] * (hi - lo))))
            out.append(Request(i, "fit", t, seed=i, n=n, lam=lam))
            fits.append(i)
        else:
            m = int(m_range[0] + math.floor(u[2] * (m_range[1] - m_range[0] + 1)))
            target = fits[min(len(fits) - 1, int(u[3] * len(fits)))]
            out.append(Request(i, "variance", t, seed=i, m=m, target=target))
    return out


@dataclass
class Model:
    rid: int
    op: AttentionKernelOperator
    pre: CCCPPreconditioner
    emb: PositionEmbedding
    y: torch.Tensor
    nbytes: int
    alpha: Optional[torch.Tensor] = None
    last_use: float = 0.0


def query_points(m: int, seed: int) -> torch.Tensor:
    g = torch.Generator().manual_seed(int(seed) + 7_000_003)
    return torch.rand(m, 2, generator=g) * 100.0


def model_bytes(n: int, d: int, nr: int) -> int:
    """Device bytes of a resident model (embeddings, packed copies, CCCP
    factors, rhs and alpha)."""
    dp = (d + 1) // 2 * 2
    ldq = (nr + 3) // 4 * 4
    n256, n128 = -(-n // 256) * 256, -(-n // 128) * 128
    return (n * d * 4 + n256 * dp * 4 + n128 * dp * 8 + n * nr * 8 + n * ldq * 4 + nr * nr * 12
            + nr * nr * 8 + n * 24)


class Server:
    """Fit and variance requests on one GPU with continuous batching.

    Args:
        hbm_budget: bytes of device memory the server may hold (engine included).
        max_slots / max_points / max_pairs: engine capacity (resident solves).
        chunk: PCG iterations per engine replay.
        tol, max_iter: PCG parameters of fits and variance solves.
        num_probes: CCCP N_r (None: the reference default max(200, 2 sqrt n)).
        keep_outputs: keep alpha / sigma^2 of every request on the host.
    """

    def __init__(self, device: Optional[torch.device] = None, hbm_budget: float = 150e9,
                 max_slots: int = 64, max_points: int = 2_000_000, max_pairs: int = 200_000,
                 chunk: int = 8, tol: float = 1e-6, max_iter: int = 1000, embedding_dim: int = 10,
                 lam: float = 1e-2, num_probes: Optional[int] = None, max_nr: int = 448,
                 keep_outputs: bool = False) -> None:
        self.device = torch.device(device) if device is not None else torch.device("cuda", 0)
        self.d = embedding_dim
        self.tol, self.max_iter = tol, max_iter
        self.num_probes = num_probes
        self.keep_outputs = keep_outputs
        self.engine = SolveEngine(max_slots, max_points, max_pairs, d=embedding_dim, max_nr=max_nr,
                                  clamp=True, chunk=chunk, tol=tol, max_iter=max_iter,
                                  device=self.device)
        self.budget = float(hbm_budget) - self.engine.workspace_bytes
        if self.budget <= 0:
            raise ValueError("hbm_budget smaller than the engine workspace")
        self.build_stream = torch.cuda.Stream(device=self.device)
        self.var_stream = torch.cuda.Stream(device=self.device)
        self.emb = PositionEmbedding(2, embedding_dim, device=self.device, dtype=torch.float32)
        self.core = LAKERCore(embedding_dim=embedding_dim, pcg_tol=tol, pcg_max_iter=max_iter,
                              device=self.device, dtype=torch.float32, verbose=False)
        self.outputs: Dict[int, torch.Tensor] = {}
        # wall seconds of the last run by activity: fit preparation and
        # engine waits (main thread), variance solves (worker), idle waits
        self.stats: Dict[str, float] = {}

    # ------------------------------------------------------------------
    def _nr(self, n: int) -> int:
        nr = self.num_probes if self.num_probes is not None else max(200, int(2 * n**0.5))
        return min(nr, n)

    def prepare_fit(self, req: Request) -> Model:
        """Data, embeddings, operator and CCCP factors of a fit request."""
        x, y, _ = synthetic_field(req.n, req.seed)
        with torch.no_grad():
            E = self.emb(x.to(self.device))
        op = AttentionKernelOperator(E, lambda_reg=req.lam)
        pre = CCCPPreconditioner(num_probes=self._nr(req.n), gamma=0.1, verbose=False,
                                 device=self.device, dtype=torch.float32).build(op.matvec, req.n,
                                                                               seed=req.seed)
        return Model(req.rid, op, pre, self.emb, y.to(self.device, torch.float64),
                     model_bytes(req.n, self.d, pre.nr))

    def variance(self, model: Model, req: Request) -> torch.Tensor:
        """sigma^2 at the request's query points (float64)."""
        xq = query_points(req.m, req.seed).to(self.device)
        return self.core.predict_variance(xq, model.emb, model.op.embeddings, model.op, model.pre,
                                          model.alpha, model.op.lambda_reg).to(torch.float64)

    # ------------------------------------------------------------------
    def run(self, trace: List[Request], realtime: bool = True) -> Dict[int, Record]:
        """Serve `trace` (arrival times relative to the start); returns a
        record per request."""
        eng = self.engine
        records = {r.rid: Record(r.rid, r.kind, r.arrival) for r in trace}
        pending = collections.deque(sorted(trace, key=lambda r: r.arrival))
        fit_queue: collections.deque = collections.deque()
        ready: collections.deque = collections.deque()  # prepared, waiting for engine room
        waiting: Dict[int, List[Request]] = collections.defaultdict(list)
        models: Dict[int, Model] = {}
        fit_requests = {r.rid: r for r in trace if r.kind == "fit"}
        fitted = set()
        inflight: Dict[int, tuple] = {}
        var_q: "queue.Queue[Optional[Request]]" = queue.Queue()
        var_outstanding = collections.Counter()  # model rid -> queued variance requests
        lock = threading.Lock()
        used = [0.0]
        t0 = time.perf_counter()
        clock = (lambda: time.perf_counter() - t0) if realtime else None
        fake_now = [0.0]

        def now() -> float:
            return clock() if realtime else fake_now[0]

        errors: List[BaseException] = []
        # set by the worker after every variance request it ends: the main
        # loop waits on it instead of spinning (a spinning loop holds the GIL
        # and starves the worker)
        wake = threading.Event()
        stats = self.stats = {"prepare_s": 0.0, "engine_wait_s": 0.0, "variance_s": 0.0,
                              "idle_s": 0.0, "replays": 0}

        def worker():
            try:
                with torch.cuda.stream(self.var_stream):
                    while True:
                        req = var_q.get()
                        if req is None:
                            return
                        with lock:
                            model = models.get(req.target)
                        rec = records[req.rid]
                        rec.start = now()
                        if model is None or model.alpha is None:  # its fit failed
                            rec.status = _lib.LAKER_ERR_CAPACITY
                            rec.finish = now()
                            wake.set()
                            continue
                        tv = time.perf_counter()
                        var = self.variance(model, req)
                        self.var_stream.synchronize()
                        stats["variance_s"] += time.perf_counter() - tv
                        rec.finish = now()
                        pcg = self.core.last_pcg
                        rec.iterations = pcg.iterations if pcg is not None else 0
                        if self.keep_outputs:
                            self.outputs[req.rid] = var.cpu()
                        with lock:
                            var_outstanding[req.target] -= 1
                            model.last_use = now()
                        wake.set()
            except BaseException as ex:  # surfaced by the main loop
                errors.append(ex)
                wake.set()

        th = threading.Thread(target=worker, daemon=True)
        th.start()

        def release_variance(model_rid: int):
            for v in waiting.pop(model_rid, []):
                var_q.put(v)

        def evict(need: float) -> bool:
            with lock:
                cands = sorted((m for m in models.values() if var_outstanding[m.rid] <= 0
                                and not waiting.get(m.rid)), key=lambda m: m.last_use)
                for m in cands:
                    if used[0] + need <= self.budget:
                        break
                    used[0] -= m.nbytes
                    del models[m.rid]
                return used[0] + need <= self.budget

        done = 0
        total = len(trace)
        try:
            while done < total:
                if errors:
                    raise errors[0]
                t = now()
                progress = False
                while pending and pending[0].arrival <= t:
                    progress = True
                    r = pending.popleft()
                    if r.kind == "fit":
                        fit_queue.append(r)
                    else:
                        with lock:
                            var_outstanding[r.target] += 1
                            resident = r.target in models and models[r.target].alpha is not None
                        if resident:
                            var_q.put(r)
                        else:
                            if r.target in fitted and not waiting.get(r.target):
                                # evicted: rebuild it ahead of new fits
                                f = fit_requests[r.target]
                                fit_queue.appendleft(Request(f.rid, "fit", f.arrival, f.seed, f.n,
                                                             f.lam, refit=True))
                            waiting[r.target].append(r)
                launched = False
                if eng.running > 0:
                    eng.launch()
                    launched = True
                # prepare one fit while the replay runs
                if fit_queue and len(ready) < 4:
                    r = fit_queue[0]
                    nr = self._nr(r.n)
                    need = model_bytes(r.n, self.d, nr)
                    nb, npairs = instance_blocks(r.n)
                    if nb * 512 > eng.cfg.max_points or npairs > eng.cfg.max_pairs or need > self.budget:
                        fit_queue.popleft()  # can never be served by this server
                        records[r.rid].status = _lib.LAKER_ERR_CAPACITY
                        records[r.rid].finish = now()
                        release_variance(r.rid)
                        progress = True
                    elif evict(need):
                        progress = True
                        fit_queue.popleft()
                        with lock:
                            used[0] += need
                        if not r.refit:
                            records[r.rid].start = now()
                        tp = time.perf_counter()
                        with torch.cuda.stream(self.build_stream):
                            model = self.prepare_fit(r)
                        stats["prepare_s"] += time.perf_counter() - tp
                        ready.append((r, model))
                if launched:
                    tw = time.perf_counter()
                    eng.sync()
                    stats["engine_wait_s"] += time.perf_counter() - tw
                    stats["replays"] += 1
                for slot in eng.finished():
                    progress = True
                    x, res = eng.collect(slot)
                    r, model = inflight.pop(slot)
                    model.alpha = x
                    fitted.add(r.rid)
                    if not r.refit:
                        rec = records[r.rid]
                        rec.finish = now()
                        rec.iterations = res.iterations
                        rec.status = res.status
                        rec.relres = res.residual_norm / max(res.rhs_norm, 1e-300)
                        if self.keep_outputs:
                            self.outputs[r.rid] = x.cpu()
                    with lock:
                        model.last_use = now()
                        models[r.rid] = model
                    release_variance(r.rid)
                while ready:
                    r, model = ready[0]
                    eng.stream.wait_stream(self.build_stream)
                    try:
                        slot = eng.admit(model.op, model.pre, model.y)
                    except EngineCapacityError:
                        break
                    ready.popleft()
                    inflight[slot] = (r, model)
                    progress = True
                # variance completions
                done = sum(1 for rec in records.values() if not math.isnan(rec.finish))
                if progress or launched or done >= total:
                    continue
                # nothing can move until a variance request ends, a request
                # arrives or (without a real clock) time is advanced
                if not realtime and pending and var_q.empty() and not ready and not fit_queue:
                    fake_now[0] = max(fake_now[0], pending[0].arrival)
                    continue
                timeout = 0.05
                if realtime and pending:
                    timeout = min(timeout, max(pending[0].arrival - now(), 0.0))
                ti = time.perf_counter()
                wake.wait(timeout)
                wake.clear()
                stats["idle_s"] += time.perf_counter() - ti
        finally:
            var_q.put(None)
            th.join(timeout=600)
        return records


def run_plain(server: Server, trace: List[Request], realtime: bool = True) -> Dict[int, Record]:
    """The same trace served one request at a time in arrival order through the
    single-instance APIs (CCCP build + fused PCG solve; predict_variance)."""
    records = {r.rid: Record(r.rid, r.kind, r.arrival) for r in trace}
    models: Dict[int, Model] = {}
    t0 = time.perf_counter()
    for r in sorted(trace, key=lambda q: q.arrival):
        t = time.perf_counter() - t0
        if realtime and r.arrival > t:
            time.sleep(r.arrival - t)
        rec = records[r.rid]
        rec.start = time.perf_counter() - t0
        if r.kind == "fit":
            model = server.prepare_fit(r)
            pcg = PreconditionedConjugateGradient(tol=server.tol, max_iter=server.max_iter, verbose=False)
            model.alpha = pcg.solve(model.op.matvec, model.pre.apply, model.y)
            models[r.rid] = model
            rec.iterations = pcg.iterations
            rec.relres = pcg.residual_norm / max(float(torch.linalg.norm(model.y)), 1e-300)
        else:
            var = server.variance(models[r.target], r)
            torch.cuda.synchronize(server.device)
            del var
        torch.cuda.synchronize(server.device)
        rec.finish = time.perf_counter() - t0
    return records


def summarize(records: Dict[int, Record]) -> dict:
    """Throughput and latency percentiles of a served trace."""
    recs = [r for r in records.values() if not math.isnan(r.finish)]
    if not recs:
        return {}
    span = max(r.finish for r in recs) - min(r.arrival for r in recs)
    lat = sorted(r.latency * 1e3 for r in recs)

    def pct(v, p):
        return v[min(len(v) - 1, int(round(p / 100.0 * (len(v) - 1))))]

    out = {"requests": len(recs), "makespan_s": span, "requests_per_s": len(recs) / span,
           "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "mean_ms": statistics.fmean(lat)}
    for kind in ("fit", "variance"):
        lk = sorted(r.latency * 1e3 for r in recs if r.kind == kind)
        if lk:
            out[f"{kind}_count"] = len(lk)
            out[f"{kind}_p50_ms"] = pct(lk, 50)
            out[f"{kind}_p99_ms"] = pct(lk, 99)
    fits = [r for r in recs if r.kind == "fit"]
    out["solves_per_s"] = len(fits) / span
    out["max_fit_relres"] = max((r.relres for r in fits), default=float("nan"))
    return out
