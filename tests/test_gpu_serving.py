"""GPU tests of the serving loop (continuous batching of fit and variance
requests).

Every result must be the same alone and in the mix: a fit's alpha and a
variance query's sigma^2 from a server run over a whole trace are compared
with the same request served by a fresh server on its own (bit for bit; the
stated tolerance, 1e-12 relative, only allows for a library reduction order
that is not fixed).  Fits are held to the solve bar (true float64 relative
residual <= 1e-6) and agree with the one-at-a-time path to its accuracy.
"""

import math

import numpy as np
import pytest
import torch

from oracle import laker_oracle as O

pytestmark = pytest.mark.gpu

ALONE_MIX_RTOL = 1e-12


def small_server(cuda, **kw):
    from laker_b200.serving import Server

    args = dict(device=cuda, hbm_budget=8e9, max_slots=8, max_points=40_000, max_pairs=2_000,
                chunk=8, tol=1e-6, max_iter=2000, keep_outputs=True)
    args.update(kw)
    return Server(**args)


def rel(a, b):
    a, b = a.double(), b.double()
    return float(torch.linalg.norm(a - b) / max(float(torch.linalg.norm(b)), 1e-300))


def test_serving_alone_equals_mix(cuda):
    from laker_b200.serving import Request, make_trace, run_plain, summarize

    trace = make_trace(12, rate=1e4, seed=3, n_range=(600, 2500), m_range=(16, 40))
    srv = small_server(cuda)
    recs = srv.run(trace)
    assert all(not math.isnan(r.finish) and r.status == 0 for r in recs.values())
    s = summarize(recs)
    assert s["requests"] == len(trace) and s["p99_ms"] >= s["p50_ms"] > 0
    fits = [r for r in trace if r.kind == "fit"]
    variances = [r for r in trace if r.kind == "variance"]
    assert fits and variances
    # the solve bar, with the float64 oracle
    for r in fits[:2]:
        model = srv.prepare_fit(r)
        E = model.op.embeddings.double().cpu().numpy()
        assert O.relres(E, r.lam, srv.outputs[r.rid].numpy(), model.y.cpu().numpy()) <= 1e-6
    # alone: a fresh server per request (a variance query brings its target fit)
    for r in fits[:2] + variances[:2]:
        solo_trace = [r] if r.kind == "fit" else [
            next(f for f in fits if f.rid == r.target), r]
        solo_trace = [Request(q.rid, q.kind, 0.0, q.seed, q.n, q.lam, q.m, q.target) for q in solo_trace]
        solo = small_server(cuda)
        solo.run(solo_trace)
        assert rel(solo.outputs[r.rid], srv.outputs[r.rid]) <= ALONE_MIX_RTOL
    # one-at-a-time path: same answers to the solve's accuracy
    plain = small_server(cuda)
    precs = run_plain(plain, trace, realtime=False)
    assert all(p.relres <= 1e-6 for p in precs.values() if p.kind == "fit")


def test_serving_eviction_and_refit(cuda):
    from laker_b200.serving import Request, model_bytes

    # room for about two resident models: later queries need refits
    ns = [1500, 1800, 1600, 1700]
    trace = [Request(i, "fit", 0.0, i, n, 1e-2) for i, n in enumerate(ns)]
    trace += [Request(10 + i, "variance", 0.5, 10 + i, m=24, target=i) for i in range(len(ns))]
    probe = small_server(cuda)
    budget = probe.engine.workspace_bytes + 2.2 * max(model_bytes(n, 10, 200) for n in ns)
    srv = small_server(cuda, hbm_budget=budget)
    recs = srv.run(trace)
    assert all(not math.isnan(r.finish) and r.status == 0 for r in recs.values())
    big = small_server(cuda)
    big.run(trace)
    for r in trace:
        assert rel(srv.outputs[r.rid], big.outputs[r.rid]) <= ALONE_MIX_RTOL
