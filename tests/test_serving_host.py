"""Host logic of the workload generators and the serving loop's bookkeeping,
on the CPU: the Poisson trace (70 % fits / 30 % variance queries against an
earlier fit, n log-uniform, m uniform, seed per request), the 1024-instance
batch draw (n and lambda log-uniform from a meta-seed generator), the
latency summary and the HBM footprints the admission control uses."""

import math

import pytest


def test_trace_shape_and_determinism():
    from laker_b200.serving import make_trace

    t1 = make_trace(2000, rate=100.0, seed=0, n_range=(1000, 50000), m_range=(16, 256))
    t2 = make_trace(2000, rate=100.0, seed=0, n_range=(1000, 50000), m_range=(16, 256))
    assert [(r.kind, r.arrival, r.n, r.m, r.target, r.seed) for r in t1] == \
           [(r.kind, r.arrival, r.n, r.m, r.target, r.seed) for r in t2]
    assert t1[0].kind == "fit"
    arrivals = [r.arrival for r in t1]
    assert all(b > a for a, b in zip(arrivals, arrivals[1:]))
    # Poisson arrivals at 100 req/s: mean gap 10 ms
    mean_gap = arrivals[-1] / (len(arrivals) - 1)
    assert 0.009 < mean_gap < 0.011
    fits = [r for r in t1 if r.kind == "fit"]
    var = [r for r in t1 if r.kind == "variance"]
    assert abs(len(fits) / len(t1) - 0.7) < 0.04
    assert all(1000 <= r.n < 50000 for r in fits)
    assert all(16 <= r.m <= 256 for r in var)
    fit_ids = set()
    for r in t1:  # a variance query targets a fit that arrived before it
        if r.kind == "fit":
            fit_ids.add(r.rid)
        else:
            assert r.target in fit_ids
    assert all(r.seed == r.rid for r in t1)
    # log-uniform n: about half of the fits below the geometric mean
    gm = math.sqrt(1000 * 50000)
    assert abs(sum(r.n < gm for r in fits) / len(fits) - 0.5) < 0.06
    assert make_trace(50, 100.0, seed=1)[5].arrival != t1[5].arrival


def test_batch_instances_draw():
    from laker_b200 import batch_instances

    ns, lams = batch_instances(1024)
    assert len(ns) == len(lams) == 1024
    assert all(500 <= n <= 20000 for n in ns)
    assert all(1e-3 <= lam <= 1e-1 for lam in lams)
    assert (ns, lams) == batch_instances(1024)
    assert batch_instances(1024, meta_seed=7) != (ns, lams)
    gm = math.sqrt(500 * 20000)
    assert abs(sum(n < gm for n in ns) / 1024 - 0.5) < 0.06
    assert abs(sum(lam < 1e-2 for lam in lams) / 1024 - 0.5) < 0.06


def test_summarize_records():
    from laker_b200.serving import Record, summarize

    recs = {}
    for i in range(10):
        r = Record(i, "fit" if i % 2 == 0 else "variance", arrival=0.1 * i)
        r.start, r.finish, r.relres = 0.1 * i, 0.1 * i + 0.01 * (i + 1), 1e-7 * i
        recs[i] = r
    recs[10] = Record(10, "fit", arrival=5.0)  # not finished: left out
    s = summarize(recs)
    assert s["requests"] == 10 and s["fit_count"] == 5 and s["variance_count"] == 5
    assert s["makespan_s"] == pytest.approx(0.9 + 0.10)
    assert s["requests_per_s"] == pytest.approx(10 / 1.0)
    assert s["p50_ms"] <= s["p99_ms"] == pytest.approx(100.0)
    assert s["max_fit_relres"] == pytest.approx(8e-7)
    assert summarize({}) == {}


def test_footprints_grow_with_the_problem():
    from laker_b200.engine import engine_bytes_per_instance
    from laker_b200.serving import model_bytes

    assert model_bytes(2000, 10, 200) < model_bytes(4000, 10, 200) < model_bytes(4000, 10, 300)
    # the CCCP basis dominates a resident model: n x N_r in FP64 and FP32
    assert model_bytes(50000, 10, 447) > 50000 * 447 * 12
    assert engine_bytes_per_instance(1000, 10, 200) < engine_bytes_per_instance(5000, 10, 200)
    # the symmetric operator's pair partials grow with the square of the blocks
    e1, e2 = engine_bytes_per_instance(10240, 10), engine_bytes_per_instance(20480, 10)
    assert e2 > 2 * e1
