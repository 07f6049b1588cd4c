"""Serving loop: admission (CPU) and same-result-alone-and-in-the-mix (GPU)."""
import threading
from collections import deque

import numpy as np
import pytest

from cuqc_b200 import graphs
from cuqc_b200.serve import Request, Server, estimate_bytes, run_poisson


def _bare_server(budget, max_batch=4, inflight=0):
    s = Server.__new__(Server)
    s.lock = threading.Condition()
    s.queue = deque()
    s.budget = budget
    s.inflight_bytes = inflight
    s.max_batch = max_batch
    return s


def _req(est, rid):
    g = graphs.random_small(10, 0.3, rid)
    return Request(graph=g, gamma=0.8, min_size=3, rid=rid, est_bytes=est)


def test_admission_respects_budget_and_order():
    s = _bare_server(budget=100)
    for i, est in enumerate([40, 40, 40, 10]):
        s.queue.append(_req(est, i))
    batch, used = s._take()
    assert [r.rid for r in batch] == [0, 1] and used == 80      # FIFO, stops at the budget
    assert s.inflight_bytes == 80
    batch2, used2 = s._take()
    assert batch2 == []                                          # nothing fits until release
    s.inflight_bytes -= used
    batch3, _ = s._take()
    assert [r.rid for r in batch3] == [2, 3]


def test_admission_batch_cap_and_oversized_request():
    s = _bare_server(budget=100, max_batch=2)
    for i in range(3):
        s.queue.append(_req(10, i))
    batch, _ = s._take()
    assert len(batch) == 2
    # a query larger than the whole budget still runs when nothing else is in flight
    s2 = _bare_server(budget=100)
    s2.queue.append(_req(1000, 9))
    b, _ = s2._take()
    assert [r.rid for r in b] == [9]


def test_estimate_grows_with_graph():
    a = graphs.random_small(40, 0.2, 1)
    b = graphs.random_small(200, 0.2, 1)
    assert estimate_bytes(b, 0.8, 5) > estimate_bytes(a, 0.8, 5) > 0


@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix():
    import cuqc_b200 as Q
    from oracle import oracle

    reqs, specs = [], []
    for i in range(40):
        rng = np.random.default_rng(900 + i)
        g = graphs.random_small(int(rng.integers(20, 90)), float(rng.uniform(0.08, 0.35)), 900 + i,
                                planted=int(rng.integers(0, 4)), size=int(rng.integers(6, 14)),
                                density=0.95)
        gm = [0.75, 0.8, 0.9, 0.95][i % 4]
        ms = int(rng.integers(4, 9))
        specs.append((g, gm, ms))
        reqs.append(Request(graph=g, gamma=gm, min_size=ms, rid=i))
    srv = Server(slots=3)
    try:
        stats = run_poisson(srv, reqs, rate=2000.0, seed=1)
    finally:
        srv.close()
    assert stats["errors"] == 0
    with Q.Context(device=0) as ctx:
        for (g, gm, ms), r in zip(specs, reqs):
            alone = ctx.mine(g, gm, ms).sets
            assert r.result.sets == alone == oracle.solve(g, gm, ms)[0]
