"""Serving: a request loop that mines queries as they arrive.

* Slots: K library contexts, each with its own CUDA stream and a cap on its
  persistent grid (`max_blocks` = its share of the SMs), so launches from
  different slots run on the device at the same time.
* Admission: each query's device footprint is estimated from its graph
  (CSR + two-hop lists, the root task's bit matrices, the record arena and
  result buffers); a query is admitted when a slot is free and the footprints
  in flight plus its own fit the budget (a fraction of free HBM).
* Continuous batching: a free slot takes every queued query that fits (up to
  `max_batch`) and mines them in one persistent launch (qc_mine_batch); queries
  that arrive while others are on the GPU wait only for the next free slot.
* Device-resident graphs: a query's graph object is handed to the library once
  (one qc_graph per distinct graph object, kept by the server); each slot's
  context keeps the graphs it has mined on the device, so repeated queries on a
  graph skip the upload.  A graph object is treated as immutable once queued.
* Warm-up: optional queries mined once on every slot before the server
  accepts work, so device buffers are sized before the first timed query.
* Latency of each query = completion time - arrival time; the server reports
  p50/p99 and instances/s.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import Context, DeviceGraph


@dataclass
class Request:
    graph: object
    gamma: float
    min_size: int
    arrival: float = 0.0
    rid: int = 0
    est_bytes: int = 0
    done: threading.Event = field(default_factory=threading.Event)
    result: object = None
    error: object = None
    finish: float = 0.0


def estimate_bytes(g, gamma, min_size):
    """Upper estimate of the device memory one query needs."""
    import math
    need = math.ceil(gamma * (min_size - 1))
    deg = np.diff(np.asarray(g.off))
    t = int((deg >= need).sum())            # level-0 survivors bound the root
    w = (t + 31) // 32
    root = 2 * 4 * t * w + 8 * t
    csr = 8 * 2 * (g.n + 1) + 4 * (int(g.off[-1]) + int(g.off2[-1] if g.off2 is not None else 0))
    return csr + 4 * root + (64 << 20)      # root + its first children + fixed buffers


class Server:
    def __init__(self, slots=2, device=0, budget_fraction=0.8, max_batch=64, sms=148, warm=None,
                 warps_per_block=8):
        self.lock = threading.Condition()
        self.dev_graphs = {}  # id(graph) -> (graph, DeviceGraph)
        self.queue = deque()
        self.inflight_bytes = 0
        self.completed = []
        self.stop = False
        free = self._free_bytes(device)
        self.budget = int(free * budget_fraction)
        self.max_batch = max_batch
        share = max(1, sms // slots)
        self.ctxs = [Context(device=device, warps_per_block=warps_per_block, max_blocks=share)
                     for _ in range(slots)]
        if warm:
            for c in self.ctxs:
                c.mine_batch([self._dev(g) for g, _, _ in warm], [gm for _, gm, _ in warm],
                             [ms for _, _, ms in warm])
        self.threads = [threading.Thread(target=self._worker, args=(c,), daemon=True)
                        for c in self.ctxs]
        for t in self.threads:
            t.start()

    def _dev(self, g):
        """The library graph for a query's graph object (made once)."""
        if isinstance(g, DeviceGraph):
            return g
        hit = self.dev_graphs.get(id(g))
        if hit is None or hit[0] is not g:
            hit = (g, DeviceGraph.from_graph(g))
            self.dev_graphs[id(g)] = hit
        return hit[1]

    @staticmethod
    def _free_bytes(device):
        try:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            return free
        except Exception:
            return 64 << 30

    def submit(self, req: Request):
        req.arrival = req.arrival or time.perf_counter()
        req.est_bytes = req.est_bytes or estimate_bytes(req.graph, req.gamma, req.min_size)
        with self.lock:
            self.queue.append(req)
            self.lock.notify_all()
        return req

    def _take(self):
        """Admitted queries for one launch (called with the lock held)."""
        batch, used = [], 0
        while self.queue and len(batch) < self.max_batch:
            r = self.queue[0]
            if self.inflight_bytes + used + r.est_bytes > self.budget and (batch or self.inflight_bytes):
                break
            batch.append(self.queue.popleft())
            used += r.est_bytes
        self.inflight_bytes += used
        return batch, used

    def _worker(self, ctx):
        while True:
            with self.lock:
                while not self.stop and not self.queue:
                    self.lock.wait(0.05)
                if self.stop and not self.queue:
                    return
                batch, used = self._take()
            if not batch:
                time.sleep(0.0005)
                continue
            try:
                with self.lock:
                    dgs = [self._dev(r.graph) for r in batch]
                res = ctx.mine_batch(dgs, [r.gamma for r in batch], [r.min_size for r in batch])
                now = time.perf_counter()
                for r, x in zip(batch, res):
                    r.result, r.finish = x, now
            except Exception as e:  # the whole launch failed: report to each query
                now = time.perf_counter()
                for r in batch:
                    r.error, r.finish = e, now
            with self.lock:
                self.inflight_bytes -= used
                self.completed.extend(batch)
                self.lock.notify_all()
            for r in batch:
                r.done.set()

    def close(self):
        with self.lock:
            self.stop = True
            self.lock.notify_all()
        for t in self.threads:
            t.join()
        for c in self.ctxs:
            c.close()


def run_poisson(server, requests, rate, seed=0):
    """Submit `requests` with Poisson arrivals at `rate` per second; wait for
    all; return latency percentiles (ms) and throughput."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(requests))
    t0 = time.perf_counter()
    nxt = t0
    for r, gap in zip(requests, gaps):
        nxt += gap
        delay = nxt - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        r.arrival = time.perf_counter()
        server.submit(r)
    for r in requests:
        r.done.wait()
    t1 = time.perf_counter()
    lat = np.array([(r.finish - r.arrival) * 1000.0 for r in requests])
    errors = sum(1 for r in requests if r.error is not None)
    return {"rate": rate, "n": len(requests), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "instances_per_s": len(requests) / (t1 - t0), "errors": errors}
