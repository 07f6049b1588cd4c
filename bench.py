"""Benchmark: maximal gamma-quasi-clique enumeration on the B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cfg1|cfg2|...]

A step is one full mining pass over one instance: level 0, the persistent
expansion kernel and the device non-maximal removal (everything qc_mine does
once the graph is resident in HBM).  `value` is instances/s over the K timed
steps, device-timed with CUDA events on the library's own stream; L2 is
flushed (a 256 MiB write) before every step and the flush is not timed.
`e2e` is the same metric through the public C ABI from host arrays: graph
construction from host CSR, host->device copy, mining, and the device->host
read of the result, all inside the timed region.

Under torchrun (N > 1) every rank mines its own replica of the instance on its
own GPU (instances are independent: weak scaling, no data-path collective);
the elapsed time is the max over ranks.

--impl reference times the reference's own CPU implementation of the path (its
host routines, compiled from the reference sources into
oracle/_ref/libqc_refcpu.so) on the host cores, one instance per core.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from cuqc_b200 import graphs  # noqa: E402

WORKLOADS = {
    # Erdos-Renyi G(1000, 0.02) + 5 disjoint planted groups of 30 at 0.95
    "cfg1": dict(desc="ER G(n=1000,p=0.02) + 5 planted groups of 30 @0.95, gamma=0.9, min_size=20",
                 gen="erdos_renyi_planted",
                 kw=dict(n=1000, p=0.02, groups=5, group_size=30, density=0.95, seed=1),
                 gamma="0.9", min_size=20),
    # Chung-Lu n=8000, exponent 2.1, mean degree 40 + 200 planted groups
    "cfg2": dict(desc="Chung-Lu n=8000 beta=2.1 mean deg 40 + 200 planted groups 15-60 @0.85-1.0, "
                      "gamma=0.8, min_size=15",
                 gen="chung_lu_planted",
                 kw=dict(n=8000, beta=2.1, mean_degree=40, n_groups=200, size_range=(15, 60),
                         density_range=(0.85, 1.0), seed=2),
                 gamma="0.8", min_size=15),
}
# Batched workload: independent instances of uneven size (graphs.batch_instance)
BATCH_WORKLOADS = {"cfg3": dict(desc="independent instances: n log-uniform 200-5000, Chung-Lu "
                                     "mean deg 10-50 + 1-20 planted groups 10-40 @0.8-1.0, "
                                     "gamma in {0.6,0.7,0.8,0.9,0.95}, min_size 5-30")}
DEFAULT_WORKLOAD = "cfg1"
L2_FLUSH_BYTES = 256 << 20


def load_traffic():
    """DRAM bytes per expand_kernel launch on config 1 from the committed ncu
    summary (profiles/expand_kernel_cfg1.md), or None."""
    p = os.path.join(ROOT, "profiles", "expand_kernel_cfg1.md")
    if os.path.exists(p):
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1])
    return None


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region.

    Reads NVML (the library nvidia-smi reports from) every 2 ms from a thread, so
    a timed region of a few tens of milliseconds still gets samples; falls back
    to `nvidia-smi -lms 200` where NVML is missing.  Read-only: no setting of the
    GPU is touched."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device, period_s=0.002):
        self.device = device
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.rows = []
        self.path = tempfile.mktemp(suffix=".csv")

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(
                uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _poll(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), [n for n in self.NAMES if r & bits[n]]))
            except Exception:
                pass
            self.stop.wait(self.period)

    def __enter__(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            self.sm_max = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            self.nvml = nv
            return self
        except Exception:
            self.nvml = None
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.nvml:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.nvml:
            if not self.rows:
                return {"sm_mhz": None, "sm_max_mhz": self.sm_max, "reasons": ["no samples"],
                        "samples": 0, "source": "nvml"}
            return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.sm_max,
                    "reasons": sorted({n for r in self.rows for n in r[1]}),
                    "samples": len(self.rows), "source": "nvml, every 2 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi -lms 200"}


def arm_config(w):
    """The workload as both arms report it (the same dict, so the two lines
    can be matched): name, generator description, gamma and min_size."""
    spec = WORKLOADS[w]
    return {"workload": w, "desc": spec["desc"], "gamma": spec["gamma"],
            "min_size": spec["min_size"], "seed": spec["kw"]["seed"]}


def make_graph(w):
    spec = WORKLOADS[w]
    return getattr(graphs, spec["gen"])(**spec["kw"]), spec


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU path
# ---------------------------------------------------------------------------

def _refcpu_one(args):
    path, gamma, ms = args
    from oracle import oracle
    d = tempfile.mkdtemp(prefix="refcpu_")
    t = {}
    import io
    import contextlib
    with contextlib.redirect_stdout(io.StringIO()):
        text, _ = oracle.refcpu_run(path, gamma, ms, workdir=d, times=t)
    return t["enum_ms"] + t["rm_ms"], text.count("\n")


def cpu_reference_rate(path, spec, procs, instances):
    """instances/s of the reference CPU path: `instances` runs on `procs`
    processes (spawned); each run's time excludes file parsing."""
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_refcpu_one, [(path, spec["gamma"], spec["min_size"])] * instances)
    wall = time.perf_counter() - t0
    per = [r[0] for r in res]
    # throughput from the per-run enumeration+removal times, `procs` at a time
    busy_s = sum(per) / 1000.0 / procs
    return instances / busy_s, per, wall, res[0][1]


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = args.workload
    g, spec = make_graph(w)
    d = tempfile.mkdtemp()
    path = os.path.join(d, "g.txt")
    graphs.write_serialized(g, path)
    from oracle import oracle
    if not oracle.refcpu_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libqc_refcpu.so absent"}))
        return
    procs = max(1, os.cpu_count() or 1)
    for _ in range(args.warmup):
        cpu_reference_rate(path, spec, procs, procs)
    rates, step_ms = [], []
    for _ in range(args.steps):
        r, per, wall, nmax = cpu_reference_rate(path, spec, procs, procs)
        rates.append(r)
        step_ms.append(statistics.mean(per))
    value = statistics.mean(rates)
    line = {
        "impl": "reference", "metric": "instances/s (maximal gamma-quasi-clique enumeration)",
        "value": value, "unit": "instances/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(step_ms), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": arm_config(w),
        "parallelism": "one instance per host core",
        "cpu_baseline": {"value": value, "unit": "instances/s", "cores": procs,
                         "kind": "reference",
                         "sample": "%d full instances per step, one per core; time = the "
                                   "reference's enumeration + RemoveNonMax (file parse excluded)"
                                   % procs},
        "e2e": {"value": value, "unit": "instances/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "maximal": nmax,
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

BATCH_MANIFEST = os.path.join(ROOT, "tests", "golden", "cfg3_batch.json")


def _digest(sets):
    import hashlib
    text = "".join("%d %s \n" % (len(x), " ".join(map(str, x))) for x in sets)
    return hashlib.sha1(text.encode()).hexdigest()


def run_batch(args, standalone=True):
    """Batched vs plain on the multi-instance workload: every instance of the
    manifest (tests/golden/cfg3_batch.json) in one persistent launch against
    one launch per instance.  Returns the measurement as a dict."""
    import torch

    import cuqc_b200 as Q

    with open(BATCH_MANIFEST) as f:
        man = json.load(f)
    rows = man["instances"][: args.instances]
    inst = [graphs.batch_instance(r["i"]) for r in rows]
    gs = [x[0] for x in inst]
    gms = [float(x[1]) for x in inst]
    mss = [x[2] for x in inst]
    # the batched launch on its own context, its settings picked by the
    # library's tuner (qc_tune_batch) on the first 64 instances, each candidate
    # timed twice after a warm-up (a sample of 32 timed once picked 4 or 8
    # warps a block from run to run); the plain launches on another context
    # with the defaults
    ctx = Q.Context(device=0)
    pctx = Q.Context(device=0)
    dgs = [Q.DeviceGraph.from_graph(g) for g in gs]
    ns = min(64, len(dgs))
    tuned = ctx.tune_batch(dgs[:ns], gms[:ns], mss[:ns], repeats=2) if args.tune else None
    dev = torch.device("cuda", 0)
    streams = {id(ctx): torch.cuda.ExternalStream(ctx.stream, device=dev),
               id(pctx): torch.cuda.ExternalStream(pctx.stream, device=dev)}

    def timed(c, fn):
        stream = streams[id(c)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    for _ in range(args.warmup):
        ref = ctx.mine_batch(dgs, gms, mss)
        pctx.mine(dgs[0], gms[0], mss[0])
    # parity with the oracle's results recorded in the manifest
    bad = [r["i"] for r, x in zip(rows, ref) if _digest(x.sets) != r["digest"]]
    if bad:
        raise SystemExit("batched results differ from the oracle on instances %s" % bad[:10])
    ref_flat = [x.flat.tobytes() for x in ref]
    batched_ms, plain_ms = [], []
    for _ in range(args.steps):
        res, ms = timed(ctx, lambda: ctx.mine_batch(dgs, gms, mss))
        assert [r.flat.tobytes() for r in res] == ref_flat
        batched_ms.append(ms)
    [pctx.mine(d, gm, m) for d, gm, m in zip(dgs, gms, mss)]  # every graph resident
    for _ in range(max(1, args.steps // 2)):
        res, ms = timed(pctx, lambda: [pctx.mine(d, gm, m) for d, gm, m in zip(dgs, gms, mss)])
        assert [r.flat.tobytes() for r in res] == ref_flat
        plain_ms.append(ms)
    st = ref[0].stats
    b = statistics.median(batched_ms)
    p = statistics.median(plain_ms)
    n_inst = len(rows)
    out = {
        "value": n_inst / (b / 1000.0), "unit": "instances/s", "ms_per_step": b,
        "instances": n_inst, "kernel_ms": st["kernel_ms"], "tasks": st["tasks"],
        "plain": {"value": n_inst / (p / 1000.0), "unit": "instances/s", "ms_per_step": p,
                  "form": "one qc_mine launch per instance, one context, default settings, "
                          "graphs resident"},
        "tuned": tuned,
        "batched_over_plain": p / b,
        "maximal_total": sum(r["maximal"] for r in rows),
        "workload": "cfg3: %s; the first %d draws whose oracle search tree stays within %d "
                    "tasks and %d parent-vertex reads (%.0f%% of draws; the rest run for "
                    "minutes to hours each)" % (BATCH_WORKLOADS["cfg3"]["desc"], n_inst,
                                               man["budget"]["max_tasks"],
                                               man["budget"]["max_parent_vertices"],
                                               100 * man["kept_fraction"]),
        "parity": "every instance's maximal sets equal the oracle's (digests in the manifest)",
    }
    ctx.close()
    pctx.close()
    if standalone:
        line = {
            "metric": "instances/s (batched: all instances in one persistent launch)",
            "value": out["value"], "unit": "instances/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": b, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "cfg3", "instances": n_inst, "l2": "inputs resident; no flush",
                       "parallelism": "one persistent launch"},
            "batched": out,
        }
        print(json.dumps(line))
    return out


def run_budgeted(args, w="cfg2"):
    """A workload whose search does not finish in minutes (config 2: its planted
    groups of up to 60 vertices at density 0.85 make an astronomically large
    enumeration tree), measured under a fixed time budget: the expansion kernel
    stops after `budget_ms` and reports the tasks and branches it expanded
    (qc_context_last_stats); the reference's own CPU path runs on the same graph
    under a wall-clock budget checked between its levels."""
    import cuqc_b200 as Q

    g, spec = make_graph(w)
    gamma, ms = float(spec["gamma"]), spec["min_size"]
    budget = args.budget_ms
    out = {"workload": "%s: %s" % (w, spec["desc"]), "budget_ms": budget}
    with Q.Context(device=0, time_limit_ms=budget) as ctx:
        dg = ctx.upload(g)
        ctx.mine_budgeted(dg, gamma, ms)  # sizes the buffers
        runs = [ctx.mine_budgeted(dg, gamma, ms) for _ in range(2)]
    st = runs[-1][1]
    sec = st["kernel_ms"] / 1000.0
    out["ours"] = {"finished": runs[-1][2], "kernel_ms": st["kernel_ms"], "tasks": st["tasks"],
                   "branches": st["branches"], "emitted": st["emitted"],
                   "root_size": st["root_size"], "max_task": st["max_task"],
                   "tasks_per_s": st["tasks"] / sec, "branches_per_s": st["branches"] / sec,
                   "arena_peak_bytes": st["arena_peak"]}
    from oracle import oracle
    if args.cpu_baseline and oracle.refcpu_available():
        d = tempfile.mkdtemp()
        path = os.path.join(d, "g.txt")
        graphs.write_serialized(g, path)
        r = oracle.refcpu_budget(path, spec["gamma"], ms, budget, workdir=d)
        sec_r = r["elapsed_ms"] / 1000.0
        out["reference_cpu"] = dict(r, cores=1, tasks_per_s=r["tasks"] / sec_r if sec_r else None,
                                    note="the reference's own CPU path; its budget is checked "
                                         "between levels, so a level that starts before the "
                                         "budget ends runs to completion")
    return out


def run_serving(args, standalone=True):
    """Serving: Poisson arrivals of mining queries, 90% drawn from the batched
    workload's instances and 10% config-1-sized graphs (ER n=1000 + 5 planted
    groups of 30, reseeded per query); latency p50/p99 and instances/s per rate,
    against serial one-at-a-time launches of the same queries."""
    import random

    import cuqc_b200 as Q
    from cuqc_b200.serve import Request, Server, run_poisson

    with open(BATCH_MANIFEST) as f:
        man = json.load(f)
    rows = man["instances"]
    rng = random.Random(5)
    pool = [graphs.batch_instance(r["i"]) for r in rows[:64]]
    big = [(graphs.erdos_renyi_planted(1000, 0.02, 5, 30, 0.95, seed=100 + j), "0.9", 20)
           for j in range(4)]
    n_req = args.serve_requests
    specs = [big[rng.randrange(len(big))] if rng.random() < 0.1 else pool[rng.randrange(len(pool))]
             for _ in range(n_req)]
    # serial reference: one plain launch at a time, back to back
    with Q.Context(device=0) as ctx:
        for g, gm, ms in specs[:8]:
            ctx.mine(g, float(gm), ms)
        t0 = time.perf_counter()
        alone = [ctx.mine(g, float(gm), ms).flat.tobytes() for g, gm, ms in specs]
        serial_s = time.perf_counter() - t0
    rates_out = []
    # every slot mines the distinct query graphs once before the timed rates
    warm = [(g, float(gm), ms) for g, gm, ms in pool + big]
    srv = Server(slots=args.serve_slots, warm=warm, warps_per_block=args.serve_warps)
    try:
        for rate in args.serve_rates:
            reqs = [Request(graph=g, gamma=float(gm), min_size=ms, rid=i)
                    for i, (g, gm, ms) in enumerate(specs)]
            st = run_poisson(srv, reqs, rate=rate, seed=int(rate))
            same = all(r.error is None and r.result.flat.tobytes() == a
                       for r, a in zip(reqs, alone))
            st["same_as_alone"] = same
            rates_out.append(st)
    finally:
        srv.close()
    line = {
        "metric": "serving latency p50/p99 (ms) and instances/s under Poisson arrivals",
        "value": rates_out[-1]["instances_per_s"], "unit": "instances/s", "n_gpus": 1,
        "steps": len(args.serve_rates), "warmup": 8, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": "cfg5", "requests_per_rate": n_req, "slots": args.serve_slots,
                   "warps_per_block": args.serve_warps,
                   "mix": "90% batched-workload instances (first 64 of the manifest), 10% "
                          "config-1-sized graphs"},
        "rates": rates_out,
        "serial": {"instances_per_s": n_req / serial_s, "form": "one qc_mine at a time"},
    }
    if standalone:
        print(json.dumps(line))
    return line


GOLDEN = os.path.join(ROOT, "tests", "golden")


def _golden_graph(case, workdir):
    """Path of a golden case's serialized graph (stored, or regenerated from
    its recorded generator parameters and checked against its digest)."""
    import hashlib

    if case["stored_graph"]:
        return os.path.join(GOLDEN, case["name"] + ".graph")
    g = getattr(graphs, case["generator"])(**case["kwargs"])
    path = os.path.join(workdir, case["name"] + ".graph")
    graphs.write_serialized(g, path)
    with open(path, "rb") as f:
        if hashlib.sha256(f.read()).hexdigest() != case["graph_sha256"]:
            raise SystemExit("generator output drifted for " + case["name"])
    return path


def _stdout_ms(text, key):
    for line in text.splitlines():
        if line.startswith("--->:%s: " % key):
            return float(line.split(":")[2].split()[0])
    return None


def run_refbin_compare(args):
    """The drop-in CLI on every golden graph the reference binary completed on a
    B200 (its stdout is frozen in tests/golden/refbin_logs/), run the same way
    here: one process per graph, each in its own directory.  Prints both
    programs' ENUMERATION and TOTAL lines, this build's expansion-kernel time,
    and whether the result files are identical.  The reference binary is not
    run; its numbers come from its logs."""
    import cuqc_b200 as Q

    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        cases = [c for c in json.load(f) if c.get("refbin") == "ok"]
    work = tempfile.mkdtemp(prefix="refbin_cmp_")
    rows = []
    for c in cases:
        path = _golden_graph(c, work)
        with open(os.path.join(GOLDEN, "refbin_logs", c["name"] + ".refbin.log")) as f:
            ref_log = f.read()
        d = os.path.join(work, c["name"])
        os.makedirs(d, exist_ok=True)
        enum, kern, total = [], [], []
        same = True
        for _ in range(max(1, args.steps)):
            out = os.path.join(d, "out.txt")
            rc, text = Q.cli(path, c["gamma"], c["min_size"], out, 0, cwd=d)
            if rc != 0:
                raise SystemExit("cuQC failed on %s: %s" % (c["name"], text[-400:]))
            enum.append(_stdout_ms(text, "ENUMERATION TIME"))
            kern.append(_stdout_ms(text, "EXPANSION KERNEL TIME"))
            total.append(_stdout_ms(text, "TOTAL TIME"))
            with open(out) as f1, open(os.path.join(GOLDEN, c["name"] + ".refbin.result")) as f2:
                same = same and f1.read() == f2.read()
        rows.append({"graph": c["name"], "gamma": c["gamma"], "min_size": c["min_size"],
                     "ref_enumeration_ms": _stdout_ms(ref_log, "ENUMERATION TIME"),
                     "ref_total_ms": _stdout_ms(ref_log, "TOTAL TIME"),
                     "enumeration_ms": statistics.median(enum),
                     "expansion_kernel_ms": statistics.median(kern),
                     "total_ms": statistics.median(total),
                     "result_identical": same})
    ratios = [r["ref_enumeration_ms"] / max(r["enumeration_ms"], 1.0) for r in rows]
    line = {
        "metric": "ENUMERATION TIME line of the drop-in CLI vs the reference binary's (ms)",
        "value": statistics.median(r["enumeration_ms"] for r in rows), "unit": "ms",
        "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": 0,
        "dtype": "int32", "data": "golden graphs the reference binary completed on a B200",
        "config": {"workload": "refbin-goldens", "graphs": len(rows),
                   "reference": "frozen stdout of the reference binary (main.cu built for "
                                "sm_100a, one run per graph on a B200 of this pool)"},
        "graphs": rows,
        "all_results_identical": all(r["result_identical"] for r in rows),
        "min_ratio_at_1ms_floor": min(ratios),
    }
    print(json.dumps(line))


def max_over_ranks(x, dist=None, device=None):
    """The largest of every rank's `x` (each rank passes its own; with no
    process group, x itself).  Every rank takes this step, in the same order."""
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(warmup, steps, step, ok, barrier, dist=None, device=None):
    """The timed loop every rank runs on its own replica of the instance
    (instances are independent: no data-path collective).  `step()` mines once
    and returns (result, device ms); `ok(result)` checks it against this rank's
    expected result.  After `warmup` untimed steps and a barrier, `steps` timed
    steps; the job's time is the slowest rank's (max over ranks) and the rate
    counts every rank's steps.  Returns (rate per second, slowest total ms,
    the timed results)."""
    for _ in range(warmup):
        step()
    barrier()
    elapsed = 0.0
    outs = []
    for _ in range(steps):
        r, ms = step()
        if not ok(r):
            raise SystemExit("a replica's result differs from its expected result")
        elapsed += ms
        outs.append(r)
    barrier()
    slowest = max_over_ranks(elapsed, dist, device)
    world = dist.get_world_size() if dist else 1
    return world * steps / (slowest / 1000.0), slowest, outs


def replica_device():
    """The GPU of this rank: one process per GPU, rank i of a node on GPU
    LOCAL_RANK (torchrun sets it)."""
    return int(os.environ.get("LOCAL_RANK", os.environ.get("RANK", "0")))


def spawn_ranks(args):
    """`bench.py --gpus N` started without a launcher: run the same command
    under torch.distributed.run with N ranks on this node (127.0.0.1
    rendezvous) and return its exit code; rank 0 prints the JSON line."""
    import socket

    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(args.gpus), "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def run_ours(args):
    import torch

    import cuqc_b200 as Q

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = replica_device()
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    w = args.workload
    g, spec = make_graph(w)
    gamma, ms = float(spec["gamma"]), spec["min_size"]
    ctx = Q.Context(device=local)
    dg = ctx.upload(g)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()

    def step():
        with torch.cuda.stream(stream):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        res = ctx.mine(dg, gamma, ms)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        launch_log.append(res.stats["kernel_launches"])
        return res, e0.elapsed_time(e1)

    res = ctx.mine(dg, gamma, ms)
    ref_sets = res.sets
    launch_log = [res.stats["kernel_launches"]]  # the context's cumulative launch count
    for _ in range(args.warmup):
        step()
    with ClockSampler(local) as clocks:  # sampled over the timed steps only
        value, elapsed_max, outs = replica_rate(
            0, args.steps, step, lambda r: r.sets == ref_sets, barrier, dist, dev)
    stats = [r.stats for r in outs]
    launches = launch_log[-1] - launch_log[args.warmup]  # the timed steps' own launches

    # e2e: from host CSR arrays through the C ABI, result read back
    barrier()
    e2e_t0 = time.perf_counter()
    outs = []
    for _ in range(args.steps):
        dg2 = Q.DeviceGraph.from_graph(g)
        r2 = ctx.mine(dg2, gamma, ms)
        dg2.close()
        outs.append(r2)  # the result is on the host; checked after the timed loop
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - e2e_t0
    assert all(r2.sets == ref_sets for r2 in outs)
    e2e_value = world * args.steps / max_over_ranks(e2e_s, dist, dev)
    h2d = 8 * (g.n + 1) * 2 + 4 * g.m + 4 * g.m2
    d2h = 4 * sum(1 + len(s) for s in ref_sets)

    if rank == 0:
        st = stats[-1]
        kernel_ms = statistics.mean(s["kernel_ms"] for s in stats)
        # algorithmic bytes per launch: per expanded branch 16 B per parent vertex
        # record + 4 B per entry of the added vertex's 1-hop and 2-hop rows
        # + 16 B per child vertex record + 4 B per emitted int
        b_alg = 16 * st["parent_vertices"] + 4 * st["p_rows"] + 16 * st["child_vertices"] + \
            4 * st["emitted_ints"]
        peak, peak_kind = load_peaks()
        achieved = b_alg / (kernel_ms / 1000.0) / 1e9
        line = {
            "metric": "instances/s (maximal gamma-quasi-clique enumeration)",
            "value": value, "unit": "instances/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator: %s)" % spec["desc"],
            "config": arm_config(w),
            "l2": "flushed before every step (256 MiB write, untimed)",
            "parallelism": "replicas (one instance per GPU per step)",
            "enum_ms": statistics.mean(s["enum_ms"] for s in stats),
            "kernel_ms": kernel_ms,
            "filter_ms": statistics.mean(s["filter_ms"] for s in stats),
            "tasks": st["tasks"], "branches": st["branches"],
            "tasks_per_s": st["tasks"] / (elapsed_max / args.steps / 1000.0),
            "maximal": len(ref_sets),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": load_traffic() if w == "cfg1" else None,
                         "traffic_source": "ncu capture summarised in profiles/expand_kernel_cfg1.md",
                         "kernel": "expand_kernel", "peak_source": peak_kind,
                         "alg_bytes_per_launch": b_alg},
            "e2e": {"value": e2e_value, "unit": "instances/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        if args.batch and world == 1 and os.path.exists(BATCH_MANIFEST):
            ctx.close()
            ctx = None
            line["batched"] = run_batch(args, standalone=False)
        if args.serve_in_default and world == 1:
            if ctx is not None:
                ctx.close()
                ctx = None
            import copy
            a2 = copy.copy(args)
            a2.serve_requests, a2.serve_rates = 150, [30.0, 100.0]
            sv = run_serving(a2, standalone=False)
            line["serving"] = {"workload": "cfg5", "config": sv["config"], "rates": sv["rates"],
                               "serial": sv["serial"]}
        if args.budget_ms > 0 and world == 1:
            if ctx is not None:
                ctx.close()
                ctx = None
            line["cfg2_budgeted"] = run_budgeted(args)
        if args.cpu_baseline and world == 1:
            from oracle import oracle
            if oracle.refcpu_available():
                d = tempfile.mkdtemp()
                path = os.path.join(d, "g.txt")
                graphs.write_serialized(g, path)
                procs = 1
                rate, per, wall, nmax = cpu_reference_rate(path, spec, procs, args.cpu_instances)
                line["cpu_baseline"] = {
                    "value": rate, "unit": "instances/s", "cores": procs, "kind": "reference",
                    "sample": "%d full instance(s) on 1 core; the reference's own CPU path "
                              "(enumeration + RemoveNonMax, file parse excluded)"
                              % args.cpu_instances}
        print(json.dumps(line))
    if ctx is not None:
        ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(WORKLOADS) + sorted(BATCH_WORKLOADS) + ["cfg5", "refbin-goldens"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-instances", type=int, default=8)
    ap.add_argument("--instances", type=int, default=256, help="batched workload size")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="batched launch with default settings instead of qc_tune_batch's")
    ap.add_argument("--no-batch", dest="batch", action="store_false",
                    help="skip the batched-vs-plain comparison in the default run")
    ap.add_argument("--budget-ms", type=int, default=500,
                    help="time budget of the config-2 measurement in the default run (0: skip)")
    ap.add_argument("--no-serve", dest="serve_in_default", action="store_false",
                    help="skip the short serving measurement in the default run")
    ap.add_argument("--serve-requests", type=int, default=300)
    ap.add_argument("--serve-slots", type=int, default=2)
    ap.add_argument("--serve-warps", type=int, default=8, help="warps per block of each slot")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[10, 30, 100, 300, 1000])
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args))
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "cfg5":
        run_serving(args)
    elif args.workload == "refbin-goldens":
        run_refbin_compare(args)
    elif args.workload == "cfg2":
        b = run_budgeted(args, "cfg2")
        o = b["ours"]
        print(json.dumps({
            "metric": "tasks expanded/s under a %d ms time budget (the search does not finish)"
                      % args.budget_ms,
            "value": o["tasks_per_s"], "unit": "tasks/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": {"workload": "cfg2", "budget_ms": args.budget_ms},
            "cfg2_budgeted": b}))
    elif args.workload in BATCH_WORKLOADS:
        run_batch(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
