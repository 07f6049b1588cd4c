"""B200-native maximal gamma-quasi-clique miner (drop-in for Mike12041204/cuQC).

Python host mirror of the C ABI in include/qc.h (libqc.so).  The reference's
only interface is its CLI (main.cu:416-519) over a serialized graph file and
a result file; ``mine`` is the in-process equivalent of one CLI run and
``cli`` runs the drop-in command line itself.

There is no CPU path: if the CUDA library is missing or no GPU is visible,
every mining call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import graphs

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqc.so")
CLI_PATH = os.path.join(HERE, "cuQC")
CONVERT_PATH = os.path.join(HERE, "qc_convert")  # graph-format tools (csrc/convert.cpp)

# qc_status
STATUS = {
    0: "QC_OK", 1: "QC_ERR_ARGS", 2: "QC_ERR_IO", 3: "QC_ERR_FORMAT", 4: "QC_ERR_CUDA",
    5: "QC_ERR_NOMEM", 6: "QC_ERR_TASK_OVERFLOW", 7: "QC_ERR_RESULT_OVERFLOW",
    8: "QC_ERR_ITER_LIMIT", 9: "QC_ERR_TOO_LARGE", 10: "QC_ERR_NO_DEVICE",
}

# every symbol include/qc.h declares
EXPORTS = [
    "qc_status_str", "qc_last_error", "qc_graph_read_serialized", "qc_graph_from_csr2",
    "qc_graph_from_csr", "qc_graph_write_serialized", "qc_graph_num_vertices",
    "qc_graph_num_entries", "qc_graph_num_twohop", "qc_graph_offsets", "qc_graph_neighbors",
    "qc_graph_twohop_offsets", "qc_graph_twohop_neighbors", "qc_graph_free", "qc_config_default",
    "qc_context_create", "qc_context_free", "qc_context_upload", "qc_context_stream", "qc_mine", "qc_mine_batch", "qc_result_count",
    "qc_result_sets", "qc_result_emitted", "qc_result_stats", "qc_result_write", "qc_result_free",
    "qc_twohop_noalloc", "qc_twohop_noalloc_max_vertices", "qc_tune", "qc_maximal_sets",
    "qc_context_last_stats", "qc_root", "qc_mine_shard", "qc_graph_read_binary",
    "qc_graph_write_binary", "qc_graph_read", "qc_tune_batch", "qc_sets_write_async",
    "qc_result_write_async", "qc_writer_wait",
]


class QCError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("warps_per_block", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("arena_bytes", C.c_int64),
                ("stack_slots", C.c_int64), ("result_ints", C.c_int64),
                ("keep_emitted", C.c_int32), ("wait_limit_ms", C.c_int32),
                ("time_limit_ms", C.c_int32), ("split", C.c_int32), ("max_blocks", C.c_int32),
                ("stage_max", C.c_int32), ("shared_order", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("load_ms", C.c_double), ("enum_ms", C.c_double), ("filter_ms", C.c_double),
                ("total_ms", C.c_double)] + [(k, C.c_int64) for k in (
                    "tasks", "branches", "children", "emitted", "emitted_ints", "maximal",
                    "root_size", "max_task", "arena_peak", "kernel_launches")] + [
                    ("kernel_ms", C.c_double)] + [(k, C.c_int64) for k in (
                    "parent_vertices", "p_rows", "child_vertices", "level0_on_device")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build():
    """Compile libqc.so and the cuQC CLI for sm_100a (nvcc cross-compiles)."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "csrc")])


_lib = None


def lib():
    """The loaded CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QCError(10, "libqc.so is not built (run cuqc_b200.build())")
        L = C.CDLL(LIB_PATH)
        vp, P32, P64 = C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64)
        L.qc_status_str.restype = C.c_char_p
        L.qc_last_error.restype = C.c_char_p
        L.qc_graph_read_serialized.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.qc_graph_from_csr2.argtypes = [C.c_int32, P64, P32, P64, P32, C.POINTER(vp)]
        L.qc_graph_from_csr.argtypes = [C.c_int32, P64, P32, C.POINTER(vp)]
        L.qc_graph_write_serialized.argtypes = [vp, C.c_char_p]
        L.qc_graph_num_vertices.argtypes = [vp]
        L.qc_graph_num_entries.argtypes = [vp]
        L.qc_graph_num_entries.restype = C.c_int64
        L.qc_graph_num_twohop.argtypes = [vp]
        L.qc_graph_num_twohop.restype = C.c_int64
        for f in ("qc_graph_offsets", "qc_graph_twohop_offsets"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = P64
        for f in ("qc_graph_neighbors", "qc_graph_twohop_neighbors"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = P32
        L.qc_graph_free.argtypes = [vp]
        L.qc_config_default.argtypes = [C.POINTER(Config)]
        L.qc_context_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
        L.qc_context_free.argtypes = [vp]
        L.qc_context_upload.argtypes = [vp, vp]
        L.qc_context_stream.argtypes = [vp]
        L.qc_context_stream.restype = vp
        L.qc_mine.argtypes = [vp, vp, C.c_double, C.c_int32, C.c_int32, C.POINTER(vp)]
        L.qc_mine_batch.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_double), P32, C.c_int32,
                                    C.POINTER(vp)]
        L.qc_result_count.argtypes = [vp]
        L.qc_result_count.restype = C.c_int64
        L.qc_result_sets.argtypes = [vp, P64]
        L.qc_result_sets.restype = P32
        L.qc_result_emitted.argtypes = [vp, P64, P64]
        L.qc_result_emitted.restype = P32
        L.qc_result_stats.argtypes = [vp]
        L.qc_result_stats.restype = C.POINTER(Stats)
        L.qc_result_write.argtypes = [vp, C.c_char_p]
        L.qc_result_free.argtypes = [vp]
        L.qc_tune.argtypes = [vp, vp, C.c_double, C.c_int32, C.c_int32, C.POINTER(Config)]
        L.qc_tune_batch.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_double), P32, C.c_int32,
                                    C.c_int32, C.POINTER(Config)]
        L.qc_twohop_noalloc.argtypes = [C.c_int32, vp, vp, vp, vp, C.c_int64, P64, vp]
        L.qc_twohop_noalloc_max_vertices.restype = C.c_int32
        L.qc_maximal_sets.argtypes = [vp, P32, C.c_int64, C.c_int32, C.POINTER(vp)]
        L.qc_context_last_stats.argtypes = [vp, C.POINTER(Stats)]
        L.qc_root.argtypes = [vp, vp, C.c_double, C.c_int32, P32, C.c_int64, P32, P32]
        L.qc_graph_read_binary.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.qc_graph_write_binary.argtypes = [vp, C.c_char_p]
        L.qc_graph_read.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.qc_mine_shard.argtypes = [vp, vp, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                    C.POINTER(vp)]
        L.qc_sets_write_async.argtypes = [P32, C.c_int64, C.c_char_p, C.POINTER(vp)]
        L.qc_result_write_async.argtypes = [vp, C.c_char_p, C.POINTER(vp)]
        L.qc_writer_wait.argtypes = [vp]
        _lib = L
    return _lib


def _check(st):
    if st != 0:
        L = lib()
        raise QCError(st, L.qc_last_error().decode())


def _p64(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _p32(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class Writer:
    """A result file being written on a host thread (qc_sets_write_async);
    wait() returns once it is on disk.  Holds the set array until then."""

    def __init__(self, flat, path):
        self._flat = np.ascontiguousarray(flat, np.int32)
        self.h = C.c_void_p()
        _check(lib().qc_sets_write_async(_p32(self._flat), int(self._flat.size),
                                         os.fsencode(path), C.byref(self.h)))

    def wait(self):
        if self.h is not None:
            h, self.h = self.h, None
            _check(lib().qc_writer_wait(h))
            self._flat = None


def write_sets_async(flat, path):
    """Write flat [k, ids..]* sets as a result file in the background."""
    return Writer(flat, path)


class DeviceGraph:
    """A graph handed to the library (qc_graph)."""

    def __init__(self, handle):
        self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle

    @classmethod
    def from_graph(cls, g: graphs.Graph):
        L = lib()
        off, adj = np.ascontiguousarray(g.off, np.int64), np.ascontiguousarray(g.adj, np.int32)
        h = C.c_void_p()
        if g.off2 is None:
            _check(L.qc_graph_from_csr(int(g.n), _p64(off), _p32(adj), C.byref(h)))
        else:
            off2 = np.ascontiguousarray(g.off2, np.int64)
            adj2 = np.ascontiguousarray(g.adj2, np.int32)
            _check(L.qc_graph_from_csr2(int(g.n), _p64(off), _p32(adj), _p64(off2), _p32(adj2),
                                        C.byref(h)))
        return cls(h)

    @classmethod
    def read(cls, path):
        """A graph file of either format: binary CSR (starts with "QCSRBIN1")
        or the serialized text."""
        h = C.c_void_p()
        _check(lib().qc_graph_read(path.encode(), C.byref(h)))
        return cls(h)

    def write_binary(self, path):
        _check(lib().qc_graph_write_binary(self.h, path.encode()))

    def to_graph(self) -> graphs.Graph:
        L = lib()
        n = L.qc_graph_num_vertices(self.h)
        m, m2 = L.qc_graph_num_entries(self.h), L.qc_graph_num_twohop(self.h)
        arr = lambda p, k: np.ctypeslib.as_array(p, shape=(k,)).copy() if k else np.zeros(0, p._type_)
        return graphs.Graph(n=n, off=arr(L.qc_graph_offsets(self.h), n + 1),
                            adj=arr(L.qc_graph_neighbors(self.h), m),
                            off2=arr(L.qc_graph_twohop_offsets(self.h), n + 1),
                            adj2=arr(L.qc_graph_twohop_neighbors(self.h), m2))

    def write(self, path):
        _check(lib().qc_graph_write_serialized(self.h, path.encode()))

    def close(self):
        if self.h:
            lib().qc_graph_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Result:
    """A mining result: the maximal sets (flat [k, ids..] as returned by the
    library; `sets` converts them to sorted tuples on first use), the run's
    counters and, with keep_emitted, the raw emitted multiset."""

    def __init__(self, flat, stats, emitted=None):
        self.flat = flat
        self.stats = stats
        self.emitted = emitted
        self._sets = None

    @property
    def sets(self):
        if self._sets is None:
            self._sets = _flat_to_sets(self.flat)
        return self._sets

    def text(self):
        return "".join("%d " % len(s) + "".join("%d " % v for v in s) + "\n" for s in self.sets)

    def write(self, path):
        """The result file (the reference's format), formatted by the library."""
        write_sets_async(self.flat, path).wait()

    def write_async(self, path):
        """Start writing the result file on a host thread; returns a Writer."""
        return write_sets_async(self.flat, path)


def _flat_to_sets(flat):
    vals = flat.tolist()
    out, p = [], 0
    while p < len(vals):
        k = vals[p]
        out.append(tuple(vals[p + 1:p + 1 + k]))
        p += 1 + k
    return out


class Context:
    """qc_context: one CUDA stream plus device buffers, reused across calls."""

    def __init__(self, device=0, keep_emitted=False, **kw):
        L = lib()
        self.cfg = Config()
        L.qc_config_default(C.byref(self.cfg))
        self.cfg.device = device
        self.cfg.keep_emitted = 1 if keep_emitted else 0
        for k, v in kw.items():
            setattr(self.cfg, k, v)
        self.h = C.c_void_p()
        _check(L.qc_context_create(C.byref(self.cfg), C.byref(self.h)))

    def _result(self, r):
        L = lib()
        try:
            n = C.c_int64()
            p = L.qc_result_sets(r, C.byref(n))
            flat = np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0, np.int32)
            st = L.qc_result_stats(r).contents.as_dict()
            emitted = None
            if self.cfg.keep_emitted:
                ns, ni = C.c_int64(), C.c_int64()
                pe = L.qc_result_emitted(r, C.byref(ns), C.byref(ni))
                emitted = (np.ctypeslib.as_array(pe, shape=(ni.value,)).copy() if ni.value
                           else np.zeros(0, np.int32))
            return Result(flat, st, emitted)
        finally:
            L.qc_result_free(r)

    def upload(self, g):
        """Stage a graph on the device; later mine() calls on it skip the copy."""
        dg = g if isinstance(g, DeviceGraph) else DeviceGraph.from_graph(g)
        _check(lib().qc_context_upload(self.h, dg.h))
        return dg

    @property
    def stream(self):
        """The context's cudaStream_t as an integer."""
        return lib().qc_context_stream(self.h)

    def mine(self, g, gamma, min_size, sched=0):
        dg = g if isinstance(g, DeviceGraph) else DeviceGraph.from_graph(g)
        r = C.c_void_p()
        _check(lib().qc_mine(self.h, dg.h, float(gamma), int(min_size), int(sched), C.byref(r)))
        return self._result(r)

    def mine_files(self, jobs):
        """Mine a stream of graph files, each into its result file: jobs is an
        iterable of (graph path, gamma, min_size, result path).  Every result
        file is written on a host thread while the next graph is read and
        mined; returns each job's counters."""
        pending, stats = [], []
        try:
            for gpath, gamma, min_size, out in jobs:
                dg = DeviceGraph.read(os.fsdecode(gpath))
                try:
                    r = self.mine(dg, gamma, min_size)
                finally:
                    dg.close()
                pending.append(r.write_async(out))
                stats.append(r.stats)
                if len(pending) > 4:  # bound the results held in memory
                    pending.pop(0).wait()
        finally:
            for w in pending:
                w.wait()
        return stats

    def last_stats(self):
        """Counters of the most recent expansion on this context (dict), also
        of a run that stopped at cfg.time_limit_ms."""
        st = Stats()
        _check(lib().qc_context_last_stats(self.h, C.byref(st)))
        return st.as_dict()

    def mine_budgeted(self, g, gamma, min_size):
        """Mine with the context's time limit; returns (result or None,
        counters, finished).  A run that hits the limit gives no sets, only
        the counts of the work done until it stopped."""
        try:
            r = self.mine(g, gamma, min_size)
            return r, r.stats, True
        except QCError as e:
            if e.status != 8:
                raise
            return None, self.last_stats(), False

    def root(self, g, gamma, min_size):
        """Level 0 alone (qc_root): the root task's vertex ids in branching
        order and the number of them the cover vertex covers."""
        dg = g if isinstance(g, DeviceGraph) else DeviceGraph.from_graph(g)
        t, cov = C.c_int32(), C.c_int32()
        L = lib()
        _check(L.qc_root(self.h, dg.h, float(gamma), int(min_size), None, 0, C.byref(t),
                         C.byref(cov)))
        ids = np.zeros(max(t.value, 1), np.int32)
        _check(L.qc_root(self.h, dg.h, float(gamma), int(min_size), _p32(ids), len(ids),
                         C.byref(t), C.byref(cov)))
        return ids[: t.value].copy(), cov.value

    def mine_shard(self, g, gamma, min_size, shard, nshards):
        """Shard `shard` of `nshards` of a search split by the root's branches
        (qc_mine_shard): the maximal sets among the sets its branches emit."""
        dg = g if isinstance(g, DeviceGraph) else DeviceGraph.from_graph(g)
        r = C.c_void_p()
        _check(lib().qc_mine_shard(self.h, dg.h, float(gamma), int(min_size), int(shard),
                                   int(nshards), C.byref(r)))
        return self._result(r)

    def tune(self, g, gamma, min_size, repeats=2):
        """Pick the fastest launch shape for this device on (g, gamma,
        min_size) and keep it for later calls; returns it as a dict."""
        dg = g if isinstance(g, DeviceGraph) else DeviceGraph.from_graph(g)
        best = Config()
        _check(lib().qc_tune(self.h, dg.h, float(gamma), int(min_size), int(repeats),
                             C.byref(best)))
        self.cfg = best
        return _tuned(best)

    def tune_batch(self, gs, gammas, min_sizes, repeats=1):
        """qc_tune on a batched workload (qc_tune_batch); returns the settings."""
        dgs = [g if isinstance(g, DeviceGraph) else DeviceGraph.from_graph(g) for g in gs]
        k = len(dgs)
        ga = (C.c_void_p * k)(*[d.h for d in dgs])
        gm = np.ascontiguousarray(gammas, np.float64)
        ms = np.ascontiguousarray(min_sizes, np.int32)
        best = Config()
        _check(lib().qc_tune_batch(self.h, ga, gm.ctypes.data_as(C.POINTER(C.c_double)), _p32(ms),
                                   k, int(repeats), C.byref(best)))
        self.cfg = best
        return _tuned(best)

    def mine_batch(self, gs, gammas, min_sizes):
        L = lib()
        dgs = [g if isinstance(g, DeviceGraph) else DeviceGraph.from_graph(g) for g in gs]
        k = len(dgs)
        ga = (C.c_void_p * k)(*[d.h for d in dgs])
        gm = np.ascontiguousarray(gammas, np.float64)
        ms = np.ascontiguousarray(min_sizes, np.int32)
        outs = (C.c_void_p * k)()
        _check(L.qc_mine_batch(self.h, ga, gm.ctypes.data_as(C.POINTER(C.c_double)), _p32(ms), k,
                               outs))
        return [self._result(C.c_void_p(o)) for o in outs]

    def maximal_sets(self, flat, n_vertices):
        """The maximal sets of a family given flat as [k, ids..] per set
        (qc_maximal_sets); returns a Result."""
        f = np.ascontiguousarray(flat, np.int32)
        r = C.c_void_p()
        _check(lib().qc_maximal_sets(self.h, _p32(f), len(f), int(n_vertices), C.byref(r)))
        return self._result(r)

    def close(self):
        if self.h:
            lib().qc_context_free(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _tuned(cfg):
    return {k: getattr(cfg, k) for k in ("warps_per_block", "blocks_per_sm", "split",
                                         "stage_max", "shared_order")}


def mine(g, gamma, min_size, **kw):
    """One in-process run: maximal gamma-quasi-cliques of size >= min_size."""
    with Context(**kw) as ctx:
        return ctx.mine(g, gamma, min_size)


def cli(graph_path, gamma, min_size, out_path, sched=0, cwd=None):
    """Run the drop-in `cuQC` command line; returns (exit code, stdout)."""
    p = subprocess.run([CLI_PATH, graph_path, str(gamma), str(min_size), out_path, str(sched)],
                       capture_output=True, text=True, cwd=cwd)
    return p.returncode, p.stdout
