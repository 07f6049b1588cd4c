"""ctypes front-end of the CPU oracle (TEST INFRASTRUCTURE, not product code).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; it is the checker, never the thing measured or shipped.

* ``mine``     -- every quasi-clique the reference's rules emit
                  (restates Mike12041204/cuQC main.cu:846-2198; see qc_oracle.c)
* ``maximal``  -- maximal filter + lexicographic order (main.cu:4571-4960)
* ``twohop``   -- two-hop lists (adjToSer.cpp:115-156)
* ``brute``    -- definitional brute force for n <= 24
* ``refcpu_*`` -- the reference's own serial CPU path, compiled from the
                  reference sources by oracle/Makefile into oracle/_ref/
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libqc_oracle.so")
REFCPU_PATH = os.path.join(HERE, "_ref", "libqc_refcpu.so")
ADJTOSER_PATH = os.path.join(HERE, "_ref", "adjToSer")

MODE_HOST, MODE_BINARY, MODE_CLEAN = 0, 1, 2
_MODES = {"host": MODE_HOST, "binary": MODE_BINARY, "clean": MODE_CLEAN}


class Stats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "tasks", "lookahead_hits", "branches", "children", "emitted", "emitted_vertices",
        "parent_vertices", "p_rows", "child_vertices", "max_task", "root_size",
        "stale_uses", "stale_oob", "tasks_le32", "tasks_le64", "tasks_le128", "tasks_gt128",
        "branches_le32", "branches_le64", "branches_le128", "branches_gt128")]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


_lib = None


def build():
    """Compile qc_oracle.c (gcc, ~1 s) if the shared object is missing or stale."""
    src = os.path.join(HERE, "qc_oracle.c")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-o", LIB_PATH, src, "-lm"])


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P64, P32 = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        L.qo_mine.argtypes = [C.c_int, P64, P32, P64, P32, C.c_double, C.c_int, C.c_int,
                              P64, P64, C.POINTER(P32), C.POINTER(Stats)]
        L.qo_mine.restype = C.c_int
        L.qo_maximal.argtypes = [P32, C.c_int64, P64, P64, C.POINTER(P32)]
        L.qo_maximal.restype = C.c_int
        L.qo_twohop.argtypes = [C.c_int, P64, P32, P64, C.c_int64, P32, P64]
        L.qo_twohop.restype = C.c_int
        L.qo_brute.argtypes = [C.c_int, P64, P32, C.c_double, C.c_int, P64, P64, C.POINTER(P32)]
        L.qo_brute.restype = C.c_int
        L.qo_free.argtypes = [C.c_void_p]
        L.qo_set_task_budget.argtypes = [C.c_int64]
        _lib = L
    return _lib


def _p64(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _p32(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _take(buf, nints):
    L = lib()
    if nints == 0:
        L.qo_free(C.cast(buf, C.c_void_p))
        return np.zeros(0, np.int32)
    arr = np.ctypeslib.as_array(buf, shape=(nints,)).copy()
    L.qo_free(C.cast(buf, C.c_void_p))
    return arr


def unpack(flat):
    """[k, ids..., k, ids...] -> list of tuples."""
    out, p, flat = [], 0, np.asarray(flat)
    while p < len(flat):
        k = int(flat[p])
        out.append(tuple(int(x) for x in flat[p + 1:p + 1 + k]))
        p += 1 + k
    return out


class BudgetExceeded(RuntimeError):
    """The search tree has more tasks than the budget given to ``mine``."""


def mine(g, gamma, min_size, mode="clean", max_tasks=0):
    """Run the oracle enumeration. Returns (flat emitted sets, stats dict).
    With ``max_tasks`` > 0, raises BudgetExceeded once more tasks than that
    would be expanded."""
    L = lib()
    L.qo_set_task_budget(C.c_int64(int(max_tasks)))
    off, adj = np.ascontiguousarray(g.off, np.int64), np.ascontiguousarray(g.adj, np.int32)
    off2, adj2 = np.ascontiguousarray(g.off2, np.int64), np.ascontiguousarray(g.adj2, np.int32)
    ns, ni = C.c_int64(), C.c_int64()
    buf = C.POINTER(C.c_int32)()
    st = Stats()
    rc = L.qo_mine(int(g.n), _p64(off), _p32(adj), _p64(off2), _p32(adj2), float(gamma),
                   int(min_size), _MODES[mode], C.byref(ns), C.byref(ni), C.byref(buf),
                   C.byref(st))
    L.qo_set_task_budget(C.c_int64(0))
    if rc == -2:
        _take(buf, ni.value)
        raise BudgetExceeded("more than %d tasks" % max_tasks)
    if rc != 0:
        raise RuntimeError("oracle enumeration failed")
    return _take(buf, ni.value), st.as_dict()


def maximal(flat):
    """Maximal sets of an emitted family, each sorted, in lexicographic order."""
    L = lib()
    flat = np.ascontiguousarray(flat, np.int32)
    nsets = 0
    p = 0
    while p < len(flat):
        nsets += 1
        p += 1 + int(flat[p])
    ns, ni = C.c_int64(), C.c_int64()
    buf = C.POINTER(C.c_int32)()
    if L.qo_maximal(_p32(flat), nsets, C.byref(ns), C.byref(ni), C.byref(buf)) != 0:
        raise RuntimeError("oracle maximal filter failed")
    return unpack(_take(buf, ni.value))


def result_text(sets):
    """Result-file text in the reference's line format (main.cu:4641-4652)."""
    return "".join("%d " % len(s) + "".join("%d " % v for v in s) + "\n" for s in sets)


def solve(g, gamma, min_size, mode="clean", max_tasks=0):
    flat, st = mine(g, gamma, min_size, mode, max_tasks)
    return maximal(flat), st


def twohop(n, off, adj):
    L = lib()
    off = np.ascontiguousarray(off, np.int64)
    adj = np.ascontiguousarray(adj, np.int32)
    cap = 1 << 20
    while True:
        off2 = np.zeros(n + 1, np.int64)
        adj2 = np.zeros(max(cap, 1), np.int32)
        n2 = C.c_int64()
        rc = L.qo_twohop(n, _p64(off), _p32(adj), _p64(off2), cap, _p32(adj2), C.byref(n2))
        if rc == -2:
            cap *= 4
            continue
        if rc != 0:
            raise RuntimeError("twohop failed")
        return off2, adj2[:n2.value].copy()


def brute(g, gamma, min_size):
    L = lib()
    off, adj = np.ascontiguousarray(g.off, np.int64), np.ascontiguousarray(g.adj, np.int32)
    ns, ni = C.c_int64(), C.c_int64()
    buf = C.POINTER(C.c_int32)()
    if L.qo_brute(int(g.n), _p64(off), _p32(adj), float(gamma), int(min_size),
                  C.byref(ns), C.byref(ni), C.byref(buf)) != 0:
        raise RuntimeError("brute force needs n <= 24")
    return maximal(_take(buf, ni.value))


# ---------------------------------------------------------------------------
# the reference's own CPU path (oracle/_ref, built from the reference sources)
# ---------------------------------------------------------------------------

_refcpu = None


def refcpu_available():
    return os.path.exists(REFCPU_PATH)


def refcpu_run(graph_path, gamma_str, min_size, workdir=None, caps=None, times=None):
    """Run the reference's serial CPU enumeration + RemoveNonMax.

    Returns (result text, emitted sets from its temp file as a flat list).
    If `times` is a dict it receives load_ms, enum_ms, rm_ms."""
    global _refcpu
    if _refcpu is None:
        L = C.CDLL(REFCPU_PATH)
        L.refcpu_run.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_char_p,
                                 C.c_longlong, C.c_longlong, C.c_longlong, C.c_longlong,
                                 C.POINTER(C.c_longlong), C.POINTER(C.c_double)]
        L.refcpu_run.restype = C.c_int
        _refcpu = L
    caps = caps or (1 << 26, 1 << 28, 1 << 24, 1 << 26)
    wd = workdir or tempfile.mkdtemp(prefix="refcpu_")
    temp, out = os.path.join(wd, "temp.txt"), os.path.join(wd, "out.txt")
    lv = C.c_longlong()
    tms = (C.c_double * 3)()
    cwd = os.getcwd()
    os.chdir(wd)  # RemoveNonMax prints only; files are explicit paths
    try:
        rc = _refcpu.refcpu_run(graph_path.encode(), str(gamma_str).encode(), int(min_size),
                                temp.encode(), out.encode(), *caps, C.byref(lv), tms)
    finally:
        os.chdir(cwd)
    if rc < 0:
        raise RuntimeError("reference CPU path could not read %s" % graph_path)
    if times is not None:
        times.update(load_ms=tms[0], enum_ms=tms[1], rm_ms=tms[2])
    with open(out) as f:
        text = f.read()
    flat = []
    with open(temp) as f:
        tok = f.read().split()
    p = 0
    while p < len(tok):
        k = int(tok[p])
        flat.append(k)
        flat.extend(int(x) for x in tok[p + 1:p + 1 + k])
        p += 1 + k
    return text, np.asarray(flat, np.int32)


def refcpu_budget(graph_path, gamma_str, min_size, budget_ms, workdir=None, caps=None):
    """The reference's serial CPU enumeration under a wall-clock budget
    (checked between its levels).  Returns a dict: tasks expanded, sets
    emitted, levels, finished (bool), elapsed_ms."""
    L = C.CDLL(REFCPU_PATH)
    L.refcpu_budget.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_double,
                                C.c_longlong, C.c_longlong, C.c_longlong, C.c_longlong,
                                C.POINTER(C.c_longlong), C.POINTER(C.c_double)]
    L.refcpu_budget.restype = C.c_int
    caps = caps or (1 << 26, 1 << 28, 1 << 24, 1 << 26)
    wd = workdir or tempfile.mkdtemp(prefix="refcpu_")
    temp = os.path.join(wd, "temp.txt")
    out = (C.c_longlong * 4)()
    el = C.c_double()
    rc = L.refcpu_budget(graph_path.encode(), str(gamma_str).encode(), int(min_size),
                         temp.encode(), float(budget_ms), *caps, out, C.byref(el))
    if rc < 0:
        raise RuntimeError("reference CPU path could not read %s" % graph_path)
    try:
        os.remove(temp)
    except OSError:
        pass
    return {"tasks": int(out[0]), "emitted": int(out[1]), "levels": int(out[2]),
            "finished": bool(out[3]), "elapsed_ms": float(el.value)}


def adjtoser(adjlist_path, out_path):
    """The reference's adjacency-list -> serialized converter (adjToSer.cpp)."""
    subprocess.check_call([ADJTOSER_PATH, adjlist_path, out_path])


def root(g, gamma, min_size):
    """Level-0 root task: (ids, labels, exdeg) in Q order (main.cu:846-998)."""
    L = lib()
    if not hasattr(L, "_root_set"):
        P64, P32 = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        L.qo_root.argtypes = [C.c_int, P64, P32, P64, P32, C.c_double, C.c_int, P32, P32, P32]
        L.qo_root.restype = C.c_int
        L._root_set = True
    n = int(g.n)
    ids, lab, ex = (np.zeros(max(n, 1), np.int32) for _ in range(3))
    off, adj = np.ascontiguousarray(g.off, np.int64), np.ascontiguousarray(g.adj, np.int32)
    off2, adj2 = np.ascontiguousarray(g.off2, np.int64), np.ascontiguousarray(g.adj2, np.int32)
    r = L.qo_root(n, _p64(off), _p32(adj), _p64(off2), _p32(adj2), float(gamma), int(min_size),
                  _p32(ids), _p32(lab), _p32(ex))
    if r < 0:
        raise RuntimeError("oracle root failed")
    return ids[:r].copy(), lab[:r].copy(), ex[:r].copy()
