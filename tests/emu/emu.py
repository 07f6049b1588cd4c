"""Builds and drives the CPU-emulated expansion kernel (TEST INFRASTRUCTURE).

The product kernel source is compiled by g++ against tests/emu/cuda_emu.h;
each emulated lane is a host thread.  Used only by the CPU test suite.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SO = os.path.join(HERE, "_build", "libqc_emu.so")
SRCS = [os.path.join(HERE, "emu_expand.cpp"), os.path.join(ROOT, "cuqc_b200", "csrc", "host.cpp")]
DEPS = SRCS + [os.path.join(HERE, "cuda_emu.h"),
               os.path.join(ROOT, "cuqc_b200", "csrc", "expand_kernel.cuh"),
               os.path.join(ROOT, "cuqc_b200", "csrc", "level0_kernel.cuh"),
               os.path.join(ROOT, "cuqc_b200", "csrc", "level0_grid.cuh"),
               os.path.join(ROOT, "cuqc_b200", "csrc", "qc_device.h"),
               os.path.join(ROOT, "cuqc_b200", "csrc", "host.h")]

_lib = None


def build():
    newest = max(os.path.getmtime(p) for p in DEPS)
    if os.path.exists(SO) and os.path.getmtime(SO) >= newest:
        return
    os.makedirs(os.path.dirname(SO), exist_ok=True)
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-g", "-pthread", "-shared", "-fPIC",
                           "-Wno-unused-variable", "-o", SO] + SRCS)


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(SO)
        P64, P32 = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        L.emu_mine.argtypes = [C.c_int, P64, P32, P64, P32, C.c_double, C.c_int, C.c_int, C.c_int,
                               C.c_int, C.c_longlong, P64, C.POINTER(P32), P64, C.c_int,
                               C.c_longlong, C.c_int]
        L.emu_mine.restype = C.c_int
        L.emu_free.argtypes = [C.c_void_p]
        L.emu_level0.argtypes = [C.c_int, P64, P32, P64, C.c_double, C.c_int, C.c_int, P32, P32]
        L.emu_level0.restype = C.c_int
        L.emu_level0_grid.argtypes = L.emu_level0.argtypes
        L.emu_level0_grid.restype = C.c_int
        _lib = L
    return _lib


def mine(g, gamma, min_size, warps=2, split=4, arena_bytes=64 << 20, small_path=1, stack_cap=0,
         result_cap=0, shared_fifo=0):
    """Emitted multiset (flat [k, ids..]) and counters of the emulated kernel."""
    L = lib()
    off, adj = np.ascontiguousarray(g.off, np.int64), np.ascontiguousarray(g.adj, np.int32)
    off2, adj2 = np.ascontiguousarray(g.off2, np.int64), np.ascontiguousarray(g.adj2, np.int32)
    ni = C.c_int64()
    buf = C.POINTER(C.c_int32)()
    cnt = np.zeros(11, np.int64)
    st = L.emu_mine(int(g.n), off.ctypes.data_as(P64 := C.POINTER(C.c_int64)),
                    adj.ctypes.data_as(C.POINTER(C.c_int32)), off2.ctypes.data_as(P64),
                    adj2.ctypes.data_as(C.POINTER(C.c_int32)), float(gamma), int(min_size),
                    int(warps), int(split), int(small_path), int(arena_bytes), C.byref(ni),
                    C.byref(buf),
                    cnt.ctypes.data_as(P64), int(stack_cap), int(result_cap), int(shared_fifo))
    flat = np.zeros(0, np.int32)
    if ni.value:
        flat = np.ctypeslib.as_array(buf, shape=(ni.value,)).copy()
        L.emu_free(C.cast(buf, C.c_void_p))
    keys = ["tasks", "branches", "children", "emitted", "lookahead_hits", "status", "max_task",
            "arena_bytes", "parent_vertices", "p_rows", "child_vertices"]
    return flat, dict(zip(keys, (int(x) for x in cnt))), st


def mine_batch(gs, gammas, min_sizes, warps=3, split=2):
    """Emulated batched launch; returns per-instance emitted flat lists (local ids)."""
    L = lib()
    if not hasattr(L, "_batch_set"):
        P64, P32 = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        L.emu_mine_batch.argtypes = [C.c_int, P32, P64, P32, P64, P32, C.POINTER(C.c_double), P32,
                                     C.c_int, C.c_int, P64, C.POINTER(P32), P64]
        L.emu_mine_batch.restype = C.c_int
        L._batch_set = True
    ns = np.array([g.n for g in gs], np.int32)
    off = np.concatenate([np.asarray(g.off, np.int64) for g in gs])
    off2 = np.concatenate([np.asarray(g.off2, np.int64) for g in gs])
    adj = np.concatenate([np.asarray(g.adj, np.int32) for g in gs])
    adj2 = np.concatenate([np.asarray(g.adj2, np.int32) for g in gs])
    gm = np.asarray(gammas, np.float64)
    ms = np.asarray(min_sizes, np.int32)
    ni = C.c_int64()
    buf = C.POINTER(C.c_int32)()
    cnt = np.zeros(3, np.int64)
    P64, P32 = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
    st = L.emu_mine_batch(len(gs), ns.ctypes.data_as(P32), off.ctypes.data_as(P64),
                          adj.ctypes.data_as(P32), off2.ctypes.data_as(P64), adj2.ctypes.data_as(P32),
                          gm.ctypes.data_as(C.POINTER(C.c_double)), ms.ctypes.data_as(P32),
                          int(warps), int(split), C.byref(ni), C.byref(buf), cnt.ctypes.data_as(P64))
    flat = np.zeros(0, np.int32)
    if ni.value:
        flat = np.ctypeslib.as_array(buf, shape=(ni.value,)).copy()
        L.emu_free(C.cast(buf, C.c_void_p))
    vb = np.concatenate([[0], np.cumsum(ns)])[:-1]
    per = [[] for _ in gs]
    p = 0
    while p < len(flat):
        k = int(flat[p])
        ids = flat[p + 1:p + 1 + k]
        i = int(np.searchsorted(vb, ids[0], side="right") - 1)
        per[i].append(k)
        per[i].extend(int(x) - int(vb[i]) for x in ids)
        p += 1 + k
    return per, st


def level0(g, gamma, min_size, threads=64, grid=False):
    """Root ids (Q order) and covered count from the product's device level 0
    run as one emulated block: the one-block form (level0_kernel.cuh) or, with
    grid=True, the grid-wide form (level0_grid.cuh) as a grid of one block."""
    L = lib()
    P64, P32 = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
    off, adj = np.ascontiguousarray(g.off, np.int64), np.ascontiguousarray(g.adj, np.int32)
    off2 = np.ascontiguousarray(g.off2, np.int64)
    ids = np.zeros(max(int(g.n), 1), np.int32)
    info = np.zeros(2, np.int32)
    fn = L.emu_level0_grid if grid else L.emu_level0
    fn(int(g.n), off.ctypes.data_as(P64), adj.ctypes.data_as(P32),
                 off2.ctypes.data_as(P64), float(gamma), int(min_size), int(threads),
                 ids.ctypes.data_as(P32), info.ctypes.data_as(P32))
    return ids[: int(info[0])].copy(), int(info[1])
