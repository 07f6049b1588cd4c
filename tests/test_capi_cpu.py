"""C ABI checks that need no GPU: the library loads and exports every symbol
include/qc.h declares; graph I/O and validation through the ABI; mining fails
loudly (no CPU fallback) when no device is visible."""
import os
import re
import tempfile

import numpy as np
import pytest

import cuqc_b200 as Q
from cuqc_b200 import graphs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(Q.LIB_PATH):
        Q.build()


def declared_symbols():
    syms = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            syms += re.findall(r"\b(qc_[a-z0-9_]+)\s*\(", text)
    return sorted(set(syms))


def test_every_declared_symbol_is_exported():
    L = Q.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(Q.EXPORTS) <= set(syms)


def test_status_strings():
    L = Q.lib()
    for code in range(11):
        assert L.qc_status_str(code).decode()


def test_serialized_round_trip_through_abi():
    g = graphs.random_small(30, 0.2, 5, planted=1, size=8)
    d = tempfile.mkdtemp()
    p1, p2 = os.path.join(d, "a.txt"), os.path.join(d, "b.txt")
    graphs.write_serialized(g, p1)
    dg = Q.DeviceGraph.read(p1)
    back = dg.to_graph()
    assert back.n == g.n
    for a, b in ((back.off, g.off), (back.adj, g.adj), (back.off2, g.off2), (back.adj2, g.adj2)):
        assert np.array_equal(a, b)
    dg.write(p2)
    assert open(p1).read() == open(p2).read()


def test_from_csr2_matches_file():
    g = graphs.random_small(25, 0.3, 9)
    dg = Q.DeviceGraph.from_graph(g)
    back = dg.to_graph()
    assert np.array_equal(back.adj2, g.adj2)


@pytest.mark.parametrize("mutate,msg", [
    ("asym", "undirected"), ("selfloop", "self loop"), ("unsorted", "sorted"),
    ("range", "out of range"),
])
def test_malformed_graphs_are_rejected(mutate, msg):
    g = graphs.random_small(20, 0.3, 3)
    adj = g.adj.copy()
    off = g.off.copy()
    if mutate == "asym":
        # drop one direction of the first edge
        adj = np.delete(adj, 0)
        off = off.copy(); off[1:] -= 1
    elif mutate == "selfloop":
        v = int(np.argmax(np.diff(off) > 0)); adj[off[v]] = v
        adj[off[v]:off[v + 1]] = np.sort(adj[off[v]:off[v + 1]])
    elif mutate == "unsorted":
        v = int(np.argmax(np.diff(off) > 1)); a, b = off[v], off[v] + 1
        adj[a], adj[b] = adj[b], adj[a]
    elif mutate == "range":
        adj[0] = 10_000
    bad = graphs.Graph(n=g.n, off=off, adj=adj, off2=g.off2, adj2=g.adj2)
    with pytest.raises(Q.QCError) as e:
        Q.DeviceGraph.from_graph(bad)
    assert e.value.status == 3 and msg in str(e.value)


@pytest.mark.parametrize("mutate,msg", [
    ("unsorted", "2-hop rows must be sorted"), ("duplicate", "2-hop rows must be sorted"),
    ("range", "2-hop neighbour id out of range"), ("negative", "2-hop neighbour id out of range"),
    ("offsets", "2-hop offsets"),
])
def test_malformed_twohop_lists_are_rejected(mutate, msg):
    g = graphs.random_small(24, 0.3, 5)
    off2, adj2 = g.off2.copy(), g.adj2.copy()
    v = int(np.argmax(np.diff(off2) > 2))
    a = int(off2[v])
    if mutate == "unsorted":
        adj2[a], adj2[a + 1] = adj2[a + 1], adj2[a]
    elif mutate == "duplicate":
        adj2[a + 1] = adj2[a]
    elif mutate == "range":
        adj2[int(off2[v + 1]) - 1] = g.n  # last of a row: one past the ids
    elif mutate == "negative":
        adj2[a] = -1
    elif mutate == "offsets":
        off2[v + 1] = off2[v] - 1
    bad = graphs.Graph(n=g.n, off=g.off, adj=g.adj, off2=off2, adj2=adj2)
    with pytest.raises(Q.QCError) as e:
        Q.DeviceGraph.from_graph(bad)
    assert e.value.status == 3 and msg in str(e.value)


@pytest.mark.parametrize("which,end", [("1-hop", -1), ("2-hop", -5), ("1-hop", 1 << 62),
                                        ("2-hop", "start")])
def test_offsets_are_checked_before_the_rows_are_copied(which, end):
    # a negative or impossible entry count, or offsets not starting at 0, is a
    # format error returned before any row is read (the count would otherwise
    # size the copy of the caller's ids)
    g = graphs.random_small(16, 0.3, 2)
    off, off2 = g.off.copy(), g.off2.copy()
    o = off if which == "1-hop" else off2
    if end == "start":
        o[0] = 1
    else:
        o[-1] = end
    bad = graphs.Graph(n=g.n, off=off, adj=g.adj, off2=off2, adj2=g.adj2)
    with pytest.raises(Q.QCError) as e:
        Q.DeviceGraph.from_graph(bad)
    assert e.value.status == 3 and which + " offsets" in str(e.value)


def test_truncated_file_is_a_format_error():
    g = graphs.random_small(20, 0.3, 4)
    d = tempfile.mkdtemp()
    p = os.path.join(d, "g.txt")
    graphs.write_serialized(g, p)
    text = open(p).read()
    open(p, "w").write(text[: len(text) // 2])
    with pytest.raises(Q.QCError) as e:
        Q.DeviceGraph.read(p)
    assert e.value.status == 3


def test_missing_file_is_an_io_error():
    with pytest.raises(Q.QCError) as e:
        Q.DeviceGraph.read("/nonexistent/graph.txt")
    assert e.value.status == 2


def test_mining_without_a_device_fails_loudly(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is visible")
    g = graphs.random_small(20, 0.3, 4)
    with pytest.raises(Q.QCError) as e:
        Q.mine(g, 0.8, 4)
    assert e.value.status == 10


def test_binary_round_trip_through_abi():
    """Binary CSR file: write, read back (auto-detected), same arrays as the
    serialized text gives; a file whose size disagrees with its header, or
    with a bad magic, is refused."""
    g = graphs.random_small(40, 0.2, 6, planted=2, size=8)
    d = tempfile.mkdtemp()
    txt, binp = os.path.join(d, "g.txt"), os.path.join(d, "g.bin")
    graphs.write_serialized(g, txt)
    Q.DeviceGraph.read(txt).write_binary(binp)
    assert open(binp, "rb").read(8) == b"QCSRBIN1"
    back = Q.DeviceGraph.read(binp).to_graph()
    for a, b in ((back.off, g.off), (back.adj, g.adj), (back.off2, g.off2), (back.adj2, g.adj2)):
        assert np.array_equal(a, b)
    raw = open(binp, "rb").read()
    bad = os.path.join(d, "bad.bin")
    for blob, msg in ((raw[:-4], "does not match its header"), (b"QCSRBIN2" + raw[8:], "")):
        open(bad, "wb").write(blob)
        with pytest.raises(Q.QCError) as e:
            h = Q.C.c_void_p()
            Q._check(Q.lib().qc_graph_read_binary(bad.encode(), Q.C.byref(h)))
        assert e.value.status == 3 and msg in str(e.value)


def test_an_offset_past_the_rows_is_rejected_before_any_row_is_read():
    # a middle offset beyond the array's end (the total still right): the
    # offsets are checked before a row is read, so nothing past the array is
    g = graphs.random_small(24, 0.3, 5)
    off2 = g.off2.copy()
    off2[3] = int(g.off2[-1]) + 1000
    bad = graphs.Graph(n=g.n, off=g.off, adj=g.adj, off2=off2, adj2=g.adj2)
    with pytest.raises(Q.QCError) as e:
        Q.DeviceGraph.from_graph(bad)
    assert e.value.status == 3 and "offsets decrease" in str(e.value)
