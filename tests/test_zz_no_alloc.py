"""qc_twohop_noalloc: the two-hop builder for callers that cannot allocate
device memory (their memory is owned by their own pool or fixed plan, or they
must not allocate while serving).  It is checked through the C ABI against the
allocating builder behind qc_graph_from_csr and against the oracle's
restatement of adjToSer, on two calls in a row, with the caller's inputs and
outputs in device buffers; at n = 0, with a self loop, at its largest vertex
count, and on malformed device CSRs, which it must refuse without writing.

This file is collected last on purpose: the no-allocation entry point shares
one device array across calls, and the test must hold both in a fresh process
and after every other test has run."""
import ctypes as C

import numpy as np
import pytest

import cuqc_b200 as Q
from cuqc_b200 import graphs
from oracle import oracle

QC_ERR_FORMAT = 3


def _allocating_twohop(g):
    """off2/adj2 from the existing GPU builder (qc_graph_from_csr)."""
    L = Q.lib()
    h = C.c_void_p()
    off = np.ascontiguousarray(g.off, np.int64)
    adj = np.ascontiguousarray(g.adj, np.int32)
    Q._check(L.qc_graph_from_csr(int(g.n), Q._p64(off), Q._p32(adj), C.byref(h)))
    try:
        n, m2 = int(g.n), int(L.qc_graph_num_twohop(h))
        off2 = np.ctypeslib.as_array(L.qc_graph_twohop_offsets(h), shape=(n + 1,)).copy()
        adj2 = np.ctypeslib.as_array(L.qc_graph_twohop_neighbors(h), shape=(m2,)).copy()
    finally:
        L.qc_graph_free(h)
    return off2, adj2


def _noalloc_twohop(g, torch):
    """off2/adj2 from qc_twohop_noalloc with every buffer owned by the caller."""
    L = Q.lib()
    dev = torch.device("cuda", 0)
    d_off = torch.as_tensor(np.asarray(g.off, np.int64), device=dev)
    d_adj = torch.as_tensor(np.asarray(g.adj, np.int32) if len(g.adj) else np.zeros(1, np.int32),
                            device=dev)
    d_off2 = torch.full((g.n + 1,), -7, dtype=torch.int64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    total = C.c_int64(-1)
    # size query first (no row buffer), as a caller sizing its own buffer would
    Q._check(L.qc_twohop_noalloc(int(g.n), C.c_void_p(d_off.data_ptr()), C.c_void_p(d_adj.data_ptr()),
                                 C.c_void_p(d_off2.data_ptr()), None, 0, C.byref(total), stream))
    need = total.value
    assert need >= 0
    # a row buffer one entry short is refused with the size it needs
    if need > 0:
        short = torch.empty(need - 1, dtype=torch.int32, device=dev)
        st = L.qc_twohop_noalloc(int(g.n), C.c_void_p(d_off.data_ptr()), C.c_void_p(d_adj.data_ptr()),
                                 C.c_void_p(d_off2.data_ptr()), C.c_void_p(short.data_ptr()),
                                 need - 1, C.byref(total), stream)
        assert st == 7 and total.value == need
    d_adj2 = torch.full((max(need, 1),), -7, dtype=torch.int32, device=dev)
    Q._check(L.qc_twohop_noalloc(int(g.n), C.c_void_p(d_off.data_ptr()), C.c_void_p(d_adj.data_ptr()),
                                 C.c_void_p(d_off2.data_ptr()), C.c_void_p(d_adj2.data_ptr()),
                                 int(d_adj2.numel()), C.byref(total), stream))
    torch.cuda.synchronize(dev)
    return d_off2.cpu().numpy(), d_adj2[:need].cpu().numpy()


@pytest.mark.gpu
def test_noalloc_twohop_matches_allocating_builder_twice_in_a_row():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cases = [
        graphs.erdos_renyi_planted(1000, 0.02, 5, 30, 0.95, seed=1),
        graphs.chung_lu_planted(n=3000, beta=2.1, mean_degree=20, n_groups=20,
                                size_range=(15, 40), density_range=(0.85, 1.0), seed=4),
    ]
    for g in cases:  # two calls in a row on the shared device array
        want_off2, want_adj2 = _allocating_twohop(g)
        got_off2, got_adj2 = _noalloc_twohop(g, torch)
        assert np.array_equal(got_off2, want_off2)
        assert np.array_equal(got_adj2, want_adj2)
        ref_off2, ref_adj2 = oracle.twohop(g.n, g.off, g.adj)
        assert np.array_equal(got_off2, ref_off2)
        assert np.array_equal(got_adj2, ref_adj2)


def _csr(n, rows):
    off = np.zeros(n + 1, np.int64)
    for v, r in enumerate(rows):
        off[v + 1] = off[v] + len(r)
    adj = np.array([w for r in rows for w in r], np.int32)
    return graphs.Graph(n=n, off=off, adj=adj)


@pytest.mark.gpu
def test_noalloc_twohop_edge_cases():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    # no vertices: one offset, no entries
    g0 = graphs.Graph(n=0, off=np.zeros(1, np.int64), adj=np.zeros(0, np.int32))
    off2, adj2 = _noalloc_twohop(g0, torch)
    assert off2.tolist() == [0] and len(adj2) == 0
    # isolated vertices only
    g1 = _csr(5, [[], [], [], [], []])
    off2, adj2 = _noalloc_twohop(g1, torch)
    assert off2.tolist() == [0] * 6 and len(adj2) == 0
    # a self loop keeps v in its own two-hop row (adjToSer.cpp:115-156); the
    # allocating builder refuses self loops, so the oracle is the check
    g2 = _csr(5, [[0, 1], [0, 2], [1, 3], [2], []])
    off2, adj2 = _noalloc_twohop(g2, torch)
    ref_off2, ref_adj2 = oracle.twohop(g2.n, g2.off, g2.adj)
    assert np.array_equal(off2, ref_off2) and np.array_equal(adj2, ref_adj2)
    assert adj2[off2[0]:off2[1]].tolist() == [0, 1, 2]


@pytest.mark.gpu
def test_noalloc_twohop_at_its_largest_vertex_count():
    """A ring of qc_twohop_noalloc_max_vertices() vertices: the per-warp working
    memory is at its largest and the fewest warps run."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    n = int(Q.lib().qc_twohop_noalloc_max_vertices())
    v = np.arange(n, dtype=np.int64)
    g = graphs.from_edges(n, v, (v + 1) % n, with_twohop=False)
    got_off2, got_adj2 = _noalloc_twohop(g, torch)
    want_off2, want_adj2 = _allocating_twohop(g)
    assert np.array_equal(got_off2, want_off2)
    assert np.array_equal(got_adj2, want_adj2)
    # ring: N2(v) = {v-2, v-1, v+1, v+2}
    assert got_off2[-1] == 4 * n
    rows = np.sort(np.stack([(v - 2) % n, (v - 1) % n, (v + 1) % n, (v + 2) % n], 1), 1)
    assert np.array_equal(got_adj2.reshape(n, 4), rows.astype(np.int32))


@pytest.mark.gpu
def test_noalloc_twohop_refuses_malformed_device_csr():
    """Ids just past n still land inside the shared array, so an unchecked
    kernel could not fault on them either; the call must refuse them."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = Q.lib()
    dev = torch.device("cuda", 0)
    n = 64
    good = graphs.erdos_renyi_planted(n, 0.1, 1, 8, 1.0, seed=3)

    def call(off, adj, adj_null=False):
        d_off = torch.as_tensor(np.asarray(off, np.int64), device=dev)
        d_adj = torch.as_tensor(np.asarray(adj, np.int32), device=dev)
        d_off2 = torch.full((n + 1,), -7, dtype=torch.int64, device=dev)
        d_adj2 = torch.full((1 << 14,), -7, dtype=torch.int32, device=dev)
        total = C.c_int64(-1)
        st = L.qc_twohop_noalloc(n, C.c_void_p(d_off.data_ptr()),
                                 None if adj_null else C.c_void_p(d_adj.data_ptr()),
                                 C.c_void_p(d_off2.data_ptr()), C.c_void_p(d_adj2.data_ptr()),
                                 int(d_adj2.numel()), C.byref(total), None)
        torch.cuda.synchronize(dev)
        return st, d_adj2.cpu().numpy(), L.qc_last_error()

    for bad in (n, n + 5, -1):
        adj = np.array(good.adj, np.int32)
        adj[len(adj) // 2] = bad
        st, adj2, msg = call(good.off, adj)
        assert st == QC_ERR_FORMAT and b"outside [0, n)" in msg
        assert (adj2 == -7).all()  # no rows written
    off = np.array(good.off, np.int64)
    off[10], off[11] = off[11], off[10] - 1  # a decreasing step
    st, adj2, msg = call(off, good.adj)
    assert st == QC_ERR_FORMAT and b"offsets" in msg and (adj2 == -7).all()
    st, adj2, msg = call(good.off, good.adj, adj_null=True)
    assert st == QC_ERR_FORMAT and b"NULL" in msg and (adj2 == -7).all()
    # the shared array recovers: the next well-formed call is exact
    got_off2, got_adj2 = _noalloc_twohop(good, torch)
    ref_off2, ref_adj2 = oracle.twohop(good.n, good.off, good.adj)
    assert np.array_equal(got_off2, ref_off2) and np.array_equal(got_adj2, ref_adj2)


@pytest.mark.gpu
def test_noalloc_twohop_rejects_graphs_above_its_limit():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = Q.lib()
    limit = int(L.qc_twohop_noalloc_max_vertices())
    assert limit >= 1_000_000
    dev = torch.device("cuda", 0)
    d_off2 = torch.zeros(1, dtype=torch.int64, device=dev)
    total = C.c_int64(-1)
    # rejected before any kernel runs, so the buffers need not be that large
    st = L.qc_twohop_noalloc(limit + 32, C.c_void_p(d_off2.data_ptr()), C.c_void_p(d_off2.data_ptr()),
                             C.c_void_p(d_off2.data_ptr()), None, 0, C.byref(total), None)
    assert st == 9
    assert b"at most" in L.qc_last_error()
