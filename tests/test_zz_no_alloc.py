"""qc_twohop_noalloc: the two-hop builder for callers that cannot allocate
device memory (their memory is owned by their own pool or fixed plan, or they
must not allocate while serving).  It is checked through the C ABI against the
allocating builder behind qc_graph_from_csr, on two calls in a row, with the
caller's inputs and outputs in device buffers.

This file is collected last on purpose: the no-allocation entry point shares
one device array across calls, and the test must hold both in a fresh process
and after every other test has run."""
import ctypes as C

import numpy as np
import pytest

import cuqc_b200 as Q
from cuqc_b200 import graphs


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
    d_adj = torch.as_tensor(np.asarray(g.adj, np.int32), device=dev)
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
