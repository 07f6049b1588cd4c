"""Graphs in the reference's serialized format, and seeded synthetic workloads.

The serialized format is the one cuQC reads (Mike12041204/cuQC main.cu:82-131)
and adjToSer writes (adjToSer.cpp:159-204): seven whitespace-separated
sections

    n
    number of directed 1-hop entries (2|E|)
    number of 2-hop entries
    1-hop neighbours (rows sorted ascending)
    1-hop offsets (n+1, uint64)
    2-hop neighbours (rows sorted ascending)
    2-hop offsets (n+1, uint64)

where the 2-hop row of v is sorted(N(v) u N(N(v)) minus {v}) (adjToSer.cpp:115-156).

The generators stand in for the datasets the reference was measured on (none
ships with it): Erdos-Renyi and Chung-Lu power-law graphs with planted dense
groups, drawn from a numpy PCG64 stream with a fixed seed per workload.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Graph:
    n: int
    off: np.ndarray  # int64[n+1]
    adj: np.ndarray  # int32[2|E|], rows sorted
    off2: np.ndarray = field(default=None)  # int64[n+1]
    adj2: np.ndarray = field(default=None)  # int32, rows sorted

    @property
    def m(self) -> int:
        return int(self.off[-1])

    @property
    def m2(self) -> int:
        return int(self.off2[-1]) if self.off2 is not None else 0

    def degree(self) -> np.ndarray:
        return np.diff(self.off)


# ---------------------------------------------------------------------------
# construction
# ---------------------------------------------------------------------------

def from_edges(n: int, src, dst, with_twohop: bool = True) -> Graph:
    """Symmetric simple graph (self loops and duplicates dropped), CSR with
    sorted rows, plus its 2-hop lists."""
    src = np.asarray(src, np.int64)
    dst = np.asarray(dst, np.int64)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    a = np.concatenate([src, dst])
    b = np.concatenate([dst, src])
    key = np.unique(a * n + b)
    a, b = key // n, key % n
    off = np.zeros(n + 1, np.int64)
    np.add.at(off, a + 1, 1)
    off = np.cumsum(off)
    g = Graph(n=n, off=off, adj=b.astype(np.int32))
    if with_twohop:
        g.off2, g.adj2 = twohop_lists(g)
    return g


def twohop_lists(g: Graph):
    """2-hop rows sorted(N(v) u N(N(v)) minus {v}) via a sparse product."""
    import scipy.sparse as sp

    n = g.n
    if n == 0:
        return np.zeros(1, np.int64), np.zeros(0, np.int32)
    A = sp.csr_matrix((np.ones(g.m, np.int32), g.adj.astype(np.int64), g.off), shape=(n, n))
    A2 = (A @ A) + A
    A2 = A2.tocsr()
    A2.setdiag(0)
    A2.eliminate_zeros()
    A2.sort_indices()
    return A2.indptr.astype(np.int64), A2.indices.astype(np.int32)


# ---------------------------------------------------------------------------
# serialized format I/O
# ---------------------------------------------------------------------------

def _join(a) -> str:
    return " ".join(np.asarray(a).astype(str).tolist())


def write_serialized(g: Graph, path: str) -> None:
    with open(path, "w") as f:
        f.write("%d\n%d\n%d\n" % (g.n, g.m, g.m2))
        f.write(_join(g.adj) + "\n")
        f.write(_join(g.off) + "\n")
        f.write(_join(g.adj2) + "\n")
        f.write(_join(g.off2) + "\n")


def read_serialized(path: str) -> Graph:
    with open(path) as f:
        tok = np.array(f.read().split(), dtype=np.int64)
    n, m, m2 = int(tok[0]), int(tok[1]), int(tok[2])
    p = 3
    adj = tok[p:p + m].astype(np.int32); p += m
    off = tok[p:p + n + 1].astype(np.int64); p += n + 1
    adj2 = tok[p:p + m2].astype(np.int32); p += m2
    off2 = tok[p:p + n + 1].astype(np.int64)
    return Graph(n=n, off=off, adj=adj, off2=off2, adj2=adj2)


def write_binary(g: Graph, path: str, twohop: bool = True) -> None:
    """The binary CSR file the library reads (qc_graph_read_binary): magic
    "QCSRBIN1", int64 n, nnz, nnz2 (-1 without two-hop lists), int64 offsets,
    int32 rows padded to 8 bytes, then the two-hop offsets and rows."""
    off = np.asarray(g.off, "<i8")
    adj = np.asarray(g.adj, "<i4")
    two = twohop and g.off2 is not None
    with open(path, "wb") as f:
        f.write(b"QCSRBIN1")
        f.write(np.asarray([g.n, len(adj), len(g.adj2) if two else -1], "<i8").tobytes())
        f.write(off.tobytes())
        f.write(adj.tobytes())
        f.write(b"\0" * ((8 - (4 * len(adj)) % 8) % 8))
        if two:
            f.write(np.asarray(g.off2, "<i8").tobytes())
            f.write(np.asarray(g.adj2, "<i4").tobytes())


def write_adjlist(g: Graph, path: str) -> None:
    """Adjacency-list text (one line per vertex), the input of adjToSer."""
    with open(path, "w") as f:
        lines = [_join(g.adj[g.off[v]:g.off[v + 1]]) for v in range(g.n)]
        f.write("\n".join(lines))


# ---------------------------------------------------------------------------
# seeded generators
# ---------------------------------------------------------------------------

def _upper_bernoulli(rng, n, prob_row, block=512):
    """Edges i<j drawn independently with probability prob_row(i0, i1) -> P[i, j]."""
    src, dst = [], []
    for a in range(0, n, block):
        b = min(n, a + block)
        P = prob_row(a, b)
        R = rng.random(P.shape)
        ii, jj = np.nonzero(R < P)
        ii = ii + a
        keep = jj > ii
        src.append(ii[keep])
        dst.append(jj[keep])
    if not src:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    return np.concatenate(src), np.concatenate(dst)


def _plant(rng, members, density):
    s = len(members)
    iu, ju = np.triu_indices(s, 1)
    keep = rng.random(len(iu)) < density
    return members[iu[keep]], members[ju[keep]]


def erdos_renyi_planted(n, p, groups, group_size, density, seed):
    """G(n, p) plus `groups` disjoint planted groups of `group_size` vertices
    (taken from one seeded permutation) at intra-group edge density `density`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    src, dst = _upper_bernoulli(rng, n, lambda a, b: np.full((b - a, n), p))
    perm = rng.permutation(n)
    ss, dd = [src], [dst]
    for k in range(groups):
        s, d = _plant(rng, perm[k * group_size:(k + 1) * group_size], density)
        ss.append(s); dd.append(d)
    return from_edges(n, np.concatenate(ss), np.concatenate(dd))


def chung_lu_weights(n, beta, mean_degree):
    """Expected degrees w_i proportional to (i + i0)^(-1/(beta-1)), scaled to the
    requested mean degree; i0 is chosen so that the largest expected degree is
    the structural cutoff sqrt(n * mean_degree)."""
    e = 1.0 / (beta - 1.0)
    idx = np.arange(n, dtype=np.float64)
    cutoff = math.sqrt(n * mean_degree)

    def wmax_for(i0):
        w = (idx + i0) ** (-e)
        return w[0] / w.mean() * mean_degree

    lo, hi = 1e-9, float(n)
    if wmax_for(lo) <= cutoff:
        i0 = lo
    else:
        for _ in range(80):
            mid = 0.5 * (lo + hi)
            if wmax_for(mid) > cutoff:
                lo = mid
            else:
                hi = mid
        i0 = hi
    w = (idx + i0) ** (-e)
    return w / w.mean() * mean_degree


def chung_lu_planted(n, beta, mean_degree, n_groups, size_range, density_range, seed):
    """Chung-Lu graph (edge probability min(1, w_i w_j / sum w)) plus
    independently sampled planted groups (overlap allowed) with sizes uniform
    in size_range (inclusive) and densities uniform in density_range."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = chung_lu_weights(n, beta, mean_degree)
    W = w.sum()
    src, dst = _upper_bernoulli(rng, n, lambda a, b: np.minimum(1.0, np.outer(w[a:b], w) / W))
    ss, dd = [src], [dst]
    for _ in range(n_groups):
        s = int(rng.integers(size_range[0], size_range[1] + 1))
        d = float(rng.uniform(density_range[0], density_range[1]))
        members = rng.choice(n, size=min(s, n), replace=False)
        a, b = _plant(rng, members, d)
        ss.append(a); dd.append(b)
    return from_edges(n, np.concatenate(ss), np.concatenate(dd))


def chung_lu_sparse_planted(n, beta, mean_degree, n_groups, size_range, density_range, seed,
                            with_twohop=False):
    """Chung-Lu graph for large n in O(n + m): n * mean_degree / 2 edges whose
    two endpoints are drawn independently in proportion to the expected
    degrees w (chung_lu_weights), self loops dropped and repeats merged -- the
    edge-sampling form of the expected-degree model (each pair appears with
    probability about 1 - exp(-w_i w_j / sum w), close to min(1, w_i w_j /
    sum w) for all but the heaviest pairs).  Planted groups as in
    chung_lu_planted.  The two-hop lists are left to the GPU unless asked."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = chung_lu_weights(n, beta, mean_degree)
    m = int(round(n * mean_degree / 2.0))
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    src = np.searchsorted(cdf, rng.random(m), side="right").clip(0, n - 1)
    dst = np.searchsorted(cdf, rng.random(m), side="right").clip(0, n - 1)
    ss, dd = [src], [dst]
    for _ in range(n_groups):
        s = int(rng.integers(size_range[0], size_range[1] + 1))
        d = float(rng.uniform(density_range[0], density_range[1]))
        members = rng.choice(n, size=min(s, n), replace=False)
        a, b = _plant(rng, members, d)
        ss.append(a); dd.append(b)
    return from_edges(n, np.concatenate(ss), np.concatenate(dd), with_twohop=with_twohop)


def random_small(n, p, seed, planted=0, size=0, density=1.0):
    """Small random graph for parity sweeps."""
    rng = np.random.Generator(np.random.PCG64(seed))
    src, dst = _upper_bernoulli(rng, n, lambda a, b: np.full((b - a, n), p))
    ss, dd = [src], [dst]
    for _ in range(planted):
        members = rng.choice(n, size=min(size, n), replace=False)
        a, b = _plant(rng, members, density)
        ss.append(a); dd.append(b)
    return from_edges(n, np.concatenate(ss), np.concatenate(dd))


# ---------------------------------------------------------------------------
# multi-instance workload: independent instances of uneven size
# ---------------------------------------------------------------------------

GAMMAS_CFG3 = ("0.6", "0.7", "0.8", "0.9", "0.95")


def batch_instance(i, base_seed=3000):
    """Instance i of the batched workload: n log-uniform in [200, 5000],
    Chung-Lu exponent 2.1 with mean degree uniform in [10, 50], 1-20 planted
    groups of size 10-40 at density 0.8-1.0, gamma drawn from
    {0.6, 0.7, 0.8, 0.9, 0.95} and min_size uniform in 5..30.
    Returns (graph, gamma string, min_size)."""
    rng = np.random.Generator(np.random.PCG64(base_seed + i))
    n = int(math.floor(math.exp(rng.uniform(math.log(200), math.log(5000)))))
    d = float(rng.uniform(10, 50))
    k = int(rng.integers(1, 21))
    gamma = GAMMAS_CFG3[int(rng.integers(0, len(GAMMAS_CFG3)))]
    ms = int(rng.integers(5, 31))
    g = chung_lu_planted(n, 2.1, d, k, (10, 40), (0.8, 1.0), seed=base_seed + 100000 + i)
    return g, gamma, ms
