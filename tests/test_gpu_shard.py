"""Level 0 alone (qc_root) and one graph mined as shards of the root's
branches (qc_mine_shard), merged with qc_maximal_sets, against the oracle."""
import numpy as np
import pytest

import cuqc_b200 as Q
from cuqc_b200 import graphs
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Q.Context(device=0, keep_emitted=True)
    yield c
    c.close()


def canon(flat):
    return sorted(tuple(sorted(s)) for s in oracle.unpack(flat))


@pytest.mark.parametrize("nshards", [2, 3, 5])
@pytest.mark.parametrize("case", [(1000, 0.02, 5, 30, 0.95, 1, 0.9, 20),
                                  (300, 0.03, 3, 16, 0.95, 11, 0.8, 10)])
def test_shards_merge_to_the_whole_search(ctx, case, nshards):
    n, p, groups, size, dens, seed, gamma, ms = case
    g = graphs.erdos_renyi_planted(n, p, groups, size, dens, seed=seed)
    whole = ctx.mine(g, gamma, ms)
    parts = [ctx.mine_shard(g, gamma, ms, s, nshards) for s in range(nshards)]
    # the shards' emitted sets are the whole search's, each once
    emitted = np.concatenate([r.emitted for r in parts])
    assert canon(emitted) == canon(whole.emitted)
    assert sum(r.stats["branches"] for r in parts) == whole.stats["branches"]
    merged = ctx.maximal_sets(np.concatenate([r.flat for r in parts]), g.n)
    assert merged.sets == whole.sets == oracle.solve(g, gamma, ms)[0]


@pytest.mark.parametrize("n", [1000, 200000])
def test_root_alone_matches_the_oracle(ctx, n):
    """The root (ids in branching order, covered count) from the one-block
    device level 0 (n = 1,000) and from the grid-wide one (n = 200,000)."""
    rng = np.random.default_rng(5)
    src, dst = rng.integers(0, n, 3 * n), rng.integers(0, n, 3 * n)
    for _ in range(4):
        grp = rng.choice(n, 20, replace=False)
        iu, ju = np.triu_indices(20, 1)
        keep = rng.random(len(iu)) < 0.95
        src = np.concatenate([src, grp[iu[keep]]])
        dst = np.concatenate([dst, grp[ju[keep]]])
    ok = src != dst
    dg = Q.DeviceGraph.from_graph(graphs.from_edges(n, src[ok], dst[ok], with_twohop=False))
    g = dg.to_graph()
    ids, cov = ctx.root(dg, 0.9, 15)
    want_ids, want_lab, _ = oracle.root(g, 0.9, 15)
    assert len(want_ids) > 0
    assert ids.tolist() == want_ids.tolist()
    assert cov == int((want_lab == 2).sum())
    res = ctx.mine(dg, 0.9, 15)
    assert res.stats["level0_on_device"] == 1
    assert res.stats["root_size"] == len(want_ids)


def test_binary_graph_file_without_twohop_lists(tmp_path):
    """A binary CSR file holding only the 1-hop lists: the library builds the
    two-hop lists on the GPU (equal to the oracle's), and the drop-in CLI gives
    the same result file for it as for the serialized text of the graph."""
    g = graphs.erdos_renyi_planted(300, 0.03, 3, 16, 0.95, seed=11)
    binp, txt = str(tmp_path / "g.bin"), str(tmp_path / "g.txt")
    graphs.write_binary(g, binp, twohop=False)
    graphs.write_serialized(g, txt)
    back = Q.DeviceGraph.read(binp).to_graph()
    off2, adj2 = oracle.twohop(g.n, g.off, g.adj)
    assert np.array_equal(back.off2, off2) and np.array_equal(back.adj2, adj2)
    outs = []
    for path in (binp, txt):
        out = str(tmp_path / (path.rsplit("/", 1)[1] + ".result"))
        rc, text = Q.cli(path, "0.8", 10, out, 0, cwd=str(tmp_path))
        assert rc == 0, text
        outs.append(open(out).read())
    assert outs[0] == outs[1] == oracle.result_text(oracle.solve(g, 0.8, 10)[0])
