"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference, on a B200."""
import os
import tempfile

import numpy as np
import pytest

import cuqc_b200 as Q
from conftest import GOLDEN, golden_cases, load_case, parse_result
from cuqc_b200 import graphs
from oracle import oracle

pytestmark = pytest.mark.gpu
CASES = golden_cases()


def canon(flat):
    return sorted(tuple(sorted(s)) for s in oracle.unpack(flat))


@pytest.fixture(scope="module")
def ctx():
    c = Q.Context(device=0, keep_emitted=True)
    yield c
    c.close()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_golden_case(ctx, case):
    g, path, gamma, ms, _ = load_case(case)
    res = ctx.mine(g, float(gamma), ms)
    want_flat, st = oracle.mine(g, float(gamma), ms, "clean")
    # the device emits exactly the oracle's multiset of quasi-cliques
    assert canon(res.emitted) == canon(want_flat)
    assert res.stats["tasks"] == st["tasks"]
    assert res.stats["branches"] == st["branches"]
    # the byte-model counters behind the bench's roofline numerator, counted by
    # the kernel, equal the oracle's count of the same tree
    for k in ("children", "parent_vertices", "p_rows", "child_vertices"):
        assert res.stats[k] == st[k], k
    assert res.sets == oracle.maximal(want_flat)
    refbin = os.path.join(GOLDEN, case["name"] + ".refbin.result")
    if os.path.exists(refbin):
        assert res.text() == open(refbin).read()


@pytest.mark.parametrize("seed", range(300, 316))
def test_random_graphs(ctx, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(20, 120))
    p = float(rng.uniform(0.05, 0.35))
    g = graphs.random_small(n, p, seed, planted=int(rng.integers(0, 5)),
                            size=int(rng.integers(6, 18)), density=float(rng.uniform(0.85, 1)))
    gamma = [0.7, 0.75, 0.8, 0.85, 0.9, 0.95, 1.0][seed % 7]
    ms = int(rng.integers(4, 10))
    want_flat, st = oracle.mine(g, gamma, ms, "clean")
    res = ctx.mine(g, gamma, ms)
    assert canon(res.emitted) == canon(want_flat)
    assert res.sets == oracle.maximal(want_flat)
    # level 0 (on the device up to 65,536 vertices) gives the oracle's root
    assert res.stats["root_size"] == len(oracle.root(g, gamma, ms)[0])
    assert res.stats["tasks"] == st["tasks"] and res.stats["branches"] == st["branches"]
    for k in ("children", "parent_vertices", "p_rows", "child_vertices"):
        assert res.stats[k] == st[k], k


@pytest.mark.parametrize("n", [70000, 200000])
def test_level0_grid_above_the_block_limit(ctx, n):
    # above 65,536 vertices level 0 runs over the whole grid (one cooperative
    # launch, level0_grid.cuh); sparse background, planted groups survive
    rng = np.random.default_rng(21)
    src, dst = rng.integers(0, n, 3 * n), rng.integers(0, n, 3 * n)  # mean degree ~6
    groups = [rng.choice(n, 15, replace=False) for _ in range(2 if n < 100000 else 6)]
    for grp in groups:
        iu, ju = np.triu_indices(15, 1)
        keep = rng.random(len(iu)) < 0.95
        src = np.concatenate([src, grp[iu[keep]]])
        dst = np.concatenate([dst, grp[ju[keep]]])
    ok = src != dst
    dg = Q.DeviceGraph.from_graph(graphs.from_edges(n, src[ok], dst[ok], with_twohop=False))
    g = dg.to_graph()  # with the two-hop lists built on the device
    want_flat, st = oracle.mine(g, 0.95, 12, "clean")
    res = ctx.mine(dg, 0.95, 12)
    assert res.stats["root_size"] == len(oracle.root(g, 0.95, 12)[0])
    assert res.stats["tasks"] == st["tasks"] and res.stats["branches"] == st["branches"]
    assert res.sets == oracle.maximal(want_flat)


def test_small_arena_grows_and_stays_exact():
    g = graphs.erdos_renyi_planted(300, 0.03, 3, 16, 0.95, seed=11)
    with Q.Context(device=0, arena_bytes=1 << 16, stack_slots=64, result_ints=256) as c:
        res = c.mine(g, 0.8, 10)
    assert res.sets == oracle.solve(g, 0.8, 10)[0]


@pytest.mark.parametrize("wpb", [8, 2])
def test_children_above_the_counting_rank_limit(ctx, wpb):
    # one group of 300 at density 0.88 with min_size 270: every child keeps at
    # least 270 vertices, so each is ordered by the bitonic sort of keys padded
    # to a power of two (children of up to 256 vertices take counting ranks)
    # and worked on with its workspace in global memory (8 warps stage tasks of
    # up to 160 vertices, 2 warps up to 256)
    g = graphs.erdos_renyi_planted(600, 0.02, 1, 300, 0.88, seed=1)
    want_flat, st = oracle.mine(g, 0.9, 270, "clean")
    assert st["children"] > 0 and st["child_vertices"] >= 270 * st["children"]
    if wpb == 8:
        res = ctx.mine(g, 0.9, 270)
    else:
        with Q.Context(device=0, warps_per_block=wpb, keep_emitted=True) as c:
            res = c.mine(g, 0.9, 270)
    assert canon(res.emitted) == canon(want_flat)
    assert res.sets == oracle.maximal(want_flat)
    for k in ("tasks", "branches", "children", "parent_vertices", "p_rows", "child_vertices"):
        assert res.stats[k] == st[k], k


def test_root_larger_than_the_arena_grows_it():
    # the root's record is set up on the device: a block larger than the arena
    # stops the launch at once and the host grows the arena and runs again
    g = graphs.erdos_renyi_planted(300, 0.03, 3, 16, 0.95, seed=11)
    with Q.Context(device=0, arena_bytes=1 << 10) as c:
        res = c.mine(g, 0.8, 10)
    assert res.sets == oracle.solve(g, 0.8, 10)[0]
    assert res.stats["root_size"] == len(oracle.root(g, 0.8, 10)[0])


def test_root_emptied_by_peeling(ctx):
    # a star: the centre passes level 0's first test (degree and two-hop size)
    # but keeps no neighbour, so the root is empty only after peeling, which
    # the device learns after the host has set up the launch
    n = 21
    g = graphs.from_edges(n, [0] * (n - 1), list(range(1, n)))
    res = ctx.mine(g, 1.0, 3)
    assert res.sets == [] and res.stats["root_size"] == 0 and res.stats["tasks"] == 0


def test_repeated_calls_reuse_context(ctx):
    g = graphs.erdos_renyi_planted(300, 0.03, 3, 16, 0.95, seed=11)
    a = ctx.mine(g, 0.8, 10).sets
    b = ctx.mine(g, 0.8, 10).sets
    assert a == b == oracle.solve(g, 0.8, 10)[0]


def test_empty_result(ctx):
    case = [c for c in CASES if c["refcpu_maximal"] == 0][0]
    g, path, gamma, ms, _ = load_case(case)
    res = ctx.mine(g, float(gamma), ms)
    assert res.sets == []


@pytest.mark.parametrize("seed", range(4))
def test_device_twohop_matches(seed):
    g = graphs.random_small(200, 0.04 + 0.02 * seed, seed, planted=2, size=12)
    base = graphs.Graph(n=g.n, off=g.off, adj=g.adj)
    dg = Q.DeviceGraph.from_graph(base)
    back = dg.to_graph()
    assert np.array_equal(back.off2, g.off2) and np.array_equal(back.adj2, g.adj2)


def test_cli_matches_reference_output():
    """Config 1 through the drop-in CLI.  The reference binary faulted on this
    graph, so the result file is compared with the reference's own CPU path
    (tests/golden/er1000_planted.refcpu.result) and with the oracle."""
    case = [c for c in CASES if c["name"] == "er1000_planted"][0]
    g, path, gamma, ms, _ = load_case(case)
    d = tempfile.mkdtemp()
    out = os.path.join(d, "out.txt")
    rc, stdout = Q.cli(path, gamma, ms, out, 0, cwd=d)
    assert rc == 0, stdout
    assert stdout.splitlines()[0] == ">:PRE-PROCESSING"
    assert ">:NUMBER OF MAXIMAL CLIQUES: 1365" in stdout
    assert stdout.splitlines()[-1] == ">:PROGRAM END"
    for key in ("LOADING TIME", "ENUMERATION TIME", "EXPANSION KERNEL TIME",
                "REMOVE NON-MAX TIME", "TOTAL TIME"):
        assert ("--->:%s: " % key) in stdout
    got = open(out).read()
    assert got == open(os.path.join(GOLDEN, case["name"] + ".refcpu.result")).read()
    assert got == oracle.result_text(oracle.solve(g, float(gamma), ms, "clean")[0])


def _batch_specs(seed0, count):
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed0 + i)
        n = int(rng.integers(12, 90))
        g = graphs.random_small(n, float(rng.uniform(0.08, 0.4)), seed0 + i,
                                planted=int(rng.integers(0, 4)), size=int(rng.integers(5, 15)),
                                density=float(rng.uniform(0.85, 1.0)))
        out.append((g, [0.7, 0.8, 0.85, 0.9, 0.95, 1.0][i % 6], int(rng.integers(3, 9))))
    return out


def test_batch_matches_per_instance_oracle(ctx):
    specs = _batch_specs(500, 24)
    res = ctx.mine_batch([s[0] for s in specs], [s[1] for s in specs], [s[2] for s in specs])
    assert len(res) == len(specs)
    for (g, gm, ms), r in zip(specs, res):
        assert r.sets == oracle.solve(g, gm, ms)[0]


def test_batch_equals_plain_calls(ctx):
    specs = _batch_specs(700, 8)
    batch = ctx.mine_batch([s[0] for s in specs], [s[1] for s in specs], [s[2] for s in specs])
    for (g, gm, ms), r in zip(specs, batch):
        assert r.sets == ctx.mine(g, gm, ms).sets


def test_batch_with_golden_cases(ctx):
    loaded = [load_case(c) for c in CASES]
    res = ctx.mine_batch([x[0] for x in loaded], [float(x[2]) for x in loaded],
                         [x[3] for x in loaded])
    for case, (g, path, gamma, ms, _), r in zip(CASES, loaded, res):
        refbin = os.path.join(GOLDEN, case["name"] + ".refbin.result")
        want = open(refbin).read() if os.path.exists(refbin) else oracle.result_text(
            oracle.solve(g, float(gamma), ms)[0])
        assert r.text() == want, case["name"]


def _digest(sets):
    import hashlib
    text = "".join("%d %s \n" % (len(s), " ".join(map(str, s))) for s in sets)
    return hashlib.sha1(text.encode()).hexdigest()


def test_batched_workload_matches_oracle_digests(ctx):
    """The first 64 instances of the batched workload, in one launch, against
    the oracle's result digests recorded in the manifest."""
    import json
    man = json.load(open(os.path.join(GOLDEN, "cfg3_batch.json")))
    rows = man["instances"][:64]
    inst = [graphs.batch_instance(r["i"]) for r in rows]
    res = ctx.mine_batch([x[0] for x in inst], [float(x[1]) for x in inst], [x[2] for x in inst])
    for r, x in zip(rows, res):
        assert len(x.sets) == r["maximal"], r["i"]
        assert _digest(x.sets) == r["digest"], r["i"]


@pytest.mark.parametrize("wpb,bps,split", [(1, 1, 1), (2, 2, 3), (4, 2, 2), (8, 1, 1)])
def test_launch_shapes_agree(wpb, bps, split):
    """Every grid shape and work split gives the same sets and the same tree."""
    g = graphs.erdos_renyi_planted(1000, 0.02, 5, 30, 0.95, seed=1)
    with Q.Context(device=0, warps_per_block=wpb, blocks_per_sm=bps, split=split) as c:
        res = c.mine(g, 0.9, 20)
    assert len(res.sets) == 1365
    assert res.stats["tasks"] == 36601 and res.stats["branches"] == 68682
    assert res.sets == oracle.maximal(oracle.mine(g, 0.9, 20, "clean")[0])


def test_time_limit_stops_cleanly_and_context_stays_usable():
    """A run over its time limit stops with QC_ERR_ITER_LIMIT (every wait in
    the kernel is bounded); the same context then mines normally."""
    g, gm, ms = graphs.batch_instance(3)   # tens of millions of tasks
    small = graphs.erdos_renyi_planted(300, 0.03, 3, 16, 0.95, seed=11)
    with Q.Context(device=0, time_limit_ms=300) as c:
        with pytest.raises(Q.QCError) as e:
            c.mine(g, float(gm), ms)
        assert e.value.status == 8
        assert c.mine(small, 0.8, 10).sets == oracle.solve(small, 0.8, 10)[0]


def test_tune_picks_a_shape_and_keeps_results():
    g = graphs.erdos_renyi_planted(300, 0.03, 3, 16, 0.95, seed=11)
    want = oracle.solve(g, 0.8, 10)[0]
    with Q.Context(device=0) as c:
        best = c.tune(g, 0.8, 10, repeats=1)
        assert best["warps_per_block"] in (4, 8) and best["blocks_per_sm"] in (1, 2)
        assert best["split"] in (1, 2, 4) and best["stage_max"] in (0, 64, -1)
        assert best["shared_order"] in (0, 1, 2)
        assert c.mine(g, 0.8, 10).sets == want


def test_tune_batch_picks_settings_and_keeps_results():
    specs = _batch_specs(900, 12)
    gs = [x[0] for x in specs]
    gms = [x[1] for x in specs]
    mss = [x[2] for x in specs]
    with Q.Context(device=0) as c:
        best = c.tune_batch(gs, gms, mss, repeats=1)
        assert best["warps_per_block"] in (4, 8) and best["split"] in (1, 2, 4)
        res = c.mine_batch(gs, gms, mss)
    for (g, gm, ms), r in zip(specs, res):
        assert r.sets == oracle.solve(g, gm, ms)[0]


def test_freed_graph_buffers_are_reused_correctly():
    """A context keeps uploaded graphs on the device; once a graph is freed,
    the next new graph reuses its device buffers.  Results stay exact across
    a sequence of upload / free / upload of graphs of different sizes."""
    gs = [graphs.erdos_renyi_planted(300, 0.03, 3, 16, 0.95, seed=11),
          graphs.random_small(90, 0.2, 5, planted=2, size=12, density=0.95),
          graphs.erdos_renyi_planted(500, 0.025, 4, 18, 0.95, seed=12)]
    want = [oracle.solve(g, 0.8, 8)[0] for g in gs]
    with Q.Context(device=0) as c:
        for rnd in range(3):
            for g, w in zip(gs, want):
                dg = Q.DeviceGraph.from_graph(g)
                assert c.mine(dg, 0.8, 8).sets == w
                dg.close()
