"""The product's expansion-kernel source run on the CPU under a 32-thread warp
emulator (tests/emu) emits exactly the oracle's multiset of quasi-cliques."""
import numpy as np
import pytest

from cuqc_b200 import graphs
from oracle import oracle
import emu


def canon(flat):
    return sorted(tuple(sorted(s)) for s in oracle.unpack(flat))


CASES = [  # (n, p, seed, planted, size, gamma, min_size, warps, split); n > 32 uses both paths
    (20, 0.35, 1, 1, 7, 0.7, 4, 2, 2),
    (24, 0.3, 2, 2, 6, 0.8, 4, 1, 1000),
    (28, 0.25, 3, 1, 9, 0.9, 5, 3, 1),
    (18, 0.5, 4, 0, 0, 0.6, 4, 2, 3),
    (30, 0.2, 5, 2, 8, 1.0, 4, 2, 2),
    (26, 0.3, 6, 1, 10, 0.75, 6, 2, 4),
    (44, 0.18, 7, 2, 12, 0.8, 6, 2, 3),
    (40, 0.22, 8, 1, 14, 0.9, 7, 2, 4),
    # roots of 35-47 vertices: branches of tasks over 32 vertices that shrink
    # to 32 or fewer members and candidates finish on the register path
    (60, 0.12, 21, 2, 20, 0.9, 10, 3, 1),
    (90, 0.08, 24, 3, 16, 0.9, 8, 2, 2),
    (64, 0.2, 25, 1, 24, 0.95, 12, 2, 1),
]


@pytest.mark.parametrize("small_path,fifo", [(1, 0), (0, 0), (1, 1)])
@pytest.mark.parametrize("case", CASES)
def test_emulated_kernel_matches_oracle(case, small_path, fifo):
    """Both task paths, and the shared stack taken newest first or oldest first."""
    n, p, seed, planted, size, gamma, ms, warps, split = case
    g = graphs.random_small(n, p, seed, planted=planted, size=size, density=0.95)
    want, st = oracle.mine(g, gamma, ms, "clean")
    assert st["tasks"] < 2500, "keep emulated cases small"
    got, cnt, status = emu.mine(g, gamma, ms, warps=warps, split=split, small_path=small_path,
                                shared_fifo=fifo)
    assert status == 0
    assert canon(got) == canon(want)
    assert cnt["tasks"] == st["tasks"]
    assert cnt["branches"] == st["branches"]
    assert cnt["children"] == st["children"]
    # the byte-model counters of the bench's roofline numerator
    for k in ("parent_vertices", "p_rows", "child_vertices"):
        assert cnt[k] == st[k], k


def test_emulated_batch_matches_oracle_per_instance():
    specs = [(22, 0.3, 11, 1, 7, 0.8, 4), (30, 0.25, 12, 2, 8, 0.9, 5), (18, 0.4, 13, 0, 0, 0.7, 4),
             (26, 0.3, 14, 1, 9, 1.0, 4), (40, 0.2, 15, 1, 12, 0.85, 6)]
    gs, gms, mss = [], [], []
    for n, p, seed, pl, sz, gm, ms in specs:
        gs.append(graphs.random_small(n, p, seed, planted=pl, size=sz, density=0.95))
        gms.append(gm)
        mss.append(ms)
    per, st = emu.mine_batch(gs, gms, mss)
    assert st == 0
    for g, gm, ms, got in zip(gs, gms, mss, per):
        want, _ = oracle.mine(g, gm, ms, "clean")
        assert canon(got) == canon(want)


@pytest.mark.parametrize("grid", [False, True])
@pytest.mark.parametrize("seed", range(12))
def test_emulated_device_level0_matches_oracle_root(seed, grid):
    """The product's device level 0 (one emulated block of 64 threads; the
    one-block form and the grid-wide form) gives the oracle's root: same
    vertices in the same Q order, same covered count."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(20, 200))
    g = graphs.random_small(n, float(rng.uniform(0.03, 0.3)), 500 + seed,
                            planted=int(rng.integers(0, 4)), size=int(rng.integers(5, 16)),
                            density=float(rng.uniform(0.8, 1.0)))
    gamma = [0.5, 0.6, 0.7, 0.8, 0.9, 1.0][seed % 6]
    ms = int(rng.integers(3, 9))
    want_ids, want_lab, _ = oracle.root(g, gamma, ms)
    ids, cov = emu.level0(g, gamma, ms, grid=grid)
    assert ids.tolist() == want_ids.tolist()
    assert cov == int((want_lab == 2).sum())
