"""qc_maximal_sets (the non-maximal removal step alone, on the device) against
the oracle's restatement of the reference's RemoveNonMax, on families with
repeated sets, subsets, unsorted ids, and universes on either side of the
256 ids up to which the survivors are ordered by bit vectors."""
import random

import numpy as np
import pytest

import cuqc_b200 as Q
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Q.Context(device=0)
    yield c
    c.close()


def family(seed, universe, n_sets, max_k):
    rng = random.Random(seed)
    ids = rng.sample(range(universe * 3), universe)  # scattered ids
    sets = []
    for _ in range(n_sets):
        k = rng.randint(1, max_k)
        sets.append(rng.sample(ids, k))
    # subsets and exact copies of earlier sets, ids in any order
    for _ in range(n_sets // 3):
        s = rng.choice(sets)
        sub = rng.sample(s, rng.randint(1, len(s)))
        sets.append(sub)
        cp = list(s)
        rng.shuffle(cp)
        sets.append(cp)
    rng.shuffle(sets)
    flat = []
    for s in sets:
        flat += [len(s)] + list(s)
    return np.array(flat, np.int32), universe * 3


@pytest.mark.parametrize("seed,universe,n_sets,max_k", [
    (1, 40, 300, 12),     # at most 256 distinct ids
    (2, 200, 2000, 30),
    (3, 600, 1500, 40),   # more than 256 distinct ids
    (4, 5000, 4000, 60),
    (5, 8, 200, 8),       # many repeats and subsets
])
def test_maximal_sets_match_oracle(ctx, seed, universe, n_sets, max_k):
    flat, nv = family(seed, universe, n_sets, max_k)
    want = [tuple(s) for s in oracle.maximal(flat)]
    got = ctx.maximal_sets(flat, nv)
    assert [tuple(s) for s in got.sets] == want
    assert got.stats["maximal"] == len(want)


def test_maximal_sets_edge_cases(ctx):
    assert ctx.maximal_sets(np.zeros(0, np.int32), 10).sets == []
    assert ctx.maximal_sets(np.array([1, 3], np.int32), 10).sets == [(3,)]
    same = np.array([3, 5, 1, 2] * 7, np.int32)  # one set seven times
    assert ctx.maximal_sets(same, 10).sets == [(1, 2, 5)]
    with pytest.raises(Q.QCError):
        ctx.maximal_sets(np.array([2, 4, 4], np.int32), 10)  # repeated id
    with pytest.raises(Q.QCError):
        ctx.maximal_sets(np.array([2, 4, 10], np.int32), 10)  # id out of range
    with pytest.raises(Q.QCError):
        ctx.maximal_sets(np.array([3, 1, 2], np.int32), 10)  # truncated record
