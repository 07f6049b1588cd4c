"""One graph mined on several GPUs: the search split by the root's branches.

Each rank (one process per GPU) mines its shard of the root's branches with
qc_mine_shard, the ranks exchange their shards' maximal sets (an all-gather of
the sizes, then of the payloads), and every rank merges them with
qc_maximal_sets: the maximal sets of the union of the shards' results are the
maximal sets of the whole graph.  This is the only exchange of the search; the
reference mines on one GPU (search, main.cu:535-692), so the split has no
counterpart there.
"""
from __future__ import annotations

import numpy as np


def gather_flat(flat, dist, device=None):
    """Every rank's flat int32 array, on every rank, in rank order: the sizes
    are all-gathered first, then the payloads padded to the largest."""
    import torch

    world = dist.get_world_size()
    n = torch.tensor([len(flat)], dtype=torch.int64, device=device)
    sizes = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(sizes, n)
    sizes = [int(x.item()) for x in sizes]
    width = max(max(sizes), 1)
    mine = torch.zeros(width, dtype=torch.int32, device=device)
    if len(flat):
        mine[: len(flat)] = torch.as_tensor(np.asarray(flat, np.int32), device=device)
    parts = [torch.zeros(width, dtype=torch.int32, device=device) for _ in range(world)]
    dist.all_gather(parts, mine)
    return [p[:k].cpu().numpy() for p, k in zip(parts, sizes)]


def mine_sharded(ctx, g, gamma, min_size, dist=None, device=None):
    """The maximal gamma-quasi-cliques of g mined by all ranks together: rank r
    takes shard r of world_size.  Without a process group: one shard, which is
    the whole search.  Returns the merged Result (on every rank)."""
    if dist is None or dist.get_world_size() == 1:
        return ctx.mine(g, gamma, min_size)
    rank, world = dist.get_rank(), dist.get_world_size()
    part = ctx.mine_shard(g, gamma, min_size, rank, world)
    parts = gather_flat(part.flat, dist, device)
    merged = np.concatenate(parts) if parts else np.zeros(0, np.int32)
    return ctx.maximal_sets(merged, g.n if hasattr(g, "n") else ctx_graph_n(g))


def ctx_graph_n(dg):
    """Vertex count of a graph already handed to the library."""
    from . import lib

    return lib().qc_graph_num_vertices(dg.h)
