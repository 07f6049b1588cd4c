"""The multi-process path of bench.py on the CPU: world-size-2 gloo ranks
(127.0.0.1 rendezvous) agree on the max-over-ranks time the job rate is
computed from, and the reference arm does its work on rank 0 only."""
import os
import socket
import sys
from datetime import timedelta

import multiprocessing as mp

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist

    import bench as b

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    elapsed_ms = 100.0 + 50.0 * rank  # rank 1 is the slower one
    m = b.max_over_ranks(elapsed_ms, dist, None)
    steps = 10
    q.put((rank, m, world * steps / (m / 1000.0)))
    dist.barrier()
    dist.destroy_process_group()


def test_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [m for _, m, _ in out] == [150.0, 150.0]
    # whole-job rate: both ranks' steps over the slowest rank's time
    assert all(abs(rate - 2 * 10 / 0.150) < 1e-9 for _, _, rate in out)


def test_single_process_max_is_the_value_itself():
    assert bench.max_over_ranks(12.5) == 12.5


def test_reference_arm_works_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")

    class Args:
        workload = "cfg1"
        gpus = 2
        steps = 1
        warmup = 0

    assert bench.run_reference(Args()) is None
    assert capsys.readouterr().out == ""


def _replica_rank(rank, world, port, q):
    """One rank of the replica job with the GPU call replaced by a host stub:
    each rank mines its own copy of the instance on its own device index."""
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist

    import bench as b

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    dev = b.replica_device()
    calls = []

    def step():  # stand-in for one qc_mine on GPU `dev`: result and device ms
        calls.append(dev)
        return ("sets of instance", dev), 2.0 + rank  # rank 1 is slower

    rate, slowest, outs = b.replica_rate(3, 5, step, lambda r: r == ("sets of instance", dev),
                                         dist.barrier, dist, None)
    bad = None
    try:
        b.replica_rate(0, 1, lambda: (("other", dev), 1.0), lambda r: r[0] == "sets of instance",
                       dist.barrier, dist, None)
    except SystemExit as e:
        bad = str(e)
    q.put((rank, dev, len(calls), rate, slowest, len(outs), bad))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_dispatch_on_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_replica_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, dev, ncalls, rate, slowest, nout, bad in out:
        assert dev == rank                       # rank i mines on GPU i
        assert ncalls == 3 + 5 and nout == 5     # warm-up steps untimed, 5 timed
        assert slowest == 5 * 3.0                # the slower rank's 5 steps of 3 ms
        assert abs(rate - 2 * 5 / 0.015) < 1e-9  # both ranks' steps over that time
        assert bad is not None and "differs" in bad


def test_gpus_flag_without_launcher_spawns_ranks(monkeypatch):
    seen = {}

    def fake_call(cmd):
        seen["cmd"] = cmd
        return 0

    monkeypatch.setattr(bench.subprocess, "call", fake_call)
    monkeypatch.setattr(bench.sys, "argv", ["bench.py", "--gpus", "4", "--steps", "2"])

    class Args:
        gpus = 4

    assert bench.spawn_ranks(Args()) == 0
    cmd = seen["cmd"]
    assert cmd[1:4] == ["-m", "torch.distributed.run", "--nnodes=1"]
    assert cmd[cmd.index("--nproc-per-node") + 1] == "4"
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-4:] == ["--gpus", "4", "--steps", "2"]


def _shard_rank(rank, world, port, q):
    """One rank of a graph mined in shards, with the GPU calls replaced by host
    stand-ins: a shard's result is its share of a known family of sets, the
    merge is the oracle's maximal-set filter."""
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import numpy as np
    import torch.distributed as dist

    from cuqc_b200 import shard
    from oracle import oracle

    fam = [(0, 1, 2), (0, 1), (3, 4, 5, 6), (1, 2), (4, 5), (7,), (0, 1, 2), (6, 7, 8)]

    def pack(sets):
        out = []
        for s in sets:
            out += [len(s)] + list(s)
        return np.asarray(out, np.int32)

    class FakeResult:
        def __init__(self, flat):
            self.flat = flat
            self.sets = oracle.maximal(flat)

    class FakeCtx:
        def mine_shard(self, g, gamma, ms, s, n):
            assert (s, n) == (rank, world)
            return FakeResult(pack(fam[s::n]))

        def maximal_sets(self, flat, nv):
            return FakeResult(flat)

    class G:
        n = 9

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    r = shard.mine_sharded(FakeCtx(), G(), 0.9, 2, dist, None)
    q.put((rank, r.sets, oracle.maximal(pack(fam))))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_merge_on_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, want in out:
        assert got == want == [(0, 1, 2), (3, 4, 5, 6), (6, 7, 8)]
