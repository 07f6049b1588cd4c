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
