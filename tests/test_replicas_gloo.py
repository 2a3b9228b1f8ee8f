"""The multi-GPU path (independent replicas) with two gloo ranks on the CPU:
shards are disjoint and cover the units, the timed region's duration is the
maximum over ranks, and the whole-job rate counts every rank's units."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pfb200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    r, w, lr = replicas.rank_world()
    units = [(50000 + i, 101 + 997 * i, 100) for i in range(11)]
    mine = replicas.shard(units, r, w)
    dist.barrier()
    seconds = 1.0 + r  # a slower rank 1
    t = replicas.max_over_ranks(seconds, dist)
    rate = replicas.aggregate_rate(len(units) / w, t, w)
    dist.barrier()
    dist.destroy_process_group()
    out.put((r, w, lr, mine, t, rate, replicas.rank_seed(1, r)))


def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, s0, t0, rate0, seed0), (r1, w1, l1, s1, t1, rate1, seed1) = res
    assert (r0, r1, w0, w1, l0, l1) == (0, 1, 2, 2, 0, 1)
    assert set(s0).isdisjoint(s1) and len(s0) + len(s1) == 11
    assert t0 == t1 == 2.0                      # the slowest rank's time, on every rank
    assert rate0 == rate1 == pytest.approx(11 / 2.0)
    assert seed0 == 1 and seed1 != seed0


def test_single_process_defaults():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.shard(list(range(5)), 0, 1) == [0, 1, 2, 3, 4]
