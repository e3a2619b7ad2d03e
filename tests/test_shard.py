"""Box sharding over ranks (CPU, and two gloo ranks): every box on exactly
one rank, loads balanced by longest-processing-time-first, and the timing
reductions the bench uses (max over ranks) with a real process group."""
import os
import socket

import pytest

from lageunha_b200 import ic
from lageunha_b200 import shard


def test_assignment_covers_every_box_once():
    sizes = [ic.ensemble_spec(b)[0] ** 3 for b in range(64)]
    for nr in (1, 2, 3, 4, 8):
        a = shard.assign_boxes(sizes, nr)
        assert len(a) == nr
        flat = sorted(i for r in a for i in r)
        assert flat == list(range(64))
        loads = shard.rank_loads(sizes, a)
        # LPT: the busiest rank is within 4/3 of the mean load (the optimum's
        # lower bound) plus the largest single box
        mean = sum(loads) / nr
        assert max(loads) <= 4.0 / 3.0 * mean + max(shard.box_cost(s) for s in sizes)


def test_more_ranks_than_boxes():
    a = shard.assign_boxes([10, 20], 4)
    assert sorted(i for r in a for i in r) == [0, 1]
    assert sum(1 for r in a if not r) == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = [ic.ensemble_spec(b)[0] ** 3 for b in range(64)]
    mine = shard.assign_boxes(sizes, world)[rank]
    # a stand-in for the rank's measured time: its share of the work
    t = float(sum(shard.box_cost(sizes[i]) for i in mine))
    tmax = shard.max_over_ranks(t, dist)
    tot = shard.sum_over_ranks(float(len(mine)), dist)
    q.put((rank, mine, t, tmax, tot))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_timings():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    boxes = sorted(res[0][1] + res[1][1])
    assert boxes == list(range(64))
    assert res[0][3] == res[1][3] == max(res[0][2], res[1][2])
    assert res[0][4] == res[1][4] == 64
