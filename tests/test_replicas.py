"""The N>1 layout (independent problems per rank) with two gloo ranks on the CPU."""
import os
import socket

import pytest

from gale_b200.replicas import shard


def test_shard_covers_every_problem_once():
    items = list(range(23))
    for world in (1, 2, 3, 8):
        parts = [shard(items, r, world) for r in range(world)]
        flat = sorted(x for p in parts for x in p)
        assert flat == items
        assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        shard(items, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    from gale_b200.replicas import max_over_ranks, shard, sum_over_ranks
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    mine = shard(list(range(10)), rank, world)
    t = max_over_ranks(0.5 + rank)          # per-rank "step time"
    n = sum_over_ranks(len(mine))            # problems solved over the job
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, t, n, mine))


def test_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [1.5, 1.5]          # max over ranks
    assert [o[2] for o in out] == [10.0, 10.0]        # every problem counted once
    assert out[0][3] == [0, 2, 4, 6, 8] and out[1][3] == [1, 3, 5, 7, 9]
