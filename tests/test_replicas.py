"""Replica sharding and max-over-ranks timing, as 2 gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gpugst_b200 import replicas


def test_shard_covers_disjoint():
    for n in (0, 1, 7, 90, 901):
        for world in (1, 2, 3, 8):
            got = [list(replicas.shard(n, r, world)) for r in range(world)]
            flat = [x for g in got for x in g]
            assert flat == list(range(n))
            assert max(len(g) for g in got) - min(len(g) for g in got) <= 1
    with pytest.raises(ValueError):
        replicas.shard(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = list(replicas.shard(90, rank, world))
    t = replicas.max_over_ranks([10.0 + rank, 5.0 - rank])
    n = replicas.sum_over_ranks([len(mine)])
    out.put((rank, mine[0], len(mine), t, n))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == 0 and res[1][1] == 45 and res[0][2] == res[1][2] == 45
    for r in res:
        assert r[3] == [11.0, 5.0]  # max over ranks
        assert r[4] == [90.0]
