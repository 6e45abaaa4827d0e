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


def _leaver(rank, world, port, out):
    """Two gloo ranks; each step ends with the timing collective (max over
    ranks).  Rank 1 takes two steps and exits between steps; rank 0 must learn
    it from the heartbeat at step 2, before it enters that step's collective."""
    import datetime
    import torch.distributed as dist
    store = dist.TCPStore("127.0.0.1", port, world, rank == 0, timeout=datetime.timedelta(seconds=30))
    dist.init_process_group("gloo", store=store, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    hb = replicas.StepHeartbeat(store, rank, world, timeout_s=3.0)
    done = []
    try:
        for step in range(4):
            if rank == 1 and step == 2:
                out.put((rank, "left", done))
                return  # leaves between steps, nothing in flight
            hb.step(step)
            t = replicas.max_over_ranks([float(step + rank)])
            assert t == [float(step + 1)]
            done.append(step)
        out.put((rank, "finished", done))
    except replicas.RankLost as e:
        out.put((rank, f"lost {e.rank} at {e.step}", done))
        # the survivor keeps the store alive until the peer's process is gone
        import time
        time.sleep(0.5)


def test_rank_that_leaves_is_detected():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_leaver, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict((r, (msg, done)) for r, msg, done in (q.get(timeout=120) for _ in ps))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1] == ("left", [0, 1])
    assert res[0] == ("lost 1 at 2", [0, 1])
