"""Multi-GPU replicas: queries are independent, so each rank (one process per
GPU, torch.distributed) holds its own copy of the graph and answers its own
share of the query stream.  There is no collective on the data path; the only
collectives are the timing reduction (max over ranks) and barriers."""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int):
    """Contiguous, disjoint, covering split of range(n_items) over ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(values, device=None):
    """Element-wise max of a list of floats over all ranks (identity when not distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def sum_over_ranks(values, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.tolist()]


class RankLost(RuntimeError):
    """A peer rank stopped taking steps (it exited or hangs outside a step)."""

    def __init__(self, rank: int, step: int):
        super().__init__(f"rank {rank} did not reach step {step}")
        self.rank = rank
        self.step = step


class StepHeartbeat:
    """Host-side liveness between steps of independent replicas.

    Replicas share no data-path collective, so a rank that leaves is not seen
    by a hung collective but by this check: before step i every rank posts i
    to the key-value store of the job (torch.distributed's TCPStore) and waits,
    for at most ``timeout_s``, until every peer has posted at least i.  A peer
    that never does raises RankLost on the ranks still running, before they
    launch anything else for that step, so no kernel or collective of theirs is
    left waiting on it."""

    def __init__(self, store, rank: int, world: int, timeout_s: float = 5.0, prefix: str = "gstb/hb"):
        self.store, self.rank, self.world = store, rank, world
        self.timeout_s, self.prefix = timeout_s, prefix

    def step(self, i: int):
        import datetime
        import time
        poll = datetime.timedelta(seconds=0.05)
        self.store.set(f"{self.prefix}/{self.rank}", str(i))
        deadline = time.monotonic() + self.timeout_s
        for peer in range(self.world):
            if peer == self.rank:
                continue
            key = f"{self.prefix}/{peer}"
            while True:
                try:
                    self.store.wait([key], poll)
                    seen = int(self.store.get(key))
                except Exception:
                    seen = -1
                if seen >= i:
                    break
                if time.monotonic() > deadline:
                    raise RankLost(peer, i)
                time.sleep(0.01)
