"""Multi-GPU replica serving: a front-end over one serving loop per GPU.

Queries are independent, so the path scales by replicas: every GPU holds its
own copy of the graph and group index (gst_graph_create on that device) and
runs its own continuous-batching loop (gst_serve_*), which admits requests
by the free HBM of its own budget.  The front-end sends each request to one
replica, chosen from the replicas' live occupancy (gst_serve_stats):

  policy "free_hbm"  the replica with the most free workspace budget
                     (budget - bytes held by admitted requests), ties broken
                     by the shorter queue;
  policy "queue"     the replica with the fewest requests waiting or running,
                     ties broken by the larger free budget.

A replica that sheds the request (GST_BUSY: its pending queue is full) is
skipped and the next best one takes it; only when every replica is full is
GST_BUSY returned to the caller.  No collective and no peer memory is on the
data path: each replica reads only its own GPU's copy of the graph.

The reference runs its queries one after another on one GPU
(code/GPUGST/include/exp_GPU_nonHop.h:97-138); it has no multi-GPU path.
"""
from __future__ import annotations

from typing import Dict, List, Sequence

GST_OK, GST_BUSY, GST_NOT_FOUND = 0, 9, 10


def choose(stats: Sequence[dict], policy: str = "free_hbm") -> List[int]:
    """Replica indices in routing preference order for the given occupancies
    (dicts with pending, inflight, budget_bytes, in_use_bytes)."""
    def free(s):
        return int(s["budget_bytes"]) - int(s["in_use_bytes"])

    def queue(s):
        return int(s["pending"]) + int(s["inflight"])

    if policy == "free_hbm":
        key = lambda i: (-free(stats[i]), queue(stats[i]), i)  # noqa: E731
    elif policy == "queue":
        key = lambda i: (queue(stats[i]), -free(stats[i]), i)  # noqa: E731
    else:
        raise ValueError(f"unknown policy {policy!r}")
    return sorted(range(len(stats)), key=key)


class Router:
    """Routes requests over replica servers (engine.Server or any object with
    submit / poll / cancel / stats / close of the same meaning)."""

    def __init__(self, servers, policy: str = "free_hbm"):
        if not servers:
            raise ValueError("no replicas")
        if policy not in ("free_hbm", "queue"):
            raise ValueError(f"unknown policy {policy!r}")
        self.servers = list(servers)
        self.policy = policy
        self.owner: Dict[int, int] = {}
        self.routed = [0] * len(self.servers)

    def submit(self, req_id: int, groups, D: int = -1, ratio: float = 0.0) -> int:
        order = choose([s.stats() for s in self.servers], self.policy)
        for r in order:
            st = self.servers[r].submit(req_id, groups, D, ratio=ratio)
            if st == GST_BUSY:
                continue
            if st == GST_OK:
                self.owner[req_id] = r
                self.routed[r] += 1
            return st
        return GST_BUSY

    def poll(self, max_results: int = 1024, max_edges: int = 0):
        """Finished requests of every replica: a list of (req_id, result)."""
        out = []
        for s in self.servers:
            got = s.poll(max_results=max_results, max_edges=max_edges)
            for rid, _ in got:
                self.owner.pop(rid, None)
            out.extend(got)
        return out

    def cancel(self, req_id: int) -> int:
        r = self.owner.get(req_id)
        if r is None:
            return GST_NOT_FOUND
        return self.servers[r].cancel(req_id)

    def stats(self) -> List[dict]:
        return [s.stats() for s in self.servers]

    def close(self):
        for s in self.servers:
            s.close()


def open_replicas(graph, groups, devices, hbm_budget: int = 0, max_inflight: int = 0, policy: str = "free_hbm"):
    """One engine and serving loop per CUDA device in `devices` (each graph
    copy is created with its device current) behind a Router.  Returns
    (router, engines); close the router, then the engines."""
    import torch

    from . import engine
    engines, servers = [], []
    for d in devices:
        torch.cuda.set_device(int(d))
        E = engine.Engine.from_instance(graph, groups)
        engines.append(E)
        servers.append(engine.Server(E, hbm_budget=hbm_budget, max_inflight=max_inflight))
    return Router(servers, policy), engines
