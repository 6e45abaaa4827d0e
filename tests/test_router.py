"""Replica routing and per-replica admission on the CPU, against fake
replicas with settable occupancy (no GPU: the policy and the bookkeeping are
host logic), plus a GPU test of the real front-end on one device."""
import pytest

from gpugst_b200 import router


class FakeReplica:
    """Stands in for engine.Server: a replica with an HBM budget, a pending
    queue limit and requests that finish when the test says so."""

    def __init__(self, budget, max_pending=4, need=100):
        self.budget, self.max_pending, self.need = budget, max_pending, need
        self.pending, self.running, self.finished = [], [], []
        self.closed = False

    def stats(self):
        return {"pending": len(self.pending), "inflight": len(self.running), "budget_bytes": self.budget,
                "in_use_bytes": self.need * len(self.running)}

    def submit(self, req_id, groups, D=-1, ratio=0.0):
        if len(self.pending) >= self.max_pending:
            return router.GST_BUSY
        self.pending.append(req_id)
        self.admit()
        return router.GST_OK

    def admit(self):
        # per-replica admission: a request runs once its workspace fits the budget
        while self.pending and self.need * (len(self.running) + 1) <= self.budget:
            self.running.append(self.pending.pop(0))

    def finish_all(self):
        self.finished += [(r, "done") for r in self.running]
        self.running = []
        self.admit()

    def poll(self, max_results=1024, max_edges=0):
        out, self.finished = self.finished[:max_results], self.finished[max_results:]
        return out

    def cancel(self, req_id):
        if req_id in self.pending:
            self.pending.remove(req_id)
            self.finished.append((req_id, "cancelled"))
            return router.GST_OK
        return router.GST_NOT_FOUND

    def close(self):
        self.closed = True


def test_choose_orders_by_policy():
    st = [{"pending": 3, "inflight": 1, "budget_bytes": 1000, "in_use_bytes": 100},
          {"pending": 0, "inflight": 2, "budget_bytes": 1000, "in_use_bytes": 600},
          {"pending": 1, "inflight": 0, "budget_bytes": 500, "in_use_bytes": 0}]
    assert router.choose(st, "free_hbm") == [0, 2, 1]   # free 900, 500, 400
    assert router.choose(st, "queue") == [2, 1, 0]      # queue 1, 2, 4
    with pytest.raises(ValueError):
        router.choose(st, "random")
    with pytest.raises(ValueError):
        router.Router([FakeReplica(1)], "random")


def test_routes_to_most_free_hbm_and_spills_over_when_busy():
    a, b = FakeReplica(budget=300, max_pending=1), FakeReplica(budget=200, max_pending=1)
    R = router.Router([a, b], "free_hbm")
    for i in range(5):
        assert R.submit(i, [1, 2, 3]) == router.GST_OK
    # free budget 300 vs 200 -> a; 200 vs 200 (a's queue longer) -> b; 200 vs 100 -> a;
    # 100 vs 100 -> b; 100 vs 0 -> a: both budgets are then full
    assert a.running == [0, 2, 4] and b.running == [1, 3]
    # then the pending queues fill; with every replica full the caller gets BUSY
    assert R.submit(5, [1]) == router.GST_OK
    assert R.submit(6, [1]) == router.GST_OK
    assert R.submit(7, [1]) == router.GST_BUSY
    assert len(a.pending) == 1 and len(b.pending) == 1
    assert sum(R.routed) == 7 == len(R.owner)


def test_queue_policy_balances_and_poll_cancel_close():
    reps = [FakeReplica(budget=10_000, max_pending=100, need=10_000) for _ in range(3)]
    R = router.Router(reps, "queue")
    for i in range(9):
        assert R.submit(i, [4, 5]) == router.GST_OK
    assert [len(r.pending) + len(r.running) for r in reps] == [3, 3, 3]
    victim = next(rid for rid in range(9) if rid in reps[R.owner[rid]].pending)
    assert R.cancel(victim) == router.GST_OK
    assert R.cancel(12345) == router.GST_NOT_FOUND
    for r in reps:
        r.finish_all()
    got = dict(R.poll())
    assert got[victim] == "cancelled"
    assert len(got) == 3 + 1  # the three that ran + the cancelled one
    R.close()
    assert all(r.closed for r in reps)


@pytest.mark.gpu
def test_router_on_one_device_matches_plain(gst_lib):
    """The real front-end over two serving loops (both on device 0): every
    result equals the plain path's."""
    import time

    from gpugst_b200 import gen
    eng = gst_lib
    g, gr, qs = gen.config1()
    E1 = eng.Engine.from_instance(g, gr)
    E2 = eng.Engine.from_instance(g, gr)
    R = router.Router([eng.Server(E1, max_inflight=4), eng.Server(E2, max_inflight=4)], "queue")
    queries = list(qs[3][:24])
    for i, q in enumerate(queries):
        assert R.submit(i, q) == eng.GST_OK
    got = {}
    t0 = time.time()
    while len(got) < len(queries) and time.time() - t0 < 60:
        for rid, r in R.poll():
            got[rid] = r
        time.sleep(0.001)
    R.close()
    want = [E1.query(q).cost for q in queries]
    E1.close()
    E2.close()
    assert [got[i].cost for i in range(len(queries))] == want
    assert min(R.routed) > 0
