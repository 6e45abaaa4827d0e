"""The persistent round launch (k_rounds: a block of rounds as one cooperative
launch) against the CUDA-graph round blocks (control / light / heavy launches
per round) and the oracle, at both block sizes, and its bounded waits: a
launch whose control steps are held ends with GST_DEVICE_TIMEOUT and the
device stays usable."""
import time

import pytest

from gpugst_b200 import gen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    return gen.config1()


def _mixed(qs):
    """Unbounded and hop-bounded queries of config 1, k = 3."""
    queries = list(qs[3][:16])
    Ds = [-1] * 10 + [2, 3, 4, 2, 3, 4]
    return queries, Ds


def test_persistent_matches_graph_rounds_and_oracle(gst_lib, oracle_mod, c1):
    eng, O = gst_lib, oracle_mod
    g, gr, qs = c1
    queries, Ds = _mixed(qs)
    E = eng.Engine.from_instance(g, gr)
    got = {}
    # launch mode x rounds per launch at 256 threads a block, and both modes at 128
    configs = [(m, r, 256) for m in (0, 1) for r in (1, 4, 16)] + [(0, 4, 128), (1, 4, 128)]
    for mode, rpl, bt in configs:
        E.set_tuning(persistent=mode, rounds_per_launch=rpl, block_threads=bt)
        batch = E.query_batch(queries, Ds)
        plain = [E.query(q, D=d) for q, d in zip(queries[8:12], Ds[8:12])]
        got[(mode, rpl, bt)] = [(r.status, r.cost) for r in batch] + [(r.status, r.cost) for r in plain]
        for q, d, r in zip(queries, Ds, batch):
            if r.status == eng.GST_OK:
                assert not O.validate(g, gr, q, d, r.cost, r.root, r.edges)
    ref = got[(0, 4, 256)]
    for key, val in got.items():
        assert val == ref, key
    for (st, cost), q, d in zip(ref, queries, Ds):
        want = O.prunedpp(g, gr, q, 0) if d < 0 else O.hop(g, gr, q, d)
        if want.status != 0:
            assert st == eng.GST_NO_SOLUTION
        else:
            assert st == eng.GST_OK and cost == want.cost
    E.close()


def test_persistent_serving_matches(gst_lib, c1):
    """The serving loop over persistent launches returns the plain results."""
    eng = gst_lib
    g, gr, qs = c1
    queries, Ds = _mixed(qs)
    E = eng.Engine.from_instance(g, gr)
    E.set_tuning(persistent=1)
    want = [(r.status, r.cost) for r in (E.query(q, D=d) for q, d in zip(queries, Ds))]
    S = eng.Server(E, max_inflight=8)
    for i, (q, d) in enumerate(zip(queries, Ds)):
        assert S.submit(i, q, D=d) == eng.GST_OK
    got = {}
    t0 = time.time()
    while len(got) < len(queries) and time.time() - t0 < 60:
        for rid, r in S.poll():
            got[rid] = (r.status, r.cost)
        time.sleep(0.001)
    S.close()
    E.close()
    assert [got[i] for i in range(len(queries))] == want


def test_held_rounds_time_out_and_device_recovers(gst_lib, c1):
    """Every wait of the persistent launch is bounded: with its control steps
    held (a flag that nothing sets), the launch gives up after the limit and
    the query reports GST_DEVICE_TIMEOUT; released, the same engine answers
    the query again."""
    eng = gst_lib
    g, gr, qs = c1
    q = qs[3][0]
    E = eng.Engine.from_instance(g, gr)
    E.set_tuning(persistent=1)
    want = E.query(q)
    assert want.status == eng.GST_OK
    E.hold_rounds(True, timeout_ms=200)
    t0 = time.time()
    r = E.query(q)
    dt = time.time() - t0
    assert r.status == eng.GST_DEVICE_TIMEOUT, r.status
    assert dt < 20, dt
    E.hold_rounds(False)
    again = E.query(q)
    assert again.status == eng.GST_OK and again.cost == want.cost
    res = E.query_batch(list(qs[3][:6]))
    assert all(x.status == eng.GST_OK for x in res)
    E.close()
