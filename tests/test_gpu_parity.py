"""GPU path (through the C ABI) against the CPU oracle on the same seeded inputs.

Costs must match bit for bit; every returned tree must pass the validator
(edges exist with their weights, connected, acyclic, covers every query group,
weights sum to the cost, hop diameter <= D)."""
import numpy as np
import pytest

from gpugst_b200 import gen
from tests.cases import small_cases, tiny_cases

pytestmark = pytest.mark.gpu


def _engine(eng, g, gr):
    return eng.Engine.from_instance(g, gr)


def test_tiny_vs_brute(gst_lib, oracle_mod):
    eng, O = gst_lib, oracle_mod
    bad = []
    for i, (g, gr, q, D) in enumerate(tiny_cases(160)):
        E = _engine(eng, g, gr)
        for DD in (-1, D):
            want = O.brute(g, gr, q, DD)
            r = E.query(q, D=DD)
            if want < 0:
                if r.status != eng.GST_NO_SOLUTION:
                    bad.append((i, DD, "want no solution", r.status, r.cost))
                continue
            if r.status != eng.GST_OK or r.cost != want:
                bad.append((i, DD, want, r.status, r.cost))
                continue
            v = O.validate(g, gr, q, DD, r.cost, r.root, r.edges)
            if v:
                bad.append((i, DD, "invalid tree", v))
        E.close()
    assert not bad, bad[:10]


def test_small_plain_vs_oracle(gst_lib, oracle_mod):
    eng, O = gst_lib, oracle_mod
    bad = []
    for i, (g, gr, q) in enumerate(small_cases(24)):
        E = _engine(eng, g, gr)
        want = O.prunedpp(g, gr, q, 0)
        r = E.query(q)
        if want.status != 0:
            if r.status != eng.GST_NO_SOLUTION:
                bad.append((i, "no-solution", r.status))
        elif r.status != eng.GST_OK or r.cost != want.cost:
            bad.append((i, want.cost, r.status, r.cost))
        elif O.validate(g, gr, q, -1, r.cost, r.root, r.edges):
            bad.append((i, "invalid tree"))
        E.close()
    assert not bad, bad


def test_small_hop_vs_oracle(gst_lib, oracle_mod):
    eng, O = gst_lib, oracle_mod
    bad = []
    for i, (g, gr, q) in enumerate(small_cases(16, seed0=300, V=200, E=800, kmax=4)):
        E = _engine(eng, g, gr)
        for D in (1, 2, 3, 4):
            want = O.hop(g, gr, q, D)
            r = E.query(q, D=D)
            if want.status != 0:
                if r.status != eng.GST_NO_SOLUTION:
                    bad.append((i, D, "no-solution", r.status, r.cost))
            elif r.status != eng.GST_OK or r.cost != want.cost:
                bad.append((i, D, want.cost, r.status, r.cost))
            elif O.validate(g, gr, q, D, r.cost, r.root, r.edges):
                bad.append((i, D, "invalid tree"))
        E.close()
    assert not bad, bad


@pytest.fixture(scope="module")
def c1():
    return gen.config1()


def test_config1_plain(gst_lib, oracle_mod, c1):
    eng, O = gst_lib, oracle_mod
    g, gr, qs = c1
    E = _engine(eng, g, gr)
    bad = []
    for i, q in enumerate(qs[3]):
        want = O.prunedpp(g, gr, q, 0)
        r = E.query(q)
        if r.status != eng.GST_OK or r.cost != want.cost:
            bad.append((i, want.cost, r.status, r.cost))
        elif O.validate(g, gr, q, -1, r.cost, r.root, r.edges):
            bad.append((i, "invalid tree"))
    E.close()
    assert not bad, bad


def test_config1_hop(gst_lib, oracle_mod, c1):
    eng, O = gst_lib, oracle_mod
    g, gr, qs = c1
    E = _engine(eng, g, gr)
    bad = []
    for i, q in enumerate(qs[3][:12]):
        for D in (2, 3, 4):
            want = O.hop(g, gr, q, D)
            r = E.query(q, D=D)
            if want.status != 0:
                if r.status != eng.GST_NO_SOLUTION:
                    bad.append((i, D, "no-solution", r.status, r.cost))
            elif r.status != eng.GST_OK or r.cost != want.cost:
                bad.append((i, D, want.cost, r.status, r.cost))
            elif O.validate(g, gr, q, D, r.cost, r.root, r.edges):
                bad.append((i, D, "invalid tree"))
    E.close()
    assert not bad, bad


def test_batch_alone_vs_mixed(gst_lib, c1):
    """Each query gives the same cost alone and inside a mixed batch."""
    eng = gst_lib
    g, gr, qs = c1
    rng = np.random.default_rng(5)
    queries, Ds = [], []
    for i in range(40):
        k = int(rng.integers(2, 6))
        queries.append(rng.choice(gr.n_groups, size=k, replace=False).astype(np.uint32))
        Ds.append(int(rng.choice([-1, 2, 3, 4])))
    E = _engine(eng, g, gr)
    alone = [E.query(q, D=D) for q, D in zip(queries, Ds)]
    mixed = E.query_batch(queries, Ds)
    E.close()
    for a, m in zip(alone, mixed):
        assert a.status == m.status
        assert a.cost == m.cost


def test_queue_overflow_retry(gst_lib, oracle_mod, c1, monkeypatch):
    """Frontier lists far too small for the query: the engine reruns each
    overflowed query with 4x larger lists and still returns the optimum."""
    eng, O = gst_lib, oracle_mod
    g, gr, qs = c1
    monkeypatch.setenv("GSTB_QUEUE_CAP", "1024")
    E = _engine(eng, g, gr)
    queries = list(qs[3][:8])
    Ds = [-1] * 4 + [3] * 4
    res = E.query_batch(queries, Ds)
    one = E.query(queries[0])
    E.close()
    assert sum(r.stats["retries"] for r in res) > 0
    for q, D, r in zip(queries, Ds, res):
        want = O.prunedpp(g, gr, q, 0) if D < 0 else O.hop(g, gr, q, D)
        if want.status != 0:
            assert r.status == eng.GST_NO_SOLUTION, (D, r.status)
            continue
        assert r.status == eng.GST_OK and r.cost == want.cost, (D, want.cost, r.status, r.cost)
        assert not O.validate(g, gr, q, D, r.cost, r.root, r.edges)
    assert one.status == eng.GST_OK and one.cost == res[0].cost


def test_edge_cases(gst_lib, oracle_mod):
    eng, O = gst_lib, oracle_mod
    # path 0-1-2-3 plus isolated vertex 4
    u = np.array([0, 1, 2]); v = np.array([1, 2, 3]); w = np.array([5, 7, 11], dtype=np.int32)
    g = gen.csr_from_edges(5, u, v, w)
    ptr = np.array([0, 1, 2, 3, 4, 6, 7], dtype=np.uint64)
    mem = np.array([0, 3, 1, 4, 0, 3, 2], dtype=np.uint32)
    gr = gen.Groups(ptr, mem)
    E = eng.Engine.from_instance(g, gr)
    r = E.query([0])                      # k = 1: a single member vertex
    assert r.ok and r.cost == 0 and len(r.edges) == 0
    r = E.query([0, 4])                   # vertex 0 is in both groups
    assert r.ok and r.cost == 0
    r = E.query([0, 1])                   # 0 .. 3 along the path
    assert r.ok and r.cost == 23 and O.validate(g, gr, np.array([0, 1]), -1, r.cost, r.root, r.edges) == 0
    r = E.query([0, 1], D=2)              # needs 3 hops
    assert r.status == eng.GST_NO_SOLUTION
    r = E.query([0, 1], D=3)
    assert r.ok and r.cost == 23
    r = E.query([0, 3])                   # group 3 = {4}, isolated
    assert r.status == eng.GST_NO_SOLUTION
    r = E.query([1, 2, 5])
    assert r.ok and r.cost == O.prunedpp(g, gr, np.array([1, 2, 5]), 0).cost
    for bad_q, bad_d in (([], -1), ([0] * 9, -1), ([0, 0], -1), ([0, 99], -1), ([0, 1], 8)):
        r = E.query(bad_q, D=bad_d) if bad_q else None
        if r is not None:
            assert r.status == eng.GST_BAD_INPUT, (bad_q, bad_d, r.status)
    E.close()


def test_serve_alone_vs_in_the_mix(gst_lib, c1):
    """Continuous batching: requests submitted while others run give the same
    cost as the same request run alone (integer costs: equal)."""
    import time
    eng = gst_lib
    g, gr, qs = c1
    rng = np.random.default_rng(9)
    reqs = []
    for i in range(60):
        k = int(rng.integers(2, 6))
        reqs.append((rng.choice(gr.n_groups, size=k, replace=False).astype(np.uint32), int(rng.choice([-1, 2, 3, 4]))))
    E = _engine(eng, g, gr)
    alone = [E.query(q, D=D) for q, D in reqs]
    S = eng.Server(E, max_inflight=16)
    got = {}
    for i, (q, D) in enumerate(reqs):
        assert S.submit(i, q, D) == eng.GST_OK
        if i % 7 == 0:
            for rid, r in S.poll():
                got[rid] = r
    t0 = time.time()
    while len(got) < len(reqs) and time.time() - t0 < 120:
        for rid, r in S.poll(max_edges=4096):
            got[rid] = r
        time.sleep(0.002)
    S.close()
    E.close()
    assert len(got) == len(reqs)
    for i, a in enumerate(alone):
        assert got[i].status == a.status, (i, got[i].status, a.status)
        assert got[i].cost == a.cost, (i, got[i].cost, a.cost)
        assert got[i].latency_ms >= 0


def test_autotune_keeps_results_exact(gst_lib, oracle_mod, c1):
    """The autotuner only changes the work schedule: after tuning on a sample,
    every cost still matches the oracle; explicit settings round-trip."""
    eng, O = gst_lib, oracle_mod
    g, gr, qs = c1
    E = _engine(eng, g, gr)
    sample = list(qs[3][:16])
    t = E.autotune(sample, objective="throughput")
    assert t["delta_sssp"] in (8, 16, 32, 64) and t["delta_dp"] in (2, 4, 8, 16)
    assert t["hub_min_deg"] in (128, 256, 512, 1024) and t["cap_pct"] in (50, 60, 67, 75)
    assert t["persistent"] in (0, 1) and t["rounds_per_launch"] in (2, 4, 8, 16)
    assert t["dp_wmax"] in (4, 8, 16, 32) and t["sssp_wmax"] in (8, 16, 32) and t["merge_stage"] in (0, 6, 14, 30)
    assert t["block_threads"] in (128, 256)
    assert E.tuning() == t
    res = E.query_batch(list(qs[3][16:28]))
    for q, r in zip(qs[3][16:28], res):
        assert r.status == eng.GST_OK and r.cost == O.prunedpp(g, gr, q, 0).cost
    for persistent in (0, 1):
        want = {"delta_sssp": 8, "delta_dp": 2, "hub_min_deg": 128, "cap_pct": 100, "persistent": persistent,
                "rounds_per_launch": 2, "dp_wmax": 4, "sssp_wmax": 8, "merge_stage": 6 * persistent,
                "block_threads": 256 - 128 * persistent}
        E.set_tuning(**want)
        assert E.tuning() == want
        for q in qs[3][28:32]:
            r = E.query(q)
            assert r.status == eng.GST_OK and r.cost == O.prunedpp(g, gr, q, 0).cost
    with pytest.raises(eng.GstError):
        E.set_tuning(dp_wmax=3)  # not a power of two
    with pytest.raises(eng.GstError):
        E.set_tuning(block_threads=512)
    with pytest.raises(ValueError):
        E.set_tuning(block=1)
    E.close()


def test_progressive_mode(gst_lib, oracle_mod, c1):
    """Progressive mode (gst_query_ratio / gst_query_batch_ratio /
    gst_serve_submit_ratio): the cost is at least the optimum and at most
    ratio x the optimum (and ratio x the reported lower bound, which is at
    most the optimum); the tree is valid; ratio <= 1 and hop-bounded queries
    are exact."""
    import time
    eng, O = gst_lib, oracle_mod
    bad = []
    insts = [(c1[0], c1[1], list(c1[2][3][:16]))]
    for g, gr, q in small_cases(8, seed0=900, V=2000, E=12000, n_groups=150, smax=10, kmax=6):
        insts.append((g, gr, [q]))
    early = 0
    for g, gr, queries in insts:
        E = _engine(eng, g, gr)
        for q in queries:
            opt = O.prunedpp(g, gr, q, 0).cost
            for ratio in (1.0, 1.25, 1.5, 2.0, 4.0):
                r = E.query(q, ratio=ratio)
                lb = r.stats["lower_bound"]
                if r.status != eng.GST_OK or not (opt <= r.cost <= int(ratio * opt)) or lb > opt:
                    bad.append((q.tolist(), ratio, opt, r.status, r.cost, lb))
                    continue
                if r.cost > ratio * lb or (ratio <= 1.0 and r.cost != opt):
                    bad.append((q.tolist(), ratio, "bound", opt, r.cost, lb))
                if O.validate(g, gr, q, -1, r.cost, r.root, r.edges):
                    bad.append((q.tolist(), ratio, "invalid tree"))
                early += lb < opt
            # hop-bounded queries ignore the ratio
            h = E.query(q, D=3, ratio=2.0)
            want = O.hop(g, gr, q, 3)
            if (want.status == 0) != (h.status == eng.GST_OK) or (want.status == 0 and h.cost != want.cost):
                bad.append((q.tolist(), "hop", want.cost, h.status, h.cost))
        # batch and serving entry points agree with the bound
        res = E.query_batch(queries, ratios=[1.5] * len(queries))
        S = eng.Server(E, max_inflight=8)
        for i, q in enumerate(queries):
            S.submit(i, q, ratio=1.5)
        got = {}
        t0 = time.time()
        while len(got) < len(queries) and time.time() - t0 < 60:
            for rid, rr in S.poll(max_edges=4096):
                got[rid] = rr
            time.sleep(0.001)
        S.close()
        for i, q in enumerate(queries):
            opt = O.prunedpp(g, gr, q, 0).cost
            for tag, rr in (("batch", res[i]), ("serve", got.get(i))):
                if rr is None or rr.status != eng.GST_OK or not (opt <= rr.cost <= int(1.5 * opt)):
                    bad.append((tag, q.tolist(), opt, None if rr is None else (rr.status, rr.cost)))
        E.close()
    assert not bad, bad[:10]
    assert early > 0, "no query stopped early: the progressive exit was never exercised"
