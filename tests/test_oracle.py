"""The CPU oracle against itself, brute force and the generators (no GPU)."""
import numpy as np
import pytest

from gpugst_b200 import gen
from tests.cases import small_cases, tiny_cases


def test_generators_shape():
    g, gr, qs = gen.config1()
    assert g.V == 10_000 and g.arcs == 100_000
    deg = np.diff(g.beg_pos.astype(np.int64))
    src = np.repeat(np.arange(g.V), deg)
    assert (src != g.csr).all(), "self-loop"
    # adjacency sorted by neighbour, no duplicates
    for v in range(0, g.V, 97):
        row = g.csr[g.beg_pos[v]:g.beg_pos[v + 1]]
        assert (np.diff(row.astype(np.int64)) > 0).all()
    # symmetric with equal weights
    key = src * g.V + g.csr.astype(np.int64)
    rkey = g.csr.astype(np.int64) * g.V + src
    order = np.argsort(key)
    rorder = np.argsort(rkey)
    assert (key[order] == rkey[rorder]).all()
    assert (g.weight[order] == g.weight[rorder]).all()
    assert g.weight.min() >= 1 and g.weight.max() <= 100
    assert gr.n_groups == 2000
    cov = np.zeros(g.V, bool)
    cov[gr.members] = True
    assert cov.all(), "every vertex is in a group"
    sizes = np.diff(gr.ptr.astype(np.int64))
    assert sizes.min() >= 1
    assert qs[3].shape == (50, 3)
    for q in qs[3]:
        assert len(set(q.tolist())) == 3


@pytest.mark.parametrize("chunk", range(4))
def test_oracle_tiny_vs_brute(oracle_mod, chunk):
    O = oracle_mod
    for g, gr, q, D in tiny_cases(60, seed0=chunk * 60):
        b = O.brute(g, gr, q)
        p = O.prunedpp(g, gr, q, 0)
        d = O.dpbf(g, gr, q)
        assert b == p.cost == d.cost
        if b >= 0:
            assert O.validate(g, gr, q, -1, p.cost, p.root, p.edges) == 0
            assert O.validate(g, gr, q, -1, d.cost, d.root, d.edges) == 0
        bh = O.brute(g, gr, q, D)
        h = O.hop(g, gr, q, D)
        assert bh == h.cost
        if bh >= 0:
            assert O.validate(g, gr, q, D, h.cost, h.root, h.edges) == 0


def test_oracle_config1_exact_modes(oracle_mod):
    """PrunedDP++ with ratio 0 (exact exits only) equals plain DPBF."""
    O = oracle_mod
    g, gr, qs = gen.config1()
    for q in qs[3][:25]:
        a = O.prunedpp(g, gr, q, 0)
        b = O.dpbf(g, gr, q)
        assert a.cost == b.cost
        assert O.validate(g, gr, q, -1, a.cost, a.root, a.edges) == 0


def test_validator_rejects(oracle_mod):
    O = oracle_mod
    g, gr, qs = gen.config1()
    q = qs[3][0]
    r = O.prunedpp(g, gr, q, 0)
    assert O.validate(g, gr, q, -1, r.cost, r.root, r.edges) == 0
    assert O.validate(g, gr, q, -1, r.cost + 1, r.root, r.edges) == 4
    if len(r.edges) > 1:
        assert O.validate(g, gr, q, -1, r.cost, r.root, r.edges[1:]) != 0
        bad = r.edges.copy()
        bad[0, 2] += 1
        assert O.validate(g, gr, q, -1, r.cost, r.root, bad) == 1


def test_hop_budget_bound_keeps_the_optimum(oracle_mod):
    """The hop-budget bound the engine applies to hop-bounded DP states: a
    state (v, S, d) may be dropped when a group missing from S has no member
    within D - d hops of v, or when its cost plus the largest such distance
    exceeds an upper bound.  Applied with the optimum itself as the upper
    bound (the tightest the engine ever has), HOP_cpu must still reach the
    optimum, and must still find no tree where there is none."""
    O = oracle_mod
    checked = pruned_any = 0
    for i, (g, gr, q) in enumerate(small_cases(30, seed0=700, V=150, E=500, kmax=5)):
        for D in (0, 1, 2, 3, 4):
            ref = O.hop(g, gr, q, D)
            ub = ref.cost if ref.status == 0 else 1 << 40
            st, cost, popped = O.hop_budget(g, gr, q, D, ub)
            if ref.status != 0:
                assert st != 0, (i, D)
                continue
            assert st == 0 and cost == ref.cost, (i, D, ref.cost, st, cost)
            checked += 1
            pruned_any += popped < ref.process
    assert checked >= 50
    assert pruned_any > 0  # the bound does cut states on these instances


def _hop_limited(g, sources, b):
    """Exact cheapest-path costs over paths of at most b hops from a source set
    (Bellman-Ford rounds reading the previous round's values), numpy."""
    INF = np.iinfo(np.int64).max // 4
    d = np.full(g.V, INF, dtype=np.int64)
    d[np.asarray(sources, dtype=np.int64)] = 0
    src = np.repeat(np.arange(g.V), np.diff(g.beg_pos.astype(np.int64)))
    for _ in range(b):
        nd = d.copy()
        cand = d[src] + g.weight.astype(np.int64)
        np.minimum.at(nd, g.csr.astype(np.int64), np.where(d[src] < INF, cand, INF))
        d = nd
    return d, INF


def test_hop_centre_and_star_facts(oracle_mod):
    """The two facts the hop-bounded distance rounds rely on, checked against
    brute force: (1) a tree of hop diameter <= D exists only if some vertex
    has every query group within ceil(D/2) hops (a centre of the tree);
    (2) for every vertex with all groups within floor(D/2) hops, the sum of
    those hop-limited distances is at least the optimum (it spans a feasible
    tree), so its minimum is a valid incumbent."""
    O = oracle_mod
    checked = 0
    for g, gr, q, _ in tiny_cases(200, seed0=7000, kmax=4):
        for D in (2, 3, 4):
            opt = O.brute(g, gr, q, D)
            rows_c = [_hop_limited(g, gr.group(int(j)), (D + 1) // 2) for j in q]
            INF = rows_c[0][1]
            centre = np.all(np.stack([r[0] < INF for r in rows_c]), axis=0).any()
            if opt >= 0:
                assert centre, (q.tolist(), D)
            rows_s = [_hop_limited(g, gr.group(int(j)), D // 2)[0] for j in q]
            st = np.stack(rows_s)
            ok = np.all(st < INF, axis=0)
            if ok.any():
                star = int(st[:, ok].sum(axis=0).min())
                assert opt >= 0 and star >= opt, (q.tolist(), D, star, opt)
            checked += 1
    assert checked == 600
