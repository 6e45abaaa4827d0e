"""The oracle restatement reproduces the reference's own programs' costs
(golden fixtures made by running the reference's PrunedDP++ / HOP_cpu
sources, tests/golden/make_golden.py)."""
import numpy as np

from tests import golden_util


def test_golden_fixture_shape():
    gold = golden_util.load()
    assert set(gold["results"]) >= {"c1", "s_k456", "hop", "gstp"}
    n = sum(len(r["cost"]) for res in gold["results"].values() for r in res.values())
    assert n >= 120


def test_oracle_matches_reference_programs(oracle_mod):
    O = oracle_mod
    bad = []
    n = 0
    for name, key, g, gr, q, D, want in golden_util.cases():
        r = O.prunedpp(g, gr, q, 0) if D < 0 else O.hop(g, gr, q, D)
        n += 1
        if want is None:
            if r.status != 1:
                bad.append((name, key, q.tolist(), "want infeasible", r.cost))
        elif r.status != 0 or r.cost != want:
            bad.append((name, key, q.tolist(), want, r.cost))
        elif O.validate(g, gr, q, D, r.cost, r.root, r.edges):
            bad.append((name, key, q.tolist(), "invalid tree"))
    assert n > 0 and not bad, bad[:10]


def test_reference_progressive_exit_defect_recorded():
    """ratio=1 (the reference driver's setting) never beats the exact cost and
    is recorded beside it; it may exceed it (integer-division exit)."""
    gold = golden_util.load()
    for res in gold["results"].values():
        for r in res.values():
            if "cost_ratio1_as_written" in r:
                for a, b, ok in zip(r["cost_ratio1_as_written"], r["cost"], r["feasible"]):
                    if ok:
                        assert a >= b


def test_oracle_matches_reference_at_scale(oracle_mod):
    """The restatement reproduces the reference programs' costs on a sample of
    the benchmark-size instances (golden_scale.json): 2 queries per k on the
    170k-vertex Chung-Lu instance and the hop-bounded queries of the 2^20-vertex
    R-MAT instance that the reference solved in under 5 s.  Also checks that
    the seeded generators still reproduce those instances."""
    import hashlib
    import json
    import os

    from gpugst_b200 import gen
    O = oracle_mod
    with open(os.path.join(golden_util.HERE, "golden_scale.json")) as f:
        gold = json.load(f)

    def fp(g, gr):
        h = hashlib.sha256()
        for a in (g.beg_pos, g.csr, g.weight, gr.ptr, gr.members):
            h.update(np.ascontiguousarray(a).tobytes())
        return h.hexdigest()

    bad = []
    n = 0
    for name in ("c2", "c3"):
        g, gr, _ = gen.config2() if name == "c2" else gen.config3()
        assert fp(g, gr) == gold["fingerprint"][name], name
        for key, r in gold["results"][name].items():
            D = int(key.split("_D")[1]) if "_D" in key else -1
            picked = 0
            for q, c, ok, sec in zip(r["queries"], r["cost"], r["feasible"], r["seconds"]):
                if c is None or picked >= 2 or (D >= 0 and sec > 5.0):
                    continue
                picked += 1
                q = np.array(q, dtype=np.uint32)
                o = O.prunedpp(g, gr, q, 0) if D < 0 else O.hop(g, gr, q, D)
                n += 1
                if not ok:
                    if o.status != 1:
                        bad.append((name, key, q.tolist(), "want infeasible", o.cost))
                elif o.status != 0 or o.cost != c:
                    bad.append((name, key, q.tolist(), c, o.cost))
    assert n >= 12 and not bad, bad


def test_batched_configuration_fixture(oracle_mod):
    """The 3M-vertex batched configuration: the seeded generator reproduces
    the fingerprinted instance, and the restatement agrees with the
    reference's PrunedDP++ on the fixture's quickest unbounded query."""
    import hashlib
    import json
    import os

    from gpugst_b200 import gen
    with open(os.path.join(golden_util.HERE, "golden_scale.json")) as f:
        gold = json.load(f)
    r = gold["results"]["c4"]
    g, gr, qs, Ds = gen.config4()
    h = hashlib.sha256()
    for a in (g.beg_pos, g.csr, g.weight, gr.ptr, gr.members):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == gold["fingerprint"]["c4"]
    cand = [i for i, (D, src) in enumerate(zip(r["D"], r["source"])) if D < 0 and src.startswith("reference")]
    i = min(cand, key=lambda x: r["seconds"][x])
    q = np.array(r["queries"][i], dtype=np.uint32)
    assert (q == qs[r["index"][i]]).all()
    o = oracle_mod.prunedpp(g, gr, q, 0)
    assert o.status == 0 and o.cost == r["cost"][i]
