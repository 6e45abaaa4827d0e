"""GPU costs at the benchmark sizes equal the reference programs' own costs.

golden_scale.json (tests/golden/make_golden_scale.py) holds costs computed by
the reference's PrunedDP++ (exact mode) on the 170k-vertex / 6.8M-edge
Chung-Lu instance and by its HOP_cpu on the 2^20-vertex / 10M-edge R-MAT
instance.  The instances are regenerated here from their seeds and checked
against the recorded fingerprints first.  Every GPU cost must equal the
reference's cost bit for bit, every returned tree must pass the validator,
and the plain (gst_query) and batched (gst_query_batch) paths must agree.

Also k = 7, the largest query the ABI accepts, against brute force."""
import json
import os

import numpy as np
import pytest

from gpugst_b200 import gen
from tests.cases import tiny_cases

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _gold():
    with open(os.path.join(HERE, "golden_scale.json")) as f:
        return json.load(f)


def _fingerprint(g, gr):
    import hashlib
    h = hashlib.sha256()
    for a in (g.beg_pos, g.csr, g.weight, gr.ptr, gr.members):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _cases(gold, name):
    """(key, query, D, golden cost or None if infeasible) of every recorded query."""
    out = []
    for key, r in gold["results"][name].items():
        D = int(key.split("_D")[1]) if "_D" in key else -1
        for q, c, ok in zip(r["queries"], r["cost"], r["feasible"]):
            if c is None:  # the reference did not finish within its time limit
                continue
            out.append((key, np.array(q, dtype=np.uint32), D, c if ok else None))
    return out


def _check(eng, O, g, gr, cases, results, tag):
    bad = []
    for (key, q, D, want), r in zip(cases, results):
        if want is None:
            if r.status != eng.GST_NO_SOLUTION:
                bad.append((tag, key, q.tolist(), "want no solution", r.status, r.cost))
        elif r.status != eng.GST_OK or r.cost != want:
            bad.append((tag, key, q.tolist(), want, r.status, r.cost))
        elif O.validate(g, gr, q, D, r.cost, r.root, r.edges):
            bad.append((tag, key, q.tolist(), "invalid tree"))
    return bad


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_scale_matches_reference(gst_lib, oracle_mod, name):
    eng, O = gst_lib, oracle_mod
    gold = _gold()
    if name == "c2":
        g, gr, _ = gen.config2()
    else:
        g, gr, _ = gen.config3()
    assert _fingerprint(g, gr) == gold["fingerprint"][name], "generator no longer reproduces the instance"
    cases = _cases(gold, name)
    assert len(cases) >= 30
    E = eng.Engine.from_instance(g, gr)
    try:
        batch = E.query_batch([c[1] for c in cases], [c[2] for c in cases])
        plain = [E.query(q, D=D) for _, q, D, _ in cases]
    finally:
        E.close()
    bad = _check(eng, O, g, gr, cases, batch, "batch") + _check(eng, O, g, gr, cases, plain, "plain")
    assert not bad, bad[:10]


def test_k7_vs_brute(gst_lib, oracle_mod):
    """k = 7 query groups on tiny graphs (unbounded and hop-bounded) against
    brute force over edge subsets."""
    eng, O = gst_lib, oracle_mod
    bad = []
    n = 0
    for i, (g, gr, _, D) in enumerate(tiny_cases(60, seed0=5000, vmax=10, emax=16)):
        # seven distinct groups of the instance (it has six from the generator: add one)
        ptr = np.concatenate([gr.ptr, [gr.ptr[-1] + 1]]).astype(np.uint64)
        mem = np.concatenate([gr.members, [np.uint32(i % g.V)]]).astype(np.uint32)
        gr7 = gen.Groups(ptr, mem)
        q = np.arange(7, dtype=np.uint32)
        E = eng.Engine.from_instance(g, gr7)
        for DD in (-1, D):
            want = O.brute(g, gr7, q, DD)
            r = E.query(q, D=DD)
            n += 1
            if want < 0:
                if r.status != eng.GST_NO_SOLUTION:
                    bad.append((i, DD, "want no solution", r.status, r.cost))
            elif r.status != eng.GST_OK or r.cost != want:
                bad.append((i, DD, want, r.status, r.cost))
            elif O.validate(g, gr7, q, DD, r.cost, r.root, r.edges):
                bad.append((i, DD, "invalid tree"))
        E.close()
    assert n == 120 and not bad, bad[:10]


def test_k7_small_vs_oracle(gst_lib, oracle_mod):
    """k = 7 on 300-vertex instances against the PrunedDP++ restatement and
    the HOP_cpu restatement."""
    eng, O = gst_lib, oracle_mod
    bad = []
    for seed in range(8):
        g, gr = gen.small_instance(300, 1500, n_groups=40, smax=6, seed=700 + seed)
        rng = np.random.default_rng(seed)
        q = rng.choice(gr.n_groups, size=7, replace=False).astype(np.uint32)
        E = eng.Engine.from_instance(g, gr)
        for D in (-1, 3, 4):
            want = O.prunedpp(g, gr, q, 0) if D < 0 else O.hop(g, gr, q, D)
            r = E.query(q, D=D)
            if want.status != 0:
                if r.status != eng.GST_NO_SOLUTION:
                    bad.append((seed, D, "want no solution", r.status))
            elif r.status != eng.GST_OK or r.cost != want.cost:
                bad.append((seed, D, want.cost, r.status, r.cost))
            elif O.validate(g, gr, q, D, r.cost, r.root, r.edges):
                bad.append((seed, D, "invalid tree"))
        E.close()
    assert not bad, bad


def test_batched_configuration_matches_reference(gst_lib, oracle_mod):
    """The 3M-vertex / 117M-edge batched configuration: unbounded queries
    against the reference's own PrunedDP++ and hop-bounded ones against the
    HOP_cpu restatement (golden_scale.json "c4"), through the batched and the
    plain path, every tree validated."""
    eng, O = gst_lib, oracle_mod
    gold = _gold()
    if "c4" not in gold["results"]:
        pytest.skip("no c4 entries in golden_scale.json")
    g, gr, _, _ = gen.config4()
    assert _fingerprint(g, gr) == gold["fingerprint"]["c4"], "generator no longer reproduces the instance"
    r = gold["results"]["c4"]
    cases = [("c4", np.array(q, dtype=np.uint32), D, c if ok else None)
             for q, D, c, ok in zip(r["queries"], r["D"], r["cost"], r["feasible"])]
    assert len(cases) >= 12
    E = eng.Engine.from_instance(g, gr)
    try:
        batch = E.query_batch([c[1] for c in cases], [c[2] for c in cases])
        plain = [E.query(q, D=D) for _, q, D, _ in cases]
    finally:
        E.close()
    bad = _check(eng, O, g, gr, cases, batch, "batch") + _check(eng, O, g, gr, cases, plain, "plain")
    assert not bad, bad[:10]
