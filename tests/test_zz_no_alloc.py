"""gst_query_noalloc: the allocation-free query entry point.

Some callers cannot allocate device memory while they answer a query (a host
program that has reserved the GPU's memory for its own pool, or a loop in
which cudaMalloc / cudaFree may not run).  gst_query_noalloc keeps every
per-query buffer in one static device array inside the library.  This test
calls it through the C ABI twice in a row per query (the second call reuses
the array the first one left behind) and checks each result against
gst_query's: costs are integers, so they must be equal, and every tree must
be valid.  The file is named so that pytest collects it last.
"""
import numpy as np
import pytest

from gpugst_b200 import gen

pytestmark = pytest.mark.gpu


def test_noalloc_matches_query(gst_lib, oracle_mod):
    eng, O = gst_lib, oracle_mod
    g, gr, qs = gen.config1()
    E = eng.Engine.from_instance(g, gr)
    rng = np.random.default_rng(17)
    cases = [(q, -1) for q in qs[3][:4]]
    for k in (4, 5):
        cases.append((rng.choice(gr.n_groups, size=k, replace=False).astype(np.uint32), -1))
    cases.append((qs[3][4], 3))
    cases.append((qs[3][5], 4))
    for q, D in cases:
        want = E.query(q, D=D)
        for _ in range(2):  # two calls in a row on the shared scratch
            got = E.query_noalloc(q, D=D)
            assert got.status == want.status, (q, D, got.status, want.status)
            assert got.cost == want.cost, (q, D, got.cost, want.cost)
            if got.ok:
                assert O.validate(g, gr, q, D, got.cost, got.root, got.edges) == 0
    E.close()


def test_noalloc_rejects_oversized_query(gst_lib):
    eng = gst_lib
    g, gr, qs = gen.config1()
    E = eng.Engine.from_instance(g, gr)
    q = np.arange(7, dtype=np.uint32)  # 10,000 x 2^7 x 8 states: an 82 MB state table
    r = E.query_noalloc(q, D=7)
    assert r.status == eng.GST_SCRATCH_TOO_SMALL
    # a fitting query still works afterwards
    r2 = E.query_noalloc(qs[3][0])
    assert r2.ok and r2.cost == E.query(qs[3][0]).cost
    E.close()
