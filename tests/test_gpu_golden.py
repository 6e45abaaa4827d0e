"""GPU costs equal the reference programs' costs on every golden case."""
import pytest

from tests import golden_util

pytestmark = pytest.mark.gpu


def test_gpu_matches_golden(gst_lib, oracle_mod):
    eng, O = gst_lib, oracle_mod
    bad = []
    cache = {}
    n = 0
    for name, key, g, gr, q, D, want in golden_util.cases():
        if name not in cache:
            cache[name] = eng.Engine.from_instance(g, gr)
        E = cache[name]
        r = E.query(q, D=D)
        n += 1
        if want is None:
            if r.status != eng.GST_NO_SOLUTION:
                bad.append((name, key, q.tolist(), "want no solution", r.status, r.cost))
        elif r.status != eng.GST_OK or r.cost != want:
            bad.append((name, key, q.tolist(), want, r.status, r.cost))
        elif O.validate(g, gr, q, D, r.cost, r.root, r.edges):
            bad.append((name, key, q.tolist(), "invalid tree"))
    for E in cache.values():
        E.close()
    assert n >= 120 and not bad, bad[:10]
