"""Loads the golden fixtures produced by tests/golden/make_golden.py."""
import json
import os

import numpy as np

from gpugst_b200 import gen

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load():
    with open(os.path.join(HERE, "golden_ref.json")) as f:
        return json.load(f)


def instance(spec):
    if spec["kind"] == "config1":
        g, gr, qs = gen.config1()
        return g, gr
    g, gr = gen.small_instance(spec["V"], spec["E"], spec["n_groups"], spec["smax"], spec["seed"])
    return g, gr


def gstp_instance():
    z = np.load(os.path.join(HERE, "simple_iterative_tests.npz"))
    g = gen.Graph(len(z["beg_pos"]) - 1, z["beg_pos"], z["csr"], z["weight"])
    gr = gen.Groups(z["grp_ptr"], z["grp_v"])
    return g, gr, z["query"]


def cases():
    """Yield (name, key, graph, groups, query, D, golden cost or None if infeasible)."""
    gold = load()
    for name, res in gold["results"].items():
        if name == "gstp":
            g, gr, _ = gstp_instance()
        else:
            g, gr = instance(gold["specs"][name])
        for key, r in res.items():
            D = int(key.split("_D")[1]) if "_D" in key else -1
            for q, c, ok in zip(r["queries"], r["cost"], r["feasible"]):
                yield name, key, g, gr, np.array(q, dtype=np.uint32), D, (c if ok else None)
