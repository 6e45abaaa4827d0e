"""Generate the golden fixtures by running the reference's own CPU programs.

oracle/_ref/prunedpp_ref and oracle/_ref/hop_ref are the reference's
PrunedDP++ (code/PrunedDP++/include/CPUNONHOP.h) and HOP_cpu
(code/D-PrunedDP++/include/CPUHOP.h) compiled unchanged from the reference
tree (see oracle/Makefile).  This script writes seeded instances in the
reference's file formats, runs those programs, and stores their costs in
golden_ref.json.  It also converts the reference's GSTP fixture
(code/GPUGST/simple_iterative_tests.text) into simple_iterative_tests.npz.

Run here (where the reference tree exists):  python tests/golden/make_golden.py
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gpugst_b200 import formats, gen  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref")
# the reference tree: GSTB_REFERENCE_ROOT when set, else its mount point here
REF_ROOT = os.environ.get("GSTB_REFERENCE_ROOT", "/root/reference")
GSTP = os.path.join(REF_ROOT, "code", "GPUGST", "simple_iterative_tests.text")

# instance name -> generator spec (regenerated identically by the tests)
SPECS = {
    "c1": {"kind": "config1"},
    "s_k456": {"kind": "small", "V": 2000, "E": 12000, "n_groups": 300, "smax": 10, "seed": 21,
               "queries": {"4": [15, 41], "5": [10, 51], "6": [6, 61]}},
    "hop": {"kind": "small", "V": 800, "E": 3200, "n_groups": 150, "smax": 6, "seed": 31,
            "queries": {"3": [10, 71], "4": [6, 81]}, "D": [2, 3, 4]},
}


def instance(spec):
    if spec["kind"] == "config1":
        g, gr, qs = gen.config1()
        return g, gr, {3: qs[3]}
    g, gr = gen.small_instance(spec["V"], spec["E"], spec["n_groups"], spec["smax"], spec["seed"])
    qs = {int(k): gen.queries(gr.n_groups, n, int(k), seed=s) for k, (n, s) in spec["queries"].items()}
    return g, gr, qs


def run(cmd):
    out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
    rows = {}
    for line in out.splitlines():
        if line.startswith("RESULT "):
            _, i, cost, ok, sec, proc, cnt = line.split()
            rows[int(i)] = {"cost": int(cost), "feasible": int(ok), "seconds": float(sec), "process": int(proc)}
    return rows


def main():
    gold = {"specs": SPECS, "results": {}}
    with tempfile.TemporaryDirectory() as td:
        for name, spec in SPECS.items():
            g, gr, qs = instance(spec)
            formats.write_dataset(td, name, g, gr, qs)
            res = {}
            for k, q in qs.items():
                n = len(q)
                if "D" in spec:
                    for D in spec["D"]:
                        r = run([os.path.join(REF_BIN, "hop_ref"), td + "/", name, str(k), str(D), "0", str(n - 1)])
                        res[f"k{k}_D{D}"] = {"queries": q.tolist(), "cost": [r[i]["cost"] for i in range(n)],
                                             "feasible": [r[i]["feasible"] for i in range(n)]}
                else:
                    r0 = run([os.path.join(REF_BIN, "prunedpp_ref"), td + "/", name, str(k), "0", str(n - 1), "0"])
                    r1 = run([os.path.join(REF_BIN, "prunedpp_ref"), td + "/", name, str(k), "0", str(n - 1), "1"])
                    res[f"k{k}"] = {"queries": q.tolist(),
                                    "cost": [r0[i]["cost"] for i in range(n)],
                                    "feasible": [r0[i]["feasible"] for i in range(n)],
                                    "cost_ratio1_as_written": [r1[i]["cost"] for i in range(n)]}
            gold["results"][name] = res
            print(name, {k: v["cost"][:6] for k, v in res.items()}, flush=True)
        if os.path.exists(GSTP):
            g, gr, q = formats.read_gstp(GSTP)
            np.savez_compressed(os.path.join(HERE, "simple_iterative_tests.npz"), beg_pos=g.beg_pos, csr=g.csr,
                                weight=g.weight, grp_ptr=gr.ptr, grp_v=gr.members, query=q)
            formats.write_dataset(td, "gstp", g, gr, {len(q): q[None, :]})
            r0 = run([os.path.join(REF_BIN, "prunedpp_ref"), td + "/", "gstp", str(len(q)), "0", "0", "0"])
            r1 = run([os.path.join(REF_BIN, "prunedpp_ref"), td + "/", "gstp", str(len(q)), "0", "0", "1"])
            gold["results"]["gstp"] = {f"k{len(q)}": {"queries": [q.tolist()], "cost": [r0[0]["cost"]],
                                                      "feasible": [r0[0]["feasible"]],
                                                      "cost_ratio1_as_written": [r1[0]["cost"]]}}
            print("gstp", r0, r1)
    with open(os.path.join(HERE, "golden_ref.json"), "w") as f:
        json.dump(gold, f, indent=1)


if __name__ == "__main__":
    main()
