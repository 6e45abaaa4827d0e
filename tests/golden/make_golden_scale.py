"""Golden costs at the benchmark sizes, from the reference's own CPU programs.

Writes golden_scale.json:
  c2  Chung-Lu V=170,000, E=6.8M (gen.config2): the first 10 queries of each
      k = 3, 4, 5, solved by oracle/_ref/prunedpp_ref (PrunedDP++ of
      code/PrunedDP++/include/CPUNONHOP.h compiled unchanged, exact mode:
      ratio 0 keeps only the exits at CPUNONHOP.h:658-678);
  c3  R-MAT scale 20, E=10M (gen.config3): per cell (k, D), k = 3, 4, 5 and
      D = 2, 3, 4, the first queries of the cell's seeded set, solved by
      oracle/_ref/hop_ref (HOP_cpu of code/D-PrunedDP++/include/CPUHOP.h:107-288
      compiled unchanged).  A query that does not finish within --limit
      seconds is left out and listed under "skipped".

  c4  Chung-Lu V=3,000,000, E=117M (gen.config4, the batched configuration):
      the first 8 unbounded k = 3 and 4 unbounded k = 4 queries of its
      1,024-query set, solved by prunedpp_ref fed raw arrays (--bin: the
      reference's own structures, without the minutes its text parser needs
      at this size), and the first 6 hop-bounded queries with k <= 4, solved
      by the HOP_cpu restatement (oracle.hop; the reference's HOP_cpu has no
      raw-array driver).  Each entry records its source.

Each instance is regenerated by the tests from its seeded spec; the
fingerprint (SHA-256 over the CSR and group arrays) lets a test detect a
generator that no longer reproduces the instance the costs belong to.

Run where oracle/_ref has been built (make -C oracle ref):
    python tests/golden/make_golden_scale.py [--limit 240] [--jobs 8] [--only c2,c3,c4]
"""
import argparse
import concurrent.futures as cf
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gpugst_b200 import formats, gen  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref")
N_C2 = 10        # queries per k on c2
N_C3 = 10        # queries per (k, D) cell on c3


def fingerprint(g, gr) -> str:
    h = hashlib.sha256()
    for a in (g.beg_pos, g.csr, g.weight, gr.ptr, gr.members):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def instance(name):
    """(graph, groups, {key: queries}, {key: D}) of a scale instance."""
    if name == "c2":
        g, gr, qs = gen.config2()
        return g, gr, {f"k{k}": qs[k][:N_C2] for k in (3, 4, 5)}, {f"k{k}": -1 for k in (3, 4, 5)}
    g, gr, qs = gen.config3()
    sel = {f"k{k}_D{D}": qs[(k, D)][:N_C3] for k in (3, 4, 5) for D in (2, 3, 4)}
    return g, gr, sel, {f"k{k}_D{D}": D for k in (3, 4, 5) for D in (2, 3, 4)}


def _hop_one(args):
    """oracle.hop on one c4 query (run in a worker process)."""
    i, q, D = args
    from oracle import oracle
    g, gr, _, _ = _C4
    t0 = time.time()
    r = oracle.hop(g, gr, q, D)
    return i, r.status, r.cost, time.time() - t0


_C4 = None


def make_c4(gold, jobs, limit):
    """The c4 entries (see the module docstring)."""
    global _C4
    import multiprocessing as mp
    g, gr, qs, Ds = gen.config4()
    _C4 = (g, gr, qs, Ds)
    gold["fingerprint"]["c4"] = fingerprint(g, gr)
    un3 = [i for i in range(len(qs)) if Ds[i] < 0 and len(qs[i]) == 3][:8]
    un4 = [i for i in range(len(qs)) if Ds[i] < 0 and len(qs[i]) == 4][:4]
    hop = [i for i in range(len(qs)) if Ds[i] >= 0 and len(qs[i]) <= 4][:6]
    res = {"index": [], "queries": [], "D": [], "cost": [], "feasible": [], "seconds": [], "source": []}
    with tempfile.TemporaryDirectory() as td:
        pre = os.path.join(td, "c4")
        g.beg_pos.astype(np.uint32).tofile(pre + ".beg")
        g.csr.astype(np.uint32).tofile(pre + ".adj")
        g.weight.astype(np.int32).tofile(pre + ".w")
        gr.ptr.astype(np.uint64).tofile(pre + ".gptr")
        gr.members.astype(np.uint32).tofile(pre + ".gv")
        cmds = {}
        for k, idx in ((3, un3), (4, un4)):
            np.array([qs[i] for i in idx], dtype=np.uint32).tofile(f"{pre}.q{k}")
            for r, i in enumerate(idx):
                cmds[i] = [os.path.join(REF_BIN, "prunedpp_ref"), "--bin", pre, str(k), str(r), str(r), "0"]
        with cf.ThreadPoolExecutor(jobs) as ex:
            futs = {ex.submit(run_one, cmd, limit): i for i, cmd in cmds.items()}
            for fu in cf.as_completed(futs):
                i = futs[fu]
                r, wall = fu.result()
                print("c4", i, r, f"{wall:.0f} s", flush=True)
                if r is None:
                    continue
                for key, val in (("index", i), ("queries", qs[i].tolist()), ("D", -1), ("cost", r["cost"]),
                                 ("feasible", r["feasible"]), ("seconds", r["seconds"]),
                                 ("source", "reference PrunedDP++ (prunedpp_ref --bin, exact mode)")):
                    res[key].append(val)
    with mp.get_context("fork").Pool(min(jobs, len(hop))) as pool:
        for i, st, cost, sec in pool.imap_unordered(_hop_one, [(i, qs[i], Ds[i]) for i in hop]):
            print("c4 hop", i, st, cost, f"{sec:.0f} s", flush=True)
            for key, val in (("index", i), ("queries", qs[i].tolist()), ("D", Ds[i]), ("cost", cost if st == 0 else 0),
                             ("feasible", 1 if st == 0 else 0), ("seconds", sec),
                             ("source", "HOP_cpu restatement (oracle.hop)")):
                res[key].append(val)
    gold["results"]["c4"] = res


def run_one(cmd, limit):
    t0 = time.time()
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=limit).stdout
    except subprocess.TimeoutExpired:
        return None, time.time() - t0
    for line in out.splitlines():
        if line.startswith("RESULT "):
            _, i, cost, ok, sec, proc, cnt = line.split()
            return {"cost": int(cost), "feasible": int(ok), "seconds": float(sec)}, time.time() - t0
    raise RuntimeError(f"no RESULT line from {cmd}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--limit", type=float, default=240.0, help="seconds per reference query")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", default="c2,c3")
    args = ap.parse_args()
    path = os.path.join(HERE, "golden_scale.json")
    gold = {"results": {}, "fingerprint": {}, "skipped": {}}
    if os.path.exists(path):
        with open(path) as f:
            gold = json.load(f)
    names = args.only.split(",")
    if "c4" in names:
        make_c4(gold, args.jobs, args.limit)
        names.remove("c4")
    with tempfile.TemporaryDirectory() as td:
        for name in names:
            g, gr, sel, Ds = instance(name)
            gold["fingerprint"][name] = fingerprint(g, gr)
            # one query file per key: <name>_<key><k>.csv, read by the reference drivers
            jobs = {}
            formats.write_in(os.path.join(td, name + ".in"), g)
            formats.write_g(os.path.join(td, name + ".g"), gr)
            for key, q in sel.items():
                k = q.shape[1]
                tag = f"{name}_{key}_"
                formats.write_queries(os.path.join(td, f"{tag}{k}.csv"), q)
                for i in range(len(q)):
                    if Ds[key] < 0:
                        cmd = [os.path.join(REF_BIN, "prunedpp_ref"), td + "/", tag, str(k), str(i), str(i), "0"]
                    else:
                        cmd = [os.path.join(REF_BIN, "hop_ref"), td + "/", tag, str(k), str(Ds[key]), str(i), str(i)]
                    jobs[(key, i)] = cmd
            # the drivers read <path><name>.in / .g: link them under each query file's prefix
            for key in sel:
                for ext in (".in", ".g"):
                    dst = os.path.join(td, f"{name}_{key}_{ext}")
                    if not os.path.exists(dst):
                        os.symlink(os.path.join(td, name + ext), dst)
            res = {key: {"queries": q.tolist(), "cost": [None] * len(q), "feasible": [None] * len(q),
                         "seconds": [None] * len(q)} for key, q in sel.items()}
            skipped = []
            with cf.ThreadPoolExecutor(args.jobs) as ex:
                futs = {ex.submit(run_one, cmd, args.limit): kv for kv, cmd in jobs.items()}
                for fu in cf.as_completed(futs):
                    key, i = futs[fu]
                    r, wall = fu.result()
                    if r is None:
                        skipped.append([key, i])
                        print(name, key, i, f"skipped after {wall:.0f} s", flush=True)
                        continue
                    for fld in ("cost", "feasible", "seconds"):
                        res[key][fld][i] = r[fld]
                    print(name, key, i, r, flush=True)
            gold["results"][name] = res
            gold["skipped"][name] = sorted(skipped)
    with open(path, "w") as f:
        json.dump(gold, f, indent=1)


if __name__ == "__main__":
    main()
