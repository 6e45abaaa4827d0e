#!/usr/bin/env python
"""Benchmark: exact-optimal group Steiner tree queries/s (+ p50/p99 latency),
batched engine vs the plain one-query-at-a-time GPU path.

Workload (default "c2"): Chung-Lu power-law graph, V=170,000, E=6.8M undirected
(13.6M arcs), exponent 2.3, int32 weights uniform in [1,100]; 200,000 groups
with Zipf(1.5) sizes in [1,200]; 300 queries each at k = 3, 4, 5 (seeded
synthetic stand-in for the reference's datasets).  One step = one batch of
--batch queries through gst_query_batch (host buffers in, costs and trees out).

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

N > 1 runs one replica per GPU (queries are independent: each rank takes its
own share of the query stream; no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CACHE = os.environ.get("GSTB_CACHE", "/tmp/gstb_cache")
METRIC = "exact-optimal queries/sec + p50/p99 latency: batched serve vs plain per-query GPU"


def load_workload(name: str):
    from gpugst_b200 import gen
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"{name}.npz")
    if os.path.exists(path):
        z = np.load(path)
        g = gen.Graph(len(z["beg"]) - 1, z["beg"], z["csr"], z["w"])
        gr = gen.Groups(z["gp"], z["gv"])
        qs = {int(k[1:]): z[k] for k in z.files if k.startswith("q")}
        return g, gr, qs
    if name == "c2":
        g, gr, qs = gen.config2()
    elif name == "c1":
        g, gr, qs = gen.config1()
    else:
        raise SystemExit(f"unknown workload {name}")
    np.savez(path, beg=g.beg_pos, csr=g.csr, w=g.weight, gp=gr.ptr, gv=gr.members,
             **{f"q{k}": v for k, v in qs.items()})
    return g, gr, qs


def query_pool(qs):
    """Interleave the per-k query sets: k=3,4,5,3,4,5,..."""
    ks = sorted(qs)
    n = min(len(qs[k]) for k in ks)
    pool = []
    for i in range(n):
        for k in ks:
            pool.append(qs[k][i])
    return pool


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            t = [x.strip() for x in line.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                smax = max(smax, float(t[2]))
            except ValueError:
                continue
            for nm, val in zip(names, t[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Algorithmic bytes of a round, from the device counters (the useful bytes
# each unit of work must move).  The two round kernels share the work types
# (k_light: distance items and DP states; k_heavy: the arc chunks k_light
# hands over and the bound-table rows), so the round is the unit measured.
#   distance item       : 48 B per vertex (item id 4, flags 4, distance row
#                         32, adjacency offsets 8)
#            per arc    : 40 B ({neighbour, weight} 8 + target distance row 32,
#                         whose word 7 holds the pending-group flags)
#            per update / enqueue : 4 B / 8 B (flags 4 + list entry 4)
#   DP state            : 66 B (item id 4, flag 4, state word 8, distance
#                         row 32, complement word 8, bound 2, offsets 8)
#            per arc    : 18 B ({neighbour, weight} 8, target word 8, bound 2)
#            per merge partner : 10 B (word 8, bound 2); update 8 B; enqueue 8 B
#   bound row           : 32 B read + 2 * 2^k B written (one per vertex)
def distance_work_bytes(st):
    return 48 * st["sssp_items"] + 40 * st["sssp_arcs"] + 4 * st["sssp_updates"] + 8 * st["sssp_enqueued"]


def dp_work_bytes(st, V, ks):
    lb_rows = sum(V * (32 + 2 * (1 << k)) for k in ks)
    return (66 * st["expanded"] + 18 * st["arcs"] + 10 * st["merges"] + 8 * st["updates"]
            + 8 * st["enqueued"] + lb_rows)


def traffic_per_byte():
    """DRAM bytes per algorithmic byte of a round (both round kernels), from
    the committed ncu summary (profiles/round_kernel_traffic.json), if present."""
    p = os.path.join(ROOT, "profiles", "round_kernel_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get("dram_bytes_per_algorithmic_byte")


def cpu_baseline_port(g, gr, pool, n_per_k=3):
    """The oracle restatement of PrunedDP++ (exact mode) on one core."""
    from oracle import oracle
    oracle.build()
    sample = []
    seen = {}
    for q in pool:
        k = len(q)
        if seen.get(k, 0) < n_per_k:
            sample.append(q)
            seen[k] = seen.get(k, 0) + 1
    t0 = time.perf_counter()
    for q in sample:
        oracle.prunedpp(g, gr, q, 0)
    dt = time.perf_counter() - t0
    return {"value": len(sample) / dt, "unit": "queries/s", "cores": 1, "kind": "port",
            "sample": f"{len(sample)} queries ({n_per_k} each of k={sorted(seen)}) of the same workload, "
                      f"PrunedDP++ restatement (exact mode), {dt:.1f} s"}


def ref_dataset(name, g, gr, pool):
    """Write the workload in the reference's file formats (cached)."""
    from gpugst_b200 import formats
    d = os.path.join(CACHE, f"ref_{name}")
    if not os.path.exists(os.path.join(d, "done")):
        qs = {}
        for q in pool:
            qs.setdefault(len(q), []).append(q)
        formats.write_dataset(d, name, g, gr, {k: np.array(v) for k, v in qs.items()})
        open(os.path.join(d, "done"), "w").close()
    return d + "/"


def run_reference(args, g, gr, pool, rank, world):
    """--impl reference: the reference's own PrunedDP++ CPU program (oracle/_ref,
    compiled from the reference sources) on all usable host cores, one query per
    core per step; falls back to the oracle restatement when it is absent."""
    if rank != 0:
        return
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "prunedpp_ref")
    nproc = os.cpu_count() or 1
    try:
        import psutil
        mem_workers = int(psutil.virtual_memory().available / (3 << 30))
    except Exception:
        mem_workers = nproc
    workers = max(1, min(nproc, 32, mem_workers))
    steps = args.steps + args.warmup
    if os.path.exists(ref_bin):
        kind = "reference"
        d = ref_dataset(args.workload, g, gr, pool)
        # worker w runs the queries w, w + workers, ... of the k-interleaved pool, grouped by k file
        byk = {}
        for q in pool:
            byk.setdefault(len(q), []).append(q)
        procs = []
        assign = []  # (worker, k, index)
        for w in range(workers):
            ks = sorted(byk)
            k = ks[w % len(ks)]
            base = (w // len(ks)) * steps
            assign.append((k, base))
            procs.append(subprocess.Popen([ref_bin, d, args.workload, str(k), str(base), str(base + steps - 1), "0"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
        per = []
        for p in procs:
            out, _ = p.communicate()
            secs = [float(line.split()[4]) for line in out.splitlines() if line.startswith("RESULT ")]
            per.append(secs)
        step_times = []
        for s in range(args.warmup, steps):
            step_times.append(max(x[s] for x in per if len(x) > s))
        nq = workers * args.steps
        total = sum(step_times)
        sample = (f"{args.steps} steps x {workers} concurrent processes (one query each; k cycles 3,4,5); "
                  f"step time = slowest process's query time; graph load excluded")
    else:
        kind = "port"
        from oracle import oracle
        oracle.build()
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        total = 0.0
        nq = 0
        with ctx.Pool(workers, initializer=_ref_init, initargs=(args.workload,)) as pool_ex:
            for s in range(steps):
                batch = [pool[(s * workers + i) % len(pool)] for i in range(workers)]
                t0 = time.perf_counter()
                pool_ex.map(_ref_one, batch)
                dt = time.perf_counter() - t0
                if s >= args.warmup:
                    total += dt
                    nq += len(batch)
        sample = f"{args.steps} steps x {workers} queries in parallel processes (oracle restatement)"
    value = nq / total
    line = {"metric": METRIC, "value": value, "unit": "queries/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": {"workload": workload_desc(args.workload)},
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": workers, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


_REF_STATE = {}


def _ref_init(name):
    g, gr, _ = load_workload(name)
    _REF_STATE["g"], _REF_STATE["gr"] = g, gr


def _ref_one(q):
    from oracle import oracle
    return oracle.prunedpp(_REF_STATE["g"], _REF_STATE["gr"], q, 0).cost


def workload_desc(name):
    if name == "c2":
        return ("chung-lu V=170000 E=6.8M gamma=2.3 w~U[1,100]; 200000 zipf(1.5) groups in [1,200]; "
                "queries k=3,4,5 interleaved (300 each)")
    return name


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--batch", type=int, default=90, help="queries per step")
    ap.add_argument("--plain", type=int, default=30, help="queries timed on the plain per-query path")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve", type=int, default=360, help="queries through the serving loop")
    ap.add_argument("--inflight", type=int, default=32, help="serving loop concurrency")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    g, gr, qs = load_workload(args.workload)
    pool = query_pool(qs)

    if args.impl == "reference":
        run_reference(args, g, gr, pool, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from gpugst_b200 import build, engine, replicas
    build.build()
    E = engine.Engine.from_instance(g, gr)

    B = args.batch
    # this rank's share of the query stream
    def batch_for(step):
        base = (rank * (args.steps + args.warmup) + step) * B
        return [pool[(base + i) % len(pool)] for i in range(B)]

    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for s in range(args.warmup):
        E.query_batch(batch_for(s))
    torch.cuda.synchronize()

    h2d = d2h = 0
    dev_ms, wall_ms, lat = [], [], []
    n_ok = 0
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = E.kernel_launches()
    sampler.start()
    for s in range(args.steps):
        l2_flush.fill_(s & 0xFF)  # write > L2 between steps
        torch.cuda.synchronize()
        qb = batch_for(args.warmup + s)
        t0 = time.perf_counter()
        res = E.query_batch(qb)
        wall_ms.append(1e3 * (time.perf_counter() - t0))
        dev_ms.append(res[0].device_ms)
        lat.extend(r.latency_ms for r in res)
        n_ok += sum(r.status in (engine.GST_OK, engine.GST_NO_SOLUTION) for r in res)
        members = sum(int(gr.ptr[q[i] + 1] - gr.ptr[q[i]]) for q in qb for i in range(len(q)))
        h2d += 4 * members + 8 * 4 * len(qb)
        d2h += sum(12 * len(r.edges) + 64 for r in res)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = E.kernel_launches() - launches0
    if dist:
        dist.barrier()

    tot_dev = sum(dev_ms)
    tot_wall = sum(wall_ms)
    tot_dev, tot_wall = replicas.max_over_ranks([tot_dev, tot_wall], device="cuda")
    nq_all = B * args.steps * world
    value = nq_all / (tot_dev / 1e3)
    e2e_value = nq_all / (tot_wall / 1e3)

    # profiled pass (not timed): round-kernel device time and counters for the roofline
    E.profile(True)
    E.profile_reset()
    prof_batch = batch_for(args.warmup)
    E.query_batch(prof_batch)
    light_ms, heavy_ms, prof_rounds, st = E.profile_read()
    E.profile(False)
    dist_bytes = distance_work_bytes(st)
    dp_bytes = dp_work_bytes(st, g.V, [len(q) for q in prof_batch])
    peak, peak_kind = measured_peak_hbm()
    round_ms = light_ms + heavy_ms
    round_bytes = dist_bytes + dp_bytes
    achieved = round_bytes / (round_ms / 1e3) / 1e9 if round_ms > 0 else 0.0
    tpb = traffic_per_byte()
    per_round_alg = round_bytes / max(prof_rounds, 1)

    # continuous-batching serving loop (closed loop, `--inflight` requests on the device)
    n_serve = args.serve
    S = engine.Server(E, max_inflight=args.inflight) if n_serve > 0 else None
    serve_q = [pool[(rank * 104729 + 7 * i) % len(pool)] for i in range(n_serve)]
    lat_serve = []
    t0 = time.perf_counter()
    nxt = 0
    for nxt in range(min(args.inflight, n_serve)):
        S.submit(nxt, serve_q[nxt])
    nxt = min(args.inflight, n_serve)
    done = 0
    while done < n_serve:
        got = S.poll()
        if not got:
            time.sleep(0.0002)
            continue
        for rid, r in got:
            lat_serve.append(r.latency_ms)
            done += 1
            if nxt < n_serve:
                S.submit(nxt, serve_q[nxt])
                nxt += 1
    serve_wall = time.perf_counter() - t0
    if S is not None:
        S.close()
    serve_qps = n_serve / serve_wall if n_serve > 0 else None

    # plain per-query path (one query per call, gst_query), same workload
    plain_lat, plain_dev = [], []
    for i in range(args.plain):
        q = pool[(rank * 7919 + i * 13) % len(pool)]
        t0 = time.perf_counter()
        r = E.query(q)
        plain_lat.append(1e3 * (time.perf_counter() - t0))
        plain_dev.append(r.device_ms)
    plain_qps = len(plain_lat) / (sum(plain_lat) / 1e3) if plain_lat else None

    def pct(xs, p):
        return float(np.percentile(np.array(xs), p)) if xs else None

    out = None
    if rank == 0:
        cpu = None if args.no_cpu else cpu_baseline_port(g, gr, pool)
        out = {
            "metric": METRIC,
            "value": value,
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": tot_dev / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int32",
            "data": "synthetic",
            "config": {"workload": workload_desc(args.workload), "batch_queries_per_step": B,
                       "parallelism": f"replicas x{world}", "l2": "256 MB buffer written between steps",
                       "queries_ok": n_ok},
            "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps},
            "latency_ms": {"batched_p50": pct(lat, 50), "batched_p99": pct(lat, 99),
                           "plain_p50": pct(plain_lat, 50), "plain_p99": pct(plain_lat, 99)},
            "plain_per_query": {"value": plain_qps, "unit": "queries/s", "queries": len(plain_lat),
                                "device_ms_p50": pct(plain_dev, 50)},
            "batched_vs_plain": value / plain_qps if plain_qps else None,
            "serve_vs_plain": serve_qps / plain_qps if (plain_qps and serve_qps) else None,
            "serve": {"value": serve_qps, "unit": "queries/s", "inflight": args.inflight, "queries": n_serve,
                      "p50_ms": pct(lat_serve, 50), "p99_ms": pct(lat_serve, 99)},
            "roofline": {"bound": "hbm", "kernel": "round (k_light + k_heavy)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (per_round_alg * tpb) if tpb else None,
                         "algorithmic_bytes_per_round": per_round_alg, "rounds": prof_rounds,
                         "kernel_ms": {"k_light": light_ms, "k_heavy": heavy_ms},
                         "algorithmic_bytes": {"distance": dist_bytes, "dp": dp_bytes}},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": int(launches),
        }
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    E.close()


if __name__ == "__main__":
    main()
