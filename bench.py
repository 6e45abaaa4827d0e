#!/usr/bin/env python
"""Benchmark: exact-optimal group Steiner tree queries/s with p50/p99 latency,
batched engine and continuous-batching serving loop vs the plain
one-query-at-a-time GPU path.

Workloads (seeded synthetic stand-ins for the reference's datasets):
  c4 (default, the batched configuration): Chung-Lu power-law graph,
     V=3,000,000, E=117M undirected (234M arcs), exponent 2.1, int32 weights
     uniform in [1,100]; 1,000,000 groups with Zipf(1.3) sizes in [1,500]; a
     set of 1,024 queries with k uniform in {3,4,5,6}, half of them with a hop
     bound D uniform in {2,3,4}.  One step = one gst_query_batch call over
     --batch queries taken in order from that set (cycling), host buffers in,
     costs and trees out.  The open-loop serving configuration (c5: the same
     graph, Poisson arrivals) is measured in the same run.
  c2: Chung-Lu V=170,000, E=6.8M (13.6M arcs), exponent 2.3; 200,000 groups
     with Zipf(1.5) sizes in [1,200]; 300 queries each at k = 3, 4, 5.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                  [--workload c4|c2]

N > 1 runs one replica per GPU (queries are independent: each rank answers
its own share of the query stream; no collective on the data path).
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


# ---------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------

def load_workload(name: str):
    """(graph, groups, queries, Ds): the workload's query list in bench order."""
    from gpugst_b200 import gen
    os.makedirs(CACHE, exist_ok=True)
    path = os.path.join(CACHE, f"{name}.npz")
    if os.path.exists(path):
        z = np.load(path)
        g = gen.Graph(len(z["beg"]) - 1, z["beg"], z["csr"], z["w"])
        gr = gen.Groups(z["gp"], z["gv"])
        qs = [row[:k].astype(np.uint32) for row, k in zip(z["qs"], z["ks"])]
        return g, gr, qs, [int(d) for d in z["Ds"]]
    if name == "c4":
        g, gr, qs, Ds = gen.config4()
    elif name == "c4s":
        g, gr, qs, Ds = gen.config4_small()
    elif name in ("c1", "c2"):
        g, gr, per_k = gen.config1() if name == "c1" else gen.config2()
        ks = sorted(per_k)
        n = min(len(per_k[k]) for k in ks)
        qs = [per_k[k][i] for i in range(n) for k in ks]  # k = 3, 4, 5, 3, 4, 5, ...
        Ds = [-1] * len(qs)
    else:
        raise SystemExit(f"unknown workload {name}")
    rows = np.zeros((len(qs), 8), dtype=np.uint32)
    for i, q in enumerate(qs):
        rows[i, :len(q)] = q
    np.savez(path, beg=g.beg_pos, csr=g.csr, w=g.weight, gp=gr.ptr, gv=gr.members, qs=rows,
             ks=np.array([len(q) for q in qs]), Ds=np.array(Ds))
    return g, gr, qs, Ds


def workload_desc(name):
    if name == "c4":
        return ("chung-lu V=3000000 E=117M gamma=2.1 w~U[1,100]; 1000000 zipf(1.3) groups in [1,500]; "
                "1024 queries k~U{3..6}, half with D~U{2,3,4}")
    if name == "c4s":
        return ("chung-lu V=1000000 E=39M gamma=2.1 w~U[1,100]; 333333 zipf(1.3) groups in [1,500]; "
                "1024 queries k~U{3..6}, half with D~U{2,3,4} (the batched configuration at a third of its size)")
    if name == "c2":
        return ("chung-lu V=170000 E=6.8M gamma=2.3 w~U[1,100]; 200000 zipf(1.5) groups in [1,200]; "
                "queries k=3,4,5 interleaved (300 each)")
    return name


# ---------------------------------------------------------------------------
# Measurement helpers
# ---------------------------------------------------------------------------

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


def pct(xs, p):
    return float(np.percentile(np.array(xs), p)) if len(xs) else None


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


def dp_work_bytes(st, lb_rows_bytes):
    return (66 * st["expanded"] + 18 * st["arcs"] + 10 * st["merges"] + 8 * st["updates"]
            + 8 * st["enqueued"] + lb_rows_bytes)


def traffic_per_byte():
    """DRAM bytes per algorithmic byte of a round (both round kernels), from
    the committed ncu summary (profiles/round_kernel_traffic.json), if present."""
    p = os.path.join(ROOT, "profiles", "round_kernel_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get("dram_bytes_per_algorithmic_byte")


# ---------------------------------------------------------------------------
# CPU baseline (oracle restatement) -- run before CUDA is initialised so the
# worker processes can be forked with the graph shared copy-on-write
# ---------------------------------------------------------------------------

_CPU = {}


def _cpu_one(i):
    from oracle import oracle
    q, D = _CPU["qs"][i], _CPU["Ds"][i]
    t0 = time.perf_counter()
    r = oracle.prunedpp(_CPU["g"], _CPU["gr"], q, 0) if D < 0 else oracle.hop(_CPU["g"], _CPU["gr"], q, D)
    return i, r.status, r.cost, time.perf_counter() - t0


def cpu_baseline_port(g, gr, qs, Ds, workload):
    """The PrunedDP++ restatement (exact mode; HOP_cpu restatement for
    hop-bounded queries) on a bounded sample of the workload: one query per
    host core, all cores in parallel.  Returns (cpu_baseline dict, {query
    index: (status, cost)}) -- the costs are the bench's parity check."""
    import multiprocessing as mp
    from oracle import oracle
    oracle.build()
    cores = max(1, min(os.cpu_count() or 1, 32))
    if workload in ("c4", "c4s"):
        # unbounded k = 3 queries: the restatement takes about 30 s each on
        # this graph (k = 6 takes minutes)
        sample = [i for i in range(len(qs)) if Ds[i] < 0 and len(qs[i]) == 3][:cores]
    else:
        sample = list(range(min(len(qs), 3 * cores)))
    _CPU.update(g=g, gr=gr, qs=qs, Ds=Ds)
    t0 = time.perf_counter()
    with mp.get_context("fork").Pool(cores) as pool:
        out = pool.map(_cpu_one, sample, chunksize=1)
    wall = time.perf_counter() - t0
    costs = {i: (st, c) for i, st, c, _ in out}
    busy = sum(x[3] for x in out)
    return ({"value": len(sample) / wall, "unit": "queries/s", "cores": cores, "kind": "port",
             "sample": f"{len(sample)} queries of the workload (k in {sorted(set(len(qs[i]) for i in sample))}, "
                       f"{sum(Ds[i] >= 0 for i in sample)} hop-bounded), PrunedDP++ / HOP_cpu restatement in exact "
                       f"mode, one query per process on {cores} cores; {wall:.1f} s wall, {busy:.1f} s busy"},
            costs)


# ---------------------------------------------------------------------------
# Reference arm: the reference's own PrunedDP++ program (oracle/_ref)
# ---------------------------------------------------------------------------

def ref_dataset(name, g, gr, qs, Ds):
    """The workload as raw arrays for the reference driver's binary mode
    (oracle/ref_driver_nonhop.cpp --bin: the reference's own graph and group
    structures filled from arrays instead of parsed text; on the 3M-vertex
    graph the text files take minutes to write and the reference's parser
    over a minute to read).  Queries: the unbounded ones, one file per k."""
    d = os.path.join(CACHE, f"refbin_{name}")
    pre = os.path.join(d, name)
    if not os.path.exists(os.path.join(d, "done")):
        os.makedirs(d, exist_ok=True)
        g.beg_pos.astype(np.uint32).tofile(pre + ".beg")
        g.csr.astype(np.uint32).tofile(pre + ".adj")
        g.weight.astype(np.int32).tofile(pre + ".w")
        gr.ptr.astype(np.uint64).tofile(pre + ".gptr")
        gr.members.astype(np.uint32).tofile(pre + ".gv")
        byk = {}
        for q, D in zip(qs, Ds):
            if D < 0:
                byk.setdefault(len(q), []).append(q)
        for k, v in byk.items():
            np.array(v, dtype=np.uint32).tofile(f"{pre}.q{k}")
        open(os.path.join(d, "done"), "w").close()
    return pre


def run_reference(args, g, gr, qs, Ds, rank, world):
    """--impl reference: the reference's own PrunedDP++ CPU program
    (oracle/_ref/prunedpp_ref, compiled from the reference sources) on the
    workload's unbounded queries, one long-lived process per host core, each
    answering its own queries one after another (the reference's per-query
    loop, exp_CPU_nonHop.h:97-138).  Throughput = all timed queries / the
    busiest process's summed query time.  On the 3M-vertex workload one
    query takes the reference about two minutes, so each process answers one
    k = 3 query there (K and W of the GPU arm's step loop do not apply); on
    the smaller workloads each process answers W warm-up and K timed
    queries."""
    if rank != 0:
        return
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "prunedpp_ref")
    if not os.path.exists(ref_bin):
        raise SystemExit("oracle/_ref/prunedpp_ref missing: build it with make -C oracle ref")
    nproc = os.cpu_count() or 1
    big = args.workload in ("c4", "c4s")
    try:
        import psutil
        per_proc = (6 << 30) if big else (3 << 30)  # peak RSS of one process: about 4 GB on the 3M-vertex graph
        mem_workers = int(psutil.virtual_memory().available / per_proc)
    except Exception:
        mem_workers = nproc
    workers = max(1, min(nproc, 32, mem_workers))
    warm, timed = (0, 1) if big else (args.warmup, args.steps)
    steps = warm + timed
    pre = ref_dataset(args.workload, g, gr, qs, Ds)
    byk = {}
    for q, D in zip(qs, Ds):
        if D < 0:
            byk.setdefault(len(q), []).append(q)
    ks = [3] if big else sorted(byk)
    procs = []
    for w in range(workers):
        k = ks[w % len(ks)]
        base = ((w // len(ks)) * steps) % max(1, len(byk[k]) - steps + 1)
        procs.append(subprocess.Popen([ref_bin, "--bin", pre, str(k), str(base), str(base + steps - 1), "0"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
    per = []
    for p in procs:
        out, _ = p.communicate()
        per.append([float(line.split()[4]) for line in out.splitlines() if line.startswith("RESULT ")])
    done = [x[warm:steps] for x in per]
    nq = sum(len(x) for x in done)
    busy_max = max(sum(x) for x in done)
    value = nq / busy_max
    sample = (f"{workers} processes x {timed} timed queries each (k = {ks}) after {warm} warm-up queries; "
              f"throughput = all timed queries / the busiest process's summed query time; graph load excluded")
    line = {"metric": METRIC, "value": value, "unit": "queries/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * busy_max / max(timed, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": {"workload": workload_desc(args.workload),
                                            "queries": "the workload's unbounded queries (PrunedDP++ has no hop bound)"},
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": workers, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU legs
# ---------------------------------------------------------------------------

def closed_loop(eng, E, reqs, inflight, ratio=0.0):
    """Serve reqs [(q, D)] keeping `inflight` on the device: (q/s, latencies ms, statuses)."""
    S = eng.Server(E, max_inflight=inflight)
    lat, sts = [], []
    n = len(reqs)
    t0 = time.perf_counter()
    for i in range(min(inflight, n)):
        S.submit(i, reqs[i][0], reqs[i][1], ratio=ratio)
    nxt = min(inflight, n)
    done = 0
    while done < n:
        got = S.poll()
        if not got:
            time.sleep(0.0002)
            continue
        for rid, r in got:
            lat.append(r.latency_ms)
            sts.append(r.status)
            done += 1
            if nxt < n:
                S.submit(nxt, reqs[nxt][0], reqs[nxt][1], ratio=ratio)
                nxt += 1
    wall = time.perf_counter() - t0
    S.close()
    return n / wall, lat, sts


def open_loop(eng, E, reqs, rate, seconds, seed, max_pending, drain_s):
    """Poisson arrivals at `rate` q/s for `seconds`: every arrival is submitted
    at its time (GST_BUSY beyond max_pending pending requests: shed).  After
    the arrival window the server gets drain_s more seconds; what is still
    unfinished then is withdrawn with gst_serve_cancel."""
    from gpugst_b200 import gen
    arr = gen.poisson_arrivals(rate, seconds, seed)
    S = eng.Server(E)
    S.set_max_pending(max_pending)
    shed, results = 0, {}
    t0 = time.perf_counter()
    i = 0
    while i < len(arr) or time.perf_counter() - t0 < seconds:
        now = time.perf_counter() - t0
        while i < len(arr) and arr[i] <= now:
            q, D = reqs[i % len(reqs)]
            if S.submit(i, q, D) == eng.GST_BUSY:
                shed += 1
            i += 1
        for rid, r in S.poll():
            results[rid] = r
        time.sleep(0.0005)
    t_end = time.perf_counter() - t0
    submitted = len(arr) - shed
    while len(results) < submitted and time.perf_counter() - t0 < t_end + drain_s:
        for rid, r in S.poll():
            results[rid] = r
        time.sleep(0.001)
    t_drain = time.perf_counter() - t0
    for rid in range(len(arr)):
        if rid not in results:
            S.cancel(rid)
    t1 = time.perf_counter()
    while len(results) < submitted and time.perf_counter() - t1 < 60:
        for rid, r in S.poll():
            results[rid] = r
        time.sleep(0.001)
    st = S.stats()
    S.close()
    ok = [r for r in results.values() if r.status in (eng.GST_OK, eng.GST_NO_SOLUTION)]
    lat = [r.latency_ms for r in ok]
    return {"offered_qps": rate, "seconds": seconds, "arrivals": int(len(arr)), "shed_busy": shed,
            "completed": len(ok), "completed_qps": len(ok) / t_drain,
            "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
            "cancelled_unfinished": sum(r.status == eng.GST_CANCELLED for r in results.values()),
            "oom": st["oom"], "max_pending": max_pending, "drain_s": drain_s}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=["c4", "c4s", "c2", "c1"])
    ap.add_argument("--batch", type=int, default=0, help="queries per step (default: 128 on c4, 90 on c2)")
    ap.add_argument("--plain", type=int, default=300, help="queries on the plain per-query path")
    ap.add_argument("--sweep", default="1,2,4,8,16,32,64", help="closed-loop serving concurrencies")
    ap.add_argument("--sweep-queries", type=int, default=0, help="queries per sweep point (default 64 on c4)")
    ap.add_argument("--c5-rates", default="50,200,1000", help="open-loop Poisson rates (c4 only)")
    ap.add_argument("--c5-seconds", type=float, default=10.0, help="arrival window per rate")
    ap.add_argument("--c5-max-pending", type=int, default=256)
    ap.add_argument("--c5-drain", type=float, default=5.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--modes", type=int, default=1,
                    help="compare the round-launch modes (CUDA-graph blocks, persistent launches, 128-thread "
                         "blocks) on rank 0")
    ap.add_argument("--modes-plain", type=int, default=60, help="plain queries per launch mode")
    ap.add_argument("--c2-sweep", type=int, default=1,
                    help="with the batched configuration, also run the plain path and the serving sweep on the "
                         "170k-vertex workload (0: off)")
    args = ap.parse_args()
    big = args.workload in ("c4", "c4s")
    B = args.batch or (128 if big else 90)
    n_sweep = args.sweep_queries or (64 if big else 256)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    g, gr, qs, Ds = load_workload(args.workload)
    nq_set = len(qs)

    if args.impl == "reference":
        run_reference(args, g, gr, qs, Ds, rank, world)
        return

    cpu, cpu_costs = None, {}
    if rank == 0 and not args.no_cpu:
        cpu, cpu_costs = cpu_baseline_port(g, gr, qs, Ds, args.workload)

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

    def batch_for(step):
        # this rank's share of the query stream: the set in order, cycling
        base = (rank * (args.steps + args.warmup) + step) * B
        idx = [(base + i) % nq_set for i in range(B)]
        return [qs[i] for i in idx], [Ds[i] for i in idx]

    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for s in range(args.warmup):
        E.query_batch(*batch_for(s))
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
        qb, Db = batch_for(args.warmup + s)
        t0 = time.perf_counter()
        res = E.query_batch(qb, Db)
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
    tot_dev, tot_wall = replicas.max_over_ranks([sum(dev_ms), sum(wall_ms)], device="cuda")
    nq_all = B * args.steps * world
    value = nq_all / (tot_dev / 1e3)
    e2e_value = nq_all / (tot_wall / 1e3)

    # parity: the oracle's costs on the cpu sample against the GPU's (batched and plain)
    parity = None
    if rank == 0 and cpu_costs:
        idx = sorted(cpu_costs)
        res_b = E.query_batch([qs[i] for i in idx], [Ds[i] for i in idx])
        mism = []
        for i, r in zip(idx, res_b):
            st, c = cpu_costs[i]
            rp = E.query(qs[i], D=Ds[i])
            for rr in (r, rp):
                good = (rr.status == engine.GST_OK and st == 0 and rr.cost == c) or \
                       (rr.status == engine.GST_NO_SOLUTION and st == 1)
                if not good:
                    mism.append([i, c, rr.status, rr.cost])
        parity = {"checked": 2 * len(idx), "mismatches": len(mism), "against": "oracle restatement (exact) on the "
                  "cpu_baseline sample, batched and plain paths", "first": mism[:3]}

    # profiled pass (not timed): round-kernel device time and counters for the roofline
    E.profile(True)
    E.profile_reset()
    pq, pD = batch_for(args.warmup)
    E.query_batch(pq, pD)
    light_ms, heavy_ms, prof_rounds, st = E.profile_read()
    E.profile(False)
    dist_bytes = distance_work_bytes(st)
    lb_rows = sum(g.V * (32 + 2 * (1 << len(q))) for q in pq)
    dp_bytes = dp_work_bytes(st, lb_rows)
    peak, peak_kind = measured_peak_hbm()
    round_ms = light_ms + heavy_ms
    if E.tuning()["persistent"]:  # the rounds ran as persistent launches: one kernel
        rkernel, kernel_ms = "round (k_rounds, persistent)", {"k_rounds": light_ms}
    else:
        rkernel, kernel_ms = "round (k_light + k_heavy)", {"k_light": light_ms, "k_heavy": heavy_ms}
    round_bytes = dist_bytes + dp_bytes
    achieved = round_bytes / (round_ms / 1e3) / 1e9 if round_ms > 0 else 0.0
    tpb = traffic_per_byte()
    per_round_alg = round_bytes / max(prof_rounds, 1)

    # the round-launch modes on the same batches and plain queries (device
    # time): blocks of control / light / heavy launches as CUDA graphs, and
    # persistent cooperative launches (k_rounds), at 256 threads a block; and
    # the graph blocks at 128
    modes = None
    if rank == 0 and args.modes:
        modes = {}
        keep = E.tuning()
        for name, pv, bt in (("graph", 0, 256), ("persistent", 1, 256), ("graph_128_threads", 0, 128)):
            E.set_tuning(persistent=pv, block_threads=bt)
            E.query_batch(*batch_for(1))
            dms, nb = 0.0, 0
            for s in range(2):
                r = E.query_batch(*batch_for(2 + s))
                dms += r[0].device_ms
                nb += len(r)
            pl, pd = [], []
            for i in range(args.modes_plain):
                j = (i * 37) % nq_set
                t0 = time.perf_counter()
                rp = E.query(qs[j], D=Ds[j])
                pl.append(1e3 * (time.perf_counter() - t0))
                pd.append(rp.device_ms)
            modes[name] = {"batched_qps_device": nb / (dms / 1e3), "batched_queries": nb,
                           "plain_ms_mean": sum(pl) / len(pl), "plain_ms_p50": pct(pl, 50),
                           "plain_device_ms_mean": sum(pd) / len(pd), "plain_queries": len(pl)}
        E.set_tuning(**keep)

    # plain per-query path (one query per call, gst_query), same query set
    plain_lat, plain_dev = [], []
    for i in range(args.plain):
        j = (rank * 7919 + i) % nq_set
        t0 = time.perf_counter()
        r = E.query(qs[j], D=Ds[j])
        plain_lat.append(1e3 * (time.perf_counter() - t0))
        plain_dev.append(r.device_ms)
    plain_qps = len(plain_lat) / (sum(plain_lat) / 1e3) if plain_lat else None
    plain_dev_qps = len(plain_dev) / (sum(plain_dev) / 1e3) if plain_dev else None

    # closed-loop serving at several concurrencies (the latency / throughput trade-off)
    # (each point runs at least 8 x its concurrency requests, so that the
    # ramp-up and the drain do not dominate its rate)
    sweep = []
    for inflight in [int(x) for x in args.sweep.split(",") if x]:
        nreq = n_sweep if args.sweep_queries else max(n_sweep, 8 * inflight)
        reqs = [(qs[(rank * 104729 + 7 * i) % nq_set], Ds[(rank * 104729 + 7 * i) % nq_set]) for i in range(nreq)]
        qps, lats, sts = closed_loop(engine, E, reqs, inflight)
        sweep.append({"inflight": inflight, "qps": qps, "p50_ms": pct(lats, 50), "p99_ms": pct(lats, 99),
                      "vs_plain": qps / plain_qps if plain_qps else None, "queries": len(reqs)})

    # open-loop Poisson serving on the same resident graph (the c5 configuration)
    c5 = []
    if big and args.c5_rates:
        c5reqs = [(qs[i], Ds[i]) for i in range(nq_set)]
        for rate in [float(x) for x in args.c5_rates.split(",") if x]:
            c5.append(open_loop(engine, E, c5reqs, rate, args.c5_seconds, seed=5000 + int(rate),
                                max_pending=args.c5_max_pending, drain_s=args.c5_drain))

    # the same trade-off on the 170k-vertex workload (smaller queries: a
    # single one does not fill the GPU)
    c2 = None
    if big and args.c2_sweep and rank == 0:
        E.close()
        g2, gr2, qs2, Ds2 = load_workload("c2")
        E = engine.Engine.from_instance(g2, gr2)
        E.query_batch(qs2[:90], Ds2[:90])
        pl = []
        for i in range(100):
            t0 = time.perf_counter()
            E.query(qs2[i], D=Ds2[i])
            pl.append(1e3 * (time.perf_counter() - t0))
        p_qps = len(pl) / (sum(pl) / 1e3)
        t0 = time.perf_counter()
        rb = E.query_batch(qs2[100:190], Ds2[100:190])
        b_qps = 90 / (time.perf_counter() - t0)
        sw2 = []
        reqs2 = [(qs2[(11 * i) % len(qs2)], Ds2[(11 * i) % len(qs2)]) for i in range(256)]
        for inflight in [int(x) for x in args.sweep.split(",") if x]:
            qps, lats, _ = closed_loop(engine, E, reqs2, inflight)
            sw2.append({"inflight": inflight, "qps": qps, "p50_ms": pct(lats, 50), "p99_ms": pct(lats, 99),
                        "vs_plain": qps / p_qps, "queries": len(reqs2)})
        # round kernels' roofline on this workload (profiled 90-query batch)
        E.profile(True)
        E.profile_reset()
        q2, D2 = qs2[100:190], Ds2[100:190]
        E.query_batch(q2, D2)
        lm2, hm2, r2, st2 = E.profile_read()
        E.profile(False)
        lb2 = sum(g2.V * (32 + 2 * (1 << len(q))) for q in q2)
        bytes2 = distance_work_bytes(st2) + dp_work_bytes(st2, lb2)
        ach2 = bytes2 / ((lm2 + hm2) / 1e3) / 1e9 if lm2 + hm2 > 0 else 0.0
        c2 = {"workload": workload_desc("c2"), "plain_qps": p_qps, "plain_p50_ms": pct(pl, 50),
              "plain_p99_ms": pct(pl, 99), "batched_qps_e2e": b_qps, "batched_vs_plain_e2e": b_qps / p_qps,
              "batched_device_ms": rb[0].device_ms, "serve_sweep": sw2,
              "roofline": {"bound": "hbm", "kernel": "round (k_light + k_heavy)", "achieved": ach2, "peak": peak,
                           "unit": "GB/s", "frac": ach2 / peak, "peak_kind": peak_kind, "rounds": r2,
                           "kernel_ms": {"k_light": lm2, "k_heavy": hm2}, "algorithmic_bytes": bytes2}}

    if rank == 0:
        best_pt = max(sweep, key=lambda x: x["qps"]) if sweep else None
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
                       "queries": f"the {nq_set}-query set in order, cycling",
                       "parallelism": f"replicas x{world}", "l2": "256 MB buffer written between steps",
                       "queries_ok": n_ok},
            "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps},
            "parity": parity,
            "latency_ms": {"batched_p50": pct(lat, 50), "batched_p99": pct(lat, 99),
                           "plain_p50": pct(plain_lat, 50), "plain_p99": pct(plain_lat, 99)},
            "plain_per_query": {"value": plain_qps, "unit": "queries/s", "queries": len(plain_lat),
                                "device_value": plain_dev_qps, "device_ms_p50": pct(plain_dev, 50)},
            # like units: device throughput over device throughput, host wall over host wall
            "batched_vs_plain": {"device": value / plain_dev_qps if plain_dev_qps else None,
                                 "e2e": e2e_value / plain_qps if plain_qps else None},
            "serve_sweep": sweep,
            "serve_vs_plain_best": best_pt["vs_plain"] if best_pt else None,
            "open_loop": c5,
            "c2_170k": c2,
            "launch_modes": modes,
            "roofline": {"bound": "hbm", "kernel": rkernel, "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (per_round_alg * tpb) if tpb else None,
                         "algorithmic_bytes_per_round": per_round_alg, "rounds": prof_rounds,
                         "kernel_ms": kernel_ms,
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
