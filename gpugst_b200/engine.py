"""Python host mirror of the gstb C ABI (include/gstb.h) over ctypes.

The CUDA library ``libgstb.so`` is built in-tree by ``gpugst_b200.build``.
There is no CPU fallback: every entry point fails loudly when the library or
a CUDA device is missing.

The query surface follows the reference's: a CSR graph (beg_pos / csr /
weight, code/GPUGST/include/graph_v_of_v_idealID/csr_graph.hpp:39-128), a
group index (read_Group, graph_hash_of_mixed_weighted_read_for_GSTP.h:190-239),
and per query the k group indices plus an optional hop bound D
(DPBF_GPU, code/GPUGST/include/DPQ.cuh:63; DPBF_gpu,
code/D-GPUGST/include/DPQ.cuh:63).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgstb.so")

GST_OK, GST_NO_SOLUTION, GST_BAD_INPUT, GST_OOM = 0, 1, 2, 3
GST_DEVICE_TIMEOUT, GST_CUDA_ERROR, GST_QUEUE_OVERFLOW, GST_TRUNCATED = 4, 5, 6, 7
GST_INTERNAL, GST_BUSY, GST_NOT_FOUND, GST_SCRATCH_TOO_SMALL = 8, 9, 10, 11
GST_CANCELLED = 12
STATUS_NAMES = {0: "ok", 1: "no solution", 2: "bad input", 3: "out of memory", 4: "device timeout",
                5: "cuda error", 6: "queue overflow", 7: "truncated", 8: "internal", 9: "busy",
                10: "not found", 11: "scratch too small", 12: "cancelled"}
STAT_NAMES = ["expanded", "sssp_items", "arcs", "updates", "enqueued", "rounds", "merges", "table_bytes",
              "sssp_arcs", "sssp_updates", "sssp_enqueued", "retries", "lower_bound"]
NSTATS = len(STAT_NAMES)
GROUPS_STRIDE = 8  # row stride of gst_query_batch's groups array
KMAX = 7           # query groups at most


class GstError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        detail = ""
        if status == GST_CUDA_ERROR and _lib is not None:
            detail = f" ({_lib.gst_last_cuda_error().decode()})"
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}{detail}")


TUNING_FIELDS = ("delta_sssp", "delta_dp", "hub_min_deg", "cap_pct", "persistent", "rounds_per_launch",
                 "dp_wmax", "sssp_wmax", "merge_stage", "block_threads")


class _Tuning(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in TUNING_FIELDS]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n in TUNING_FIELDS}


class _ServeInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("pending", "inflight", "finished_unpolled", "budget_bytes",
                                               "in_use_bytes", "submitted", "completed", "rejected_busy",
                                               "cancelled", "oom")]


class _Result(ctypes.Structure):
    _fields_ = [("cost", ctypes.c_int32), ("root", ctypes.c_uint32), ("n_edges", ctypes.c_int32),
                ("max_edges", ctypes.c_int32), ("edges", ctypes.POINTER(ctypes.c_uint32)),
                ("stats", ctypes.c_uint64 * NSTATS), ("device_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double)]


_lib = None


def lib():
    """Load libgstb.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run gpugst_b200.build.build() first")
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32
        L.gst_graph_create.argtypes = [vp, vp, vp, u32, u64, ctypes.POINTER(vp)]
        L.gst_groups_set.argtypes = [vp, vp, vp, u32]
        L.gst_graph_destroy.argtypes = [vp]
        L.gst_graph_destroy.restype = None
        L.gst_query.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Result)]
        L.gst_query_batch.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int]
        L.gst_query_batch_ratio.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp, ctypes.c_int]
        L.gst_query_ratio.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(_Result)]
        L.gst_serve_submit_ratio.argtypes = [vp, u64, vp, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.gst_query_noalloc.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Result)]
        L.gst_query_noalloc.restype = ctypes.c_int
        L.gst_status_string.restype = ctypes.c_char_p
        L.gst_last_cuda_error.restype = ctypes.c_char_p
        L.gst_last_cuda_error.argtypes = []
        L.gst_tuning_get.argtypes = [vp, ctypes.POINTER(_Tuning)]
        L.gst_tuning_set.argtypes = [vp, ctypes.POINTER(_Tuning)]
        L.gst_autotune.argtypes = [vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, ctypes.POINTER(_Tuning)]
        L.gst_graph_num_vertices.restype = u32
        L.gst_graph_num_vertices.argtypes = [vp]
        L.gst_graph_num_arcs.restype = u64
        L.gst_graph_num_arcs.argtypes = [vp]
        L.gst_kernel_launches.argtypes = [vp]
        L.gst_kernel_launches.restype = u64
        L.gst_profile_enable.argtypes = [vp, ctypes.c_int]
        L.gst_profile_enable.restype = None
        L.gst_profile_read.argtypes = [vp, vp, ctypes.POINTER(u64), vp]
        L.gst_profile_read.restype = None
        L.gst_profile_reset.argtypes = [vp]
        L.gst_profile_reset.restype = None
        L.gst_serve_open.argtypes = [vp, u64, ctypes.c_int, ctypes.POINTER(vp)]
        L.gst_serve_submit.argtypes = [vp, u64, vp, ctypes.c_int, ctypes.c_int]
        L.gst_serve_poll.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.gst_serve_close.argtypes = [vp]
        L.gst_serve_cancel.argtypes = [vp, u64]
        L.gst_serve_set_max_pending.argtypes = [vp, u64]
        L.gst_serve_stats.argtypes = [vp, ctypes.POINTER(_ServeInfo)]
        L.gst_debug_fail_allocs.argtypes = [vp, ctypes.c_int]
        L.gst_debug_hold_rounds.argtypes = [vp, ctypes.c_int, ctypes.c_uint32]
        for name in ("gst_serve_open", "gst_serve_submit", "gst_serve_poll", "gst_serve_close", "gst_serve_cancel",
                     "gst_serve_set_max_pending", "gst_serve_stats", "gst_debug_fail_allocs", "gst_debug_hold_rounds"):
            getattr(L, name).restype = ctypes.c_int
        for name in ("gst_graph_create", "gst_groups_set", "gst_query", "gst_query_batch", "gst_query_batch_ratio",
                     "gst_query_ratio", "gst_serve_submit_ratio"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


@dataclass
class QueryResult:
    status: int
    cost: int
    root: int
    edges: np.ndarray  # (n, 3) uint32: u, v, w
    stats: dict = field(default_factory=dict)
    device_ms: float = 0.0
    latency_ms: float = 0.0

    @property
    def ok(self) -> bool:
        return self.status == GST_OK


class Engine:
    """A graph + group index resident on the current CUDA device."""

    def __init__(self, beg_pos, csr, weight, grp_ptr=None, grp_v=None):
        L = lib()
        self._beg = np.ascontiguousarray(beg_pos, dtype=np.uint32)
        self._csr = np.ascontiguousarray(csr, dtype=np.uint32)
        self._w = np.ascontiguousarray(weight, dtype=np.int32)
        V = len(self._beg) - 1
        h = ctypes.c_void_p()
        st = L.gst_graph_create(_ptr(self._beg), _ptr(self._csr), _ptr(self._w), V, len(self._csr),
                                ctypes.byref(h))
        if st != GST_OK:
            raise GstError(st, "gst_graph_create")
        self._h = h
        self.V = V
        if grp_ptr is not None:
            self.set_groups(grp_ptr, grp_v)

    @classmethod
    def from_instance(cls, graph, groups):
        return cls(graph.beg_pos, graph.csr, graph.weight, groups.ptr, groups.members)

    def set_groups(self, grp_ptr, grp_v):
        self._gp = np.ascontiguousarray(grp_ptr, dtype=np.uint64)
        self._gv = np.ascontiguousarray(grp_v, dtype=np.uint32)
        st = lib().gst_groups_set(self._h, _ptr(self._gp), _ptr(self._gv), len(self._gp) - 1)
        if st != GST_OK:
            raise GstError(st, "gst_groups_set")

    def close(self):
        if getattr(self, "_h", None):
            lib().gst_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _unpack(st, r, buf):
        n = min(max(r.n_edges, 0), r.max_edges)
        edges = buf[:3 * n].reshape(-1, 3).copy() if st in (GST_OK, GST_TRUNCATED) else np.zeros((0, 3), np.uint32)
        stats = {name: int(r.stats[i]) for i, name in enumerate(STAT_NAMES)}
        return QueryResult(st, r.cost, r.root, edges, stats, r.device_ms, r.latency_ms)

    def fail_allocs(self, n: int):
        """Fault injection: the next n workspace allocations fail (gst_debug_fail_allocs)."""
        st = lib().gst_debug_fail_allocs(self._h, int(n))
        if st != GST_OK:
            raise GstError(st, "gst_debug_fail_allocs")

    def hold_rounds(self, hold: bool, timeout_ms: int = 0):
        """Test hook (gst_debug_hold_rounds): while held, persistent round
        launches publish no control step, so their bounded waits expire after
        timeout_ms and the admitted queries end with GST_DEVICE_TIMEOUT."""
        st = lib().gst_debug_hold_rounds(self._h, 1 if hold else 0, int(timeout_ms))
        if st != GST_OK:
            raise GstError(st, "gst_debug_hold_rounds")

    def kernel_launches(self) -> int:
        return int(lib().gst_kernel_launches(self._h))

    def profile(self, on: bool = True):
        lib().gst_profile_enable(self._h, 1 if on else 0)

    def profile_reset(self):
        lib().gst_profile_reset(self._h)

    def profile_read(self):
        """(light_ms, heavy_ms, rounds, summed stats) accumulated while profiling."""
        ms = np.zeros(2, dtype=np.float64)
        n = ctypes.c_uint64(0)
        tot = np.zeros(NSTATS, dtype=np.uint64)
        lib().gst_profile_read(self._h, _ptr(ms), ctypes.byref(n), _ptr(tot))
        return float(ms[0]), float(ms[1]), n.value, {name: int(tot[i]) for i, name in enumerate(STAT_NAMES)}

    def tuning(self) -> dict:
        """The engine's launch parameters (gst_tuning_get)."""
        t = _Tuning()
        st = lib().gst_tuning_get(self._h, ctypes.byref(t))
        if st != GST_OK:
            raise GstError(st, "gst_tuning_get")
        return t.as_dict()

    def set_tuning(self, **kw):
        """Change launch parameters (gst_tuning_set); unnamed ones keep their values."""
        cur = self.tuning()
        unknown = set(kw) - set(TUNING_FIELDS)
        if unknown:
            raise ValueError(f"unknown launch parameters {sorted(unknown)}")
        cur.update(kw)
        t = _Tuning(*[cur[n] for n in TUNING_FIELDS])
        st = lib().gst_tuning_set(self._h, ctypes.byref(t))
        if st != GST_OK:
            raise GstError(st, "gst_tuning_set")

    def autotune(self, queries, Ds=None, objective: str = "throughput") -> dict:
        """Pick launch parameters on a sample of queries (gst_autotune);
        objective "throughput" (batches) or "latency" (one query at a time)."""
        n = len(queries)
        groups = np.zeros((n, GROUPS_STRIDE), dtype=np.uint32)
        ks = np.zeros(n, dtype=np.int32)
        for i, q in enumerate(queries):
            ks[i] = len(q)
            groups[i, :len(q)] = q
        Darr = np.full(n, -1, dtype=np.int32) if Ds is None else np.ascontiguousarray(Ds, dtype=np.int32)
        t = _Tuning()
        st = lib().gst_autotune(self._h, n, _ptr(groups), _ptr(ks), _ptr(Darr),
                                0 if objective == "throughput" else 1, ctypes.byref(t))
        if st != GST_OK:
            raise GstError(st, "gst_autotune")
        return t.as_dict()

    def query(self, groups, D: int = -1, max_edges: int = 4096, ratio: float = 0.0) -> QueryResult:
        """One synchronous query (gst_query; gst_query_ratio when ratio > 1:
        progressive mode, cost at most ratio x the optimum)."""
        g = np.ascontiguousarray(groups, dtype=np.uint32)
        buf = np.zeros(3 * max_edges, dtype=np.uint32)
        r = _Result()
        r.max_edges = max_edges
        r.edges = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        if ratio:
            st = lib().gst_query_ratio(self._h, _ptr(g), len(g), int(D), float(ratio), ctypes.byref(r))
        else:
            st = lib().gst_query(self._h, _ptr(g), len(g), int(D), ctypes.byref(r))
        if st in (GST_CUDA_ERROR, GST_INTERNAL):
            raise GstError(st, "gst_query")
        return self._unpack(st, r, buf)

    def query_noalloc(self, groups, D: int = -1, max_edges: int = 4096) -> QueryResult:
        """One query through gst_query_noalloc: every per-query device buffer
        lives in the library's static scratch array, nothing is allocated."""
        g = np.ascontiguousarray(groups, dtype=np.uint32)
        buf = np.zeros(3 * max_edges, dtype=np.uint32)
        r = _Result()
        r.max_edges = max_edges
        r.edges = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        st = lib().gst_query_noalloc(self._h, _ptr(g), len(g), int(D), ctypes.byref(r))
        if st in (GST_CUDA_ERROR, GST_INTERNAL):
            raise GstError(st, "gst_query_noalloc")
        return self._unpack(st, r, buf)

    def query_batch(self, queries, Ds=None, max_concurrent: int = 0, max_edges: int = 4096, ratios=None):
        """Many queries sharing device rounds (gst_query_batch; per-query
        progressive-mode ratios through gst_query_batch_ratio)."""
        n = len(queries)
        groups = np.zeros((n, GROUPS_STRIDE), dtype=np.uint32)
        ks = np.zeros(n, dtype=np.int32)
        for i, q in enumerate(queries):
            ks[i] = len(q)
            groups[i, :len(q)] = q
        Darr = np.full(n, -1, dtype=np.int32) if Ds is None else np.ascontiguousarray(Ds, dtype=np.int32)
        statuses = np.zeros(n, dtype=np.int32)
        res = (_Result * max(n, 1))()
        bufs = []
        for i in range(n):
            b = np.zeros(3 * max_edges, dtype=np.uint32)
            bufs.append(b)
            res[i].max_edges = max_edges
            res[i].edges = b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        if ratios is None:
            st = lib().gst_query_batch(self._h, n, _ptr(groups), _ptr(ks), _ptr(Darr), ctypes.cast(res, ctypes.c_void_p),
                                       _ptr(statuses), int(max_concurrent))
        else:
            rat = np.ascontiguousarray(ratios, dtype=np.float64)
            st = lib().gst_query_batch_ratio(self._h, n, _ptr(groups), _ptr(ks), _ptr(Darr), _ptr(rat),
                                             ctypes.cast(res, ctypes.c_void_p), _ptr(statuses), int(max_concurrent))
        if st != GST_OK:
            raise GstError(st, "gst_query_batch")
        out = [self._unpack(int(statuses[i]), res[i], bufs[i]) for i in range(n)]
        for r in out:
            if r.status in (GST_CUDA_ERROR, GST_INTERNAL):
                raise GstError(r.status, "gst_query_batch")
        return out


class Server:
    """Continuous-batching serving loop over an Engine's graph (gst_serve_*)."""

    def __init__(self, eng: Engine, hbm_budget: int = 0, max_inflight: int = 0):
        self._eng = eng
        h = ctypes.c_void_p()
        st = lib().gst_serve_open(eng._h, int(hbm_budget), int(max_inflight), ctypes.byref(h))
        if st != GST_OK:
            raise GstError(st, "gst_serve_open")
        self._h = h

    def submit(self, req_id: int, groups, D: int = -1, ratio: float = 0.0) -> int:
        g = np.ascontiguousarray(groups, dtype=np.uint32)
        if ratio:
            return int(lib().gst_serve_submit_ratio(self._h, int(req_id), _ptr(g), len(g), int(D), float(ratio)))
        return int(lib().gst_serve_submit(self._h, int(req_id), _ptr(g), len(g), int(D)))

    def poll(self, max_results: int = 1024, max_edges: int = 0):
        """Finished requests as a list of (req_id, QueryResult)."""
        ids = np.zeros(max_results, dtype=np.uint64)
        sts = np.zeros(max_results, dtype=np.int32)
        res = (_Result * max_results)()
        bufs = []
        for i in range(max_results):
            if max_edges:
                b = np.zeros(3 * max_edges, dtype=np.uint32)
                bufs.append(b)
                res[i].edges = b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
            res[i].max_edges = max_edges
        n = ctypes.c_int(0)
        st = lib().gst_serve_poll(self._h, _ptr(ids), _ptr(sts), ctypes.cast(res, ctypes.c_void_p), max_results,
                                  ctypes.byref(n))
        if st != GST_OK:
            raise GstError(st, "gst_serve_poll")
        out = []
        for i in range(n.value):
            buf = bufs[i] if max_edges else np.zeros(0, dtype=np.uint32)
            out.append((int(ids[i]), Engine._unpack(int(sts[i]), res[i], buf)))
        return out

    def cancel(self, req_id: int) -> int:
        """Withdraw a request (gst_serve_cancel): GST_OK or GST_NOT_FOUND."""
        return int(lib().gst_serve_cancel(self._h, int(req_id)))

    def set_max_pending(self, n: int):
        st = lib().gst_serve_set_max_pending(self._h, int(n))
        if st != GST_OK:
            raise GstError(st, "gst_serve_set_max_pending")

    def stats(self) -> dict:
        """Occupancy and counters (gst_serve_stats)."""
        info = _ServeInfo()
        st = lib().gst_serve_stats(self._h, ctypes.byref(info))
        if st != GST_OK:
            raise GstError(st, "gst_serve_stats")
        return {n: int(getattr(info, n)) for n, _ in _ServeInfo._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().gst_serve_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
