"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this
module; the product never does.  ``build()`` compiles gst_oracle.cpp with g++.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libgst_oracle.so")
SRC = os.path.join(HERE, "gst_oracle.cpp")

_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["g++", "-O3", "-march=x86-64-v2", "-std=c++17", "-shared", "-fPIC",
                               "-o", LIB, SRC])
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        for name in ("oracle_prunedpp", "oracle_hop", "oracle_hop_budget", "oracle_dpbf", "oracle_brute",
                     "oracle_validate"):
            getattr(_lib, name).restype = ctypes.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _query_arrays(groups, query):
    lists = [np.asarray(groups.group(int(g)), dtype=np.uint32) for g in query]
    ptr = np.zeros(len(lists) + 1, dtype=np.uint64)
    ptr[1:] = np.cumsum([len(x) for x in lists])
    qv = np.concatenate(lists).astype(np.uint32) if lists else np.zeros(0, np.uint32)
    return ptr, qv


class Result:
    __slots__ = ("status", "cost", "root", "edges", "process")

    def __init__(self, status, cost, root, edges, process):
        self.status, self.cost, self.root, self.edges, self.process = status, cost, root, edges, process

    def __repr__(self):
        return f"Result(status={self.status}, cost={self.cost}, root={self.root}, n_edges={len(self.edges)})"


def _run(fn, graph, groups, query, extra_before=(), max_edges=1 << 16):
    ptr, qv = _query_arrays(groups, query)
    cost = ctypes.c_int32(0)
    root = ctypes.c_uint32(0)
    ne = ctypes.c_int32(0)
    edges = np.zeros(3 * max_edges, dtype=np.uint32)
    stats = np.zeros(4, dtype=np.int64)
    st = fn(ctypes.c_uint32(graph.V), _p(graph.beg_pos), _p(graph.csr), _p(graph.weight),
            ctypes.c_int(len(query)), _p(ptr), _p(qv), *extra_before,
            ctypes.byref(cost), ctypes.byref(root), ctypes.byref(ne), _p(edges),
            ctypes.c_int(max_edges), _p(stats))
    n = min(ne.value, max_edges)
    return Result(st, cost.value, root.value, edges[:3 * n].reshape(-1, 3).copy(), int(stats[0]))


def prunedpp(graph, groups, query, ratio: int = 0) -> Result:
    """PrunedDP++ restatement; ratio=0 is the exact mode."""
    return _run(lib().oracle_prunedpp, graph, groups, query, (ctypes.c_int(ratio),))


def hop(graph, groups, query, D: int) -> Result:
    return _run(lib().oracle_hop, graph, groups, query, (ctypes.c_int(D),))


def hop_budget(graph, groups, query, D: int, ub: int):
    """HOP_cpu with the engine's hop-budget bound against the upper bound ub:
    (status, cost, states popped)."""
    ptr, qv = _query_arrays(groups, query)
    cost = ctypes.c_int32(0)
    stats = np.zeros(4, dtype=np.int64)
    st = lib().oracle_hop_budget(ctypes.c_uint32(graph.V), _p(graph.beg_pos), _p(graph.csr), _p(graph.weight),
                                 ctypes.c_int(len(query)), _p(ptr), _p(qv), ctypes.c_int(D), ctypes.c_int64(ub),
                                 ctypes.byref(cost), _p(stats))
    return st, cost.value, int(stats[0])


def dpbf(graph, groups, query) -> Result:
    return _run(lib().oracle_dpbf, graph, groups, query)


def brute(graph, groups, query, D: int = -1) -> int:
    ptr, qv = _query_arrays(groups, query)
    cost = ctypes.c_int32(0)
    st = lib().oracle_brute(ctypes.c_uint32(graph.V), _p(graph.beg_pos), _p(graph.csr), _p(graph.weight),
                            ctypes.c_int(len(query)), _p(ptr), _p(qv), ctypes.c_int(D), ctypes.byref(cost))
    if st == 2:
        raise ValueError("graph too large for brute force")
    return cost.value


def validate(graph, groups, query, D: int, cost: int, root: int, edges) -> int:
    """0 = valid tree; see gst_oracle.cpp for the failure codes."""
    ptr, qv = _query_arrays(groups, query)
    e = np.ascontiguousarray(np.asarray(edges, dtype=np.uint32).reshape(-1))
    return lib().oracle_validate(ctypes.c_uint32(graph.V), _p(graph.beg_pos), _p(graph.csr), _p(graph.weight),
                                 ctypes.c_int(len(query)), _p(ptr), _p(qv), ctypes.c_int(D),
                                 ctypes.c_int32(cost), ctypes.c_uint32(root), ctypes.c_int32(len(e) // 3),
                                 _p(e) if len(e) else None)
