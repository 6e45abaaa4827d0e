"""Readers and writers of the reference's on-disk formats.

* ``<name>.in``   first line "V E", then one "v1 v2 w" line per undirected
  edge; the reference adds both directions and sorts each adjacency list
  (read_input_graph, graph_hash_of_mixed_weighted_read_for_GSTP.h:75-148).
* ``<name>.g``    one line "g<id>:v v v ..." per group, ids 1..n in order;
  group index = id - 1 (read_Group, same file :190-239).
* ``<name><k>.csv``  one query per line: k group indices separated by spaces
  (read_inquire, same file :240-286).
* ``<name>_beg_pos.bin``, ``_csr.bin``, ``_weight.bin``  int64 CSR arrays as
  loaded by GPUGST+ (code/GPUGST+/include/graph.hpp:12-118).
* GSTP text instances (``input_graph Vertex|Edge``, ``group_graph ...``,
  ``group_vertices g``; graph_hash_of_mixed_weighted_read_for_GSTP :9-73):
  group vertices are extra vertex ids joined to their members by
  ``group_graph Edge`` lines.
"""
from __future__ import annotations

import os

import numpy as np

from .gen import Graph, Groups, csr_from_edges


def write_in(path: str, g: Graph) -> None:
    u, v, w = g.edges()
    with open(path, "w") as f:
        f.write(f"{g.V} {len(u)}\n")
        np.savetxt(f, np.stack([u, v, w.astype(np.int64)], axis=1), fmt="%d")


def read_in(path: str) -> Graph:
    with open(path) as f:
        V = int(float(f.readline().split()[0]))
        rows = [t for t in (line.split() for line in f) if len(t) == 3]
    data = np.array(rows, dtype=np.int64).reshape(-1, 3)
    return csr_from_edges(V, data[:, 0], data[:, 1], data[:, 2].astype(np.int32))


def write_g(path: str, gr: Groups) -> None:
    with open(path, "w") as f:
        for gi in range(gr.n_groups):
            mem = gr.group(gi)
            f.write(f"g{gi + 1}:" + " ".join(map(str, mem.tolist())) + "\n")


def read_g(path: str) -> Groups:
    lists = []
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n").rstrip(" ")
            if not line:
                continue
            head, _, rest = line.partition(":")
            gid = int(float(head[1:])) - 1
            while len(lists) <= gid:
                lists.append([])
            lists[gid] = sorted(int(x) for x in rest.split())
    ptr = np.zeros(len(lists) + 1, dtype=np.uint64)
    ptr[1:] = np.cumsum([len(x) for x in lists])
    mem = np.array([x for l in lists for x in l], dtype=np.uint32)
    return Groups(ptr, mem)


def write_queries(path: str, q: np.ndarray) -> None:
    with open(path, "w") as f:
        for row in np.asarray(q):
            f.write(" ".join(map(str, row.tolist())) + "\n")


def read_queries(path: str) -> list:
    out = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line:
                out.append(np.array([int(x) for x in line.split()], dtype=np.uint32))
    return out


def write_bin(prefix: str, g: Graph) -> None:
    g.beg_pos.astype(np.int64).tofile(prefix + "_beg_pos.bin")
    g.csr.astype(np.int64).tofile(prefix + "_csr.bin")
    g.weight.astype(np.int64).tofile(prefix + "_weight.bin")


def read_bin(prefix: str) -> Graph:
    beg = np.fromfile(prefix + "_beg_pos.bin", dtype=np.int64)
    csr = np.fromfile(prefix + "_csr.bin", dtype=np.int64)
    w = np.fromfile(prefix + "_weight.bin", dtype=np.int64)
    if len(csr) != beg[-1] or len(w) != len(csr):
        raise ValueError("inconsistent .bin CSR")
    return Graph(len(beg) - 1, beg.astype(np.uint32), csr.astype(np.uint32), w.astype(np.int32))


def write_dataset(dirpath: str, name: str, g: Graph, gr: Groups, queries: dict) -> None:
    """Write <name>.in, <name>.g and <name><k>.csv as the reference drivers expect."""
    os.makedirs(dirpath, exist_ok=True)
    write_in(os.path.join(dirpath, name + ".in"), g)
    write_g(os.path.join(dirpath, name + ".g"), gr)
    for k, q in queries.items():
        write_queries(os.path.join(dirpath, f"{name}{k}.csv"), q)


def read_gstp(path: str):
    """GSTP text instance -> (Graph, Groups, query group indices).

    The instance's group vertices (``group_vertices g``) become groups 0..n-1
    in ascending id order; each group's members are its ``group_graph Edge``
    neighbours.  Returns the input graph over its own vertex ids."""
    edges, gedges, gvs = [], [], []
    vmax = -1
    with open(path) as f:
        for line in f:
            t = line.split()
            if len(t) < 2:
                continue
            if t[0] == "input_graph" and t[1] == "Vertex":
                vmax = max(vmax, int(t[2]))
            elif t[0] == "input_graph" and t[1] == "Edge":
                a, b, w = int(t[2]), int(t[3]), int(float(t[4]))
                edges.append((a, b, w))
                vmax = max(vmax, a, b)
            elif t[0] == "group_graph" and t[1] == "Edge":
                gedges.append((int(t[2]), int(t[3])))
            elif t[0] == "group_vertices":
                gvs.append(int(t[1]))
    gvs = sorted(set(gvs))
    gindex = {g: i for i, g in enumerate(gvs)}
    members = [[] for _ in gvs]
    for a, b in gedges:
        if a in gindex and b not in gindex:
            members[gindex[a]].append(b)
        elif b in gindex and a not in gindex:
            members[gindex[b]].append(a)
    V = vmax + 1
    # an edge listed twice keeps its last weight (hash-graph insertion semantics)
    ed = {}
    for a, b, w in edges:
        if a != b:
            ed[(min(a, b), max(a, b))] = w
    keys = np.array(list(ed.keys()), dtype=np.int64).reshape(-1, 2)
    ws = np.array(list(ed.values()), dtype=np.int32)
    g = csr_from_edges(V, keys[:, 0], keys[:, 1], ws)
    ptr = np.zeros(len(gvs) + 1, dtype=np.uint64)
    ptr[1:] = np.cumsum([len(set(m)) for m in members])
    mem = np.array([x for m in members for x in sorted(set(m))], dtype=np.uint32)
    return g, Groups(ptr, mem), np.arange(len(gvs), dtype=np.uint32)
