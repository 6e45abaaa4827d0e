"""Seeded synthetic GST instances with the shapes of the reference's datasets.

The reference ships no usable dataset (its Twitch CSR blobs are missing and the
other five live off-line), so every workload here is generated:

* ``chung_lu``  -- undirected power-law graph, expected degree of vertex i
  proportional to (i + i0)^(-1/(gamma-1)), endpoints sampled proportional to
  that weight, self-loops and duplicate edges rejected until exactly E unique
  edges remain.  i0 is chosen so that the largest expected degree is about
  2*sqrt(2E) (hubs in the thousands to tens of thousands at the sizes used).
* ``rmat``      -- R-MAT / Kronecker edges with initiator (a, b, c, d) =
  (0.57, 0.19, 0.19, 0.05), the Graph500 values, vertex labels permuted,
  self-loops and duplicates dropped, symmetrised.
* ``zipf_groups`` -- group sizes ~ Zipf(s) truncated to [1, smax], members
  uniform without replacement; every vertex left uncovered is then appended to
  a uniformly random group, so every vertex is in at least one group.
* ``queries``   -- k distinct group ids, uniform.

Edge weights are int32 uniform in [1, 100].  The CSR is symmetric (both arc
directions) with each adjacency list sorted by neighbour id, which is what the
reference's ``read_input_graph`` + ``toCSR`` produce
(graph_hash_of_mixed_weighted_read_for_GSTP.h:75-148, csr_graph.hpp:39-128).
"""
from __future__ import annotations

import dataclasses
import numpy as np


@dataclasses.dataclass
class Graph:
    V: int
    beg_pos: np.ndarray  # uint32 [V+1]
    csr: np.ndarray      # uint32 [arcs]
    weight: np.ndarray   # int32  [arcs]

    @property
    def arcs(self) -> int:
        return int(self.beg_pos[-1])

    def edges(self):
        """Undirected edge list (u < v) with weights."""
        src = np.repeat(np.arange(self.V, dtype=np.int64), np.diff(self.beg_pos.astype(np.int64)))
        m = src < self.csr
        return src[m], self.csr[m].astype(np.int64), self.weight[m]


@dataclasses.dataclass
class Groups:
    ptr: np.ndarray      # uint64 [n_groups+1]
    members: np.ndarray  # uint32 [ptr[-1]], sorted within each group

    @property
    def n_groups(self) -> int:
        return len(self.ptr) - 1

    def group(self, g: int) -> np.ndarray:
        return self.members[self.ptr[g]:self.ptr[g + 1]]


def csr_from_edges(V: int, u: np.ndarray, v: np.ndarray, w: np.ndarray) -> Graph:
    """Symmetric CSR, adjacency sorted by neighbour id."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    w = np.asarray(w, dtype=np.int32)
    if len(w) and 0 <= int(w.min()) and int(w.max()) < 128 and V < (1 << 28):
        # one sort of packed (src, dst, weight) keys instead of a two-key lexsort
        key = np.concatenate([u * V + v, v * V + u])
        key *= 128
        key += np.concatenate([w, w]).astype(np.int64)
        key.sort()
        ww = (key % 128).astype(np.int32)
        key //= 128
        src = key // V
        dst = key % V
    else:
        src = np.concatenate([u, v])
        dst = np.concatenate([v, u])
        ww = np.concatenate([w, w])
        order = np.lexsort((dst, src))
        src, dst, ww = src[order], dst[order], ww[order]
    counts = np.bincount(src, minlength=V)
    beg = np.zeros(V + 1, dtype=np.uint64)
    np.cumsum(counts, out=beg[1:])
    if beg[-1] >= 2**32:
        raise ValueError("arc count exceeds uint32 offsets")
    return Graph(V, beg.astype(np.uint32), dst.astype(np.uint32), ww)


def _take_sorted(keys: np.ndarray, E: int, rng) -> np.ndarray:
    """E keys chosen uniformly at random (linear-time selection), sorted."""
    if len(keys) <= E:
        return keys
    pri = rng.random(len(keys))
    idx = np.argpartition(pri, E)[:E]
    out = keys[idx]
    out.sort()
    return out


def _sample_endpoints(cdf: np.ndarray, n: int, rng) -> np.ndarray:
    """n vertices drawn from the distribution `cdf`, in random order.  The
    uniforms are sorted before the search (cache-friendly), then the result
    is shuffled; the multiset drawn is the same as with unsorted uniforms."""
    x = rng.random(n)
    x.sort()
    a = np.searchsorted(cdf, x, side="right")
    rng.shuffle(a)
    return np.minimum(a, len(cdf) - 1)


def _sorted_unique(x: np.ndarray) -> np.ndarray:
    """Sorted distinct values (sort + mask; faster than np.unique on large
    integer arrays with mostly distinct values)."""
    x = np.sort(x)
    if len(x) == 0:
        return x
    keep = np.empty(len(x), dtype=bool)
    keep[0] = True
    np.not_equal(x[1:], x[:-1], out=keep[1:])
    return x[keep]


def _unique_edges(V: int, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    keep = a != b
    a, b = a[keep], b[keep]
    lo = np.minimum(a, b).astype(np.int64)
    hi = np.maximum(a, b).astype(np.int64)
    return _sorted_unique(lo * V + hi)


def chung_lu(V: int, E: int, gamma: float, seed: int, wmax: int = 100) -> Graph:
    rng = np.random.default_rng(seed)
    beta = 1.0 / (gamma - 1.0)
    dmax = min(2.0 * np.sqrt(2.0 * E), V / 2.0)
    davg = 2.0 * E / V
    # choose i0 so that w_0 / mean(w) ~= dmax / davg (bisection on log i0)
    idx = np.arange(V, dtype=np.float64)

    def ratio(i0):
        w = (idx + i0) ** (-beta)
        return w[0] / w.mean()

    lo, hi = 0.0, float(V)
    target = dmax / davg
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if ratio(mid) > target:
            lo = mid
        else:
            hi = mid
    i0 = 0.5 * (lo + hi)
    wts = (idx + i0) ** (-beta)
    cdf = np.cumsum(wts)
    cdf /= cdf[-1]
    keys = np.empty(0, dtype=np.int64)
    need = E
    while True:
        n = int(need * 1.15) + 1024
        a = _sample_endpoints(cdf, n, rng)
        b = _sample_endpoints(cdf, n, rng)
        new = _unique_edges(V, a, b)
        keys = new if len(keys) == 0 else _sorted_unique(np.concatenate([keys, new]))
        if len(keys) >= E:
            break
        need = E - len(keys)
    keys = _take_sorted(keys, E, rng)
    u = keys // V
    v = keys % V
    w = rng.integers(1, wmax + 1, size=len(keys), dtype=np.int32)
    return csr_from_edges(V, u, v, w)


def rmat(scale: int, E: int, seed: int, a=0.57, b=0.19, c=0.19, wmax: int = 100) -> Graph:
    rng = np.random.default_rng(seed)
    V = 1 << scale
    perm = rng.permutation(V).astype(np.int64)
    keys = np.empty(0, dtype=np.int64)
    need = E
    while True:
        n = int(need * 1.6) + 1024
        src = np.zeros(n, dtype=np.int64)
        dst = np.zeros(n, dtype=np.int64)
        for _ in range(scale):
            r = rng.random(n)
            sbit = (r >= a + b).astype(np.int64)            # quadrants c, d
            dbit = (((r >= a) & (r < a + b)) | (r >= a + b + c)).astype(np.int64)  # b, d
            src = (src << 1) | sbit
            dst = (dst << 1) | dbit
        new = _unique_edges(V, perm[src], perm[dst])
        keys = new if len(keys) == 0 else _sorted_unique(np.concatenate([keys, new]))
        if len(keys) >= E:
            break
        need = E - len(keys)
    keys = _take_sorted(keys, E, rng)
    u = keys // V
    v = keys % V
    w = rng.integers(1, wmax + 1, size=len(keys), dtype=np.int32)
    return csr_from_edges(V, u, v, w)


def zipf_groups(V: int, n_groups: int, s: float, smax: int, seed: int) -> Groups:
    rng = np.random.default_rng(seed)
    ks = np.arange(1, smax + 1, dtype=np.float64)
    p = ks ** (-s)
    p /= p.sum()
    sizes = rng.choice(np.arange(1, smax + 1), size=n_groups, p=p).astype(np.int64)
    total = int(sizes.sum())
    gid = np.repeat(np.arange(n_groups, dtype=np.int64), sizes)
    mem = rng.integers(0, V, size=total, dtype=np.int64)
    # redraw duplicates inside a group until none remain
    while True:
        key = gid * V + mem
        order = np.argsort(key, kind="stable")
        ks_sorted = key[order]
        dup = np.zeros(total, dtype=bool)
        dup[order[1:]] = ks_sorted[1:] == ks_sorted[:-1]
        nd = int(dup.sum())
        if nd == 0:
            break
        mem[dup] = rng.integers(0, V, size=nd, dtype=np.int64)
    covered = np.zeros(V, dtype=bool)
    covered[mem] = True
    unc = np.flatnonzero(~covered).astype(np.int64)
    if len(unc):
        extra_g = rng.integers(0, n_groups, size=len(unc), dtype=np.int64)
        gid = np.concatenate([gid, extra_g])
        mem = np.concatenate([mem, unc])
    order = np.lexsort((mem, gid))
    gid, mem = gid[order], mem[order]
    counts = np.bincount(gid, minlength=n_groups)
    ptr = np.zeros(n_groups + 1, dtype=np.uint64)
    np.cumsum(counts, out=ptr[1:])
    return Groups(ptr, mem.astype(np.uint32))


def queries(n_groups: int, n: int, k: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = np.empty((n, k), dtype=np.uint32)
    for i in range(n):
        out[i] = rng.choice(n_groups, size=k, replace=False)
    return out


# ---------------------------------------------------------------------------
# The workloads (sizes from the reference benchmark descriptions).
# ---------------------------------------------------------------------------

def config1(seed: int = 1):
    """V=10k, E=50k Chung-Lu (gamma 2.5); 2,000 Zipf(1.5) groups in [1,50]; 50 queries k=3."""
    g = chung_lu(10_000, 50_000, 2.5, seed=1000 + seed)
    gr = zipf_groups(g.V, 2_000, 1.5, 50, seed=2000 + seed)
    q = queries(gr.n_groups, 50, 3, seed=3000 + seed)
    return g, gr, {3: q}


def config2(seed: int = 2, n_per_k: int = 300):
    """V=170k, E=6.8M Chung-Lu (gamma 2.3); 200k Zipf(1.5) groups in [1,200]; 300 queries at each k=3,4,5."""
    g = chung_lu(170_000, 6_800_000, 2.3, seed=1000 + seed)
    gr = zipf_groups(g.V, 200_000, 1.5, 200, seed=2000 + seed)
    qs = {k: queries(gr.n_groups, n_per_k, k, seed=3000 + 10 * seed + k) for k in (3, 4, 5)}
    return g, gr, qs


def config3(seed: int = 3, n_per_cell: int = 100):
    """R-MAT scale 20, E~10M; 500k Zipf(1.5) groups in [1,200]; k in {3,4,5} x D in {2,3,4}."""
    g = rmat(20, 10_000_000, seed=1000 + seed)
    gr = zipf_groups(g.V, 500_000, 1.5, 200, seed=2000 + seed)
    qs = {(k, D): queries(gr.n_groups, n_per_cell, k, seed=3000 + 100 * seed + 10 * k + D)
          for k in (3, 4, 5) for D in (2, 3, 4)}
    return g, gr, qs


def config4(seed: int = 4, n_queries: int = 1024):
    """V=3M, E=117M Chung-Lu (gamma 2.1); 1M Zipf(1.3) groups in [1,500];
    1,024 queries, k uniform in {3,4,5,6}, half with D uniform in {2,3,4}."""
    g = chung_lu(3_000_000, 117_000_000, 2.1, seed=1000 + seed)
    gr = zipf_groups(g.V, 1_000_000, 1.3, 500, seed=2000 + seed)
    rng = np.random.default_rng(3000 + seed)
    qs, Ds = [], []
    for _ in range(n_queries):
        k = int(rng.integers(3, 7))
        qs.append(rng.choice(gr.n_groups, size=k, replace=False).astype(np.uint32))
        Ds.append(int(rng.choice([2, 3, 4])) if rng.random() < 0.5 else -1)
    return g, gr, qs, Ds


def config4_small(seed: int = 4, n_queries: int = 1024):
    """The batched configuration at a third of its size, for profiler
    captures that must stay within a few GB of device memory: V=1M, E=39M
    Chung-Lu (gamma 2.1); 333,333 Zipf(1.3) groups in [1,500]; 1,024 queries,
    k uniform in {3,4,5,6}, half with D uniform in {2,3,4}."""
    g = chung_lu(1_000_000, 39_000_000, 2.1, seed=1100 + seed)
    gr = zipf_groups(g.V, 333_333, 1.3, 500, seed=2100 + seed)
    rng = np.random.default_rng(3100 + seed)
    qs, Ds = [], []
    for _ in range(n_queries):
        k = int(rng.integers(3, 7))
        qs.append(rng.choice(gr.n_groups, size=k, replace=False).astype(np.uint32))
        Ds.append(int(rng.choice([2, 3, 4])) if rng.random() < 0.5 else -1)
    return g, gr, qs, Ds


def poisson_arrivals(rate: float, duration: float, seed: int) -> np.ndarray:
    """Arrival times (seconds) of a Poisson process of the given rate."""
    rng = np.random.default_rng(seed)
    n = int(rate * duration * 1.5) + 16
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    return t[t < duration]


def small_instance(V: int, E: int, n_groups: int, smax: int, seed: int, gamma: float = 2.5):
    """Small seeded Chung-Lu instance for parity tests."""
    E = min(E, V * (V - 1) // 2)
    g = chung_lu(V, E, gamma, seed=seed)
    gr = zipf_groups(V, n_groups, 1.5, smax, seed=seed + 7)
    return g, gr
