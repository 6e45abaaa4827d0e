// CUDA kernels of the gstb engine, sm_100a.
//
// Hot path of one query (the reference's DPBF_GPU, code/GPUGST/src/DPQ.cu:275-624,
// and DPBF_gpu, code/D-GPUGST/src/DPQ.cu:149-269, re-designed).  Every round is
//   k_control  one thread per query slot: advances the query's state machine
//              (distance rounds -> tour tables -> DP seed -> DP rounds ->
//              extraction) and writes the round's work description;
//   k_light    warp tasks: near-far splits, seeds, tour tables, extraction,
//              distance items (a vertex with its pending groups; the arcs of
//              a task's items are relaxed as one flat list by the whole warp:
//              multi-source relax, replacing dis0_init_1, DPQ.cu:241-271) and
//              DP items, one warp per state: best update from complement /
//              one-label completion, lower-bound prune, grow along the
//              weight-sorted adjacency, merge with every disjoint subset at
//              the vertex (replaces Relax, DPQ.cu:73-172 and
//              D-GPUGST/src/DPQ.cu:62-126);
//   k_heavy    the arc chunks k_light handed over in the same round (hub
//              vertices of distance items, high-degree DP states), then
//              lower-bound table rows;
//   split      near-far bucketing: far items whose cost entered the new
//              window move to the near list
//   tour       group-to-group distances and tour tables (host DP at
//              DPQ.cu:409-483, re-done on device by one warp)
//   seeds      members at distance 0 (DPQ.cu:359-368); cost-0 states of every
//              subset of a member's group mask (DPQ.cu:341-358)
//   extract    follow parents from the best full state into a tree (the
//              reference's extraction, CPUNONHOP.h:390-432 / CPUHOP.h:234-259,
//              which its GPU path leaves commented out)
#include "gst_device.cuh"

// Round kernels take their tasks by work stealing (1) or by static striding
// (0, the default: on the 170k-vertex power-law workload stealing changed the
// order of the label-correcting distance work enough to add 11% more arc
// relaxations and ran 10% slower).
#ifndef GSTB_STEAL
#define GSTB_STEAL 0
#endif

namespace gstb {

__device__ __forceinline__ uint32_t warp_sum(uint32_t x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
  return x;
}

// Bound-table entries: LB_INF marks a completion that is impossible (a group
// out of reach); finite bounds saturate at LB_INF - 1, which stays a valid
// lower bound.
constexpr uint32_t LB_INF = 0xFFFFu;
__device__ __forceinline__ bool lb_ok(uint32_t cost, uint32_t lb, uint32_t best) {
  return lb != LB_INF && (unsigned long long)cost + lb <= best;
}

// Statistics of the query a warp is working for, kept in shared memory by
// lane 0 and added to the query's counters only when the warp moves to
// another query and at kernel end (one atomic per event would queue on the
// query's control block).
struct WarpStat {
  QCtl* cur;
  uint32_t v[12];
};

__device__ __forceinline__ void ws_init(WarpStat& w) {
  w.cur = nullptr;
#pragma unroll
  for (int i = 0; i < 12; i++) w.v[i] = 0u;
}

__device__ __forceinline__ void ws_flush(WarpStat& w) {
  if (w.cur)
    for (int i = 0; i < 12; i++)
      if (w.v[i]) atomicAdd(&w.cur->stat[i], (unsigned long long)w.v[i]);
#pragma unroll
  for (int i = 0; i < 12; i++) w.v[i] = 0u;
}

// Lane 0 only.
__device__ __forceinline__ void ws_add(WarpStat& w, QCtl* c, int idx, uint32_t val) {
  if (w.cur != c) {
    ws_flush(w);
    w.cur = c;
  }
  w.v[idx] += val;
}

// Warp-local staging of list appends.  The near-out and far entries of one
// query collect in shared memory and reach the global lists in bulk: every
// warp working for a query appends to the same two counters, and one counter
// atomic per flush instead of one per warp step keeps them from queueing.
constexpr uint32_t WBUF = 256;
struct WarpBuf {
  const QDev* q;
  uint32_t nN, nF;
  uint32_t itN[WBUF], itF[WBUF];
};

__device__ __forceinline__ void wb_init(WarpBuf& b) {  // lane 0
  b.q = nullptr;
  b.nN = b.nF = 0u;
}

// Every lane of the warp calls it.
__device__ __forceinline__ void wb_flush(WarpBuf& b, uint32_t lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  __syncwarp();
  const QDev* q = b.q;
  const uint32_t nN = b.nN, nF = b.nF;
  if (q != nullptr && (nN | nF) != 0u) {
    uint32_t bN = 0, bF = 0;
    if (lane == 0) {
      if (nN) bN = atomicAdd(&q->ctl->n_near, nN);
      if (nF) bF = atomicAdd(&q->ctl->n_far, nF);
    }
    bN = __shfl_sync(FULL, bN, 0);
    bF = __shfl_sync(FULL, bF, 0);
    uint32_t* outN = q->qbuf[q->out_idx];
    uint32_t* outF = q->qbuf[q->far_idx];
    const uint32_t cap = q->cap;
    bool ovf = false;
    for (uint32_t i = lane; i < nN; i += 32u) {
      if (bN + i < cap)
        outN[bN + i] = b.itN[i];
      else
        ovf = true;
    }
    for (uint32_t i = lane; i < nF; i += 32u) {
      if (bF + i < cap)
        outF[bF + i] = b.itF[i];
      else
        ovf = true;
    }
    if (__any_sync(FULL, ovf) && lane == 0) atomicExch(&q->ctl->overflow, 1u);
  }
  __syncwarp();
  if (lane == 0) b.nN = b.nF = 0u;
  __syncwarp();
}

// Append up to U items per lane to the near-out and far lists of query q
// through the warp's buffer.  Every lane of the warp calls it; returns this
// lane's number of appended items.
template <int U>
__device__ __forceinline__ uint32_t append_lists(const bool (&takeN)[U], const bool (&takeF)[U],
                                                 const uint32_t (&item)[U], const QDev& q, uint32_t lane,
                                                 WarpBuf& b) {
  const unsigned FULL = 0xFFFFFFFFu;
  uint32_t cN = 0, cF = 0;
#pragma unroll
  for (int u = 0; u < U; u++) {
    cN += takeN[u] ? 1u : 0u;
    cF += takeF[u] ? 1u : 0u;
  }
  if (!__any_sync(FULL, (cN | cF) != 0u)) return 0u;
  uint32_t xN = cN, xF = cF;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yN = __shfl_up_sync(FULL, xN, o), yF = __shfl_up_sync(FULL, xF, o);
    if (lane >= (uint32_t)o) {
      xN += yN;
      xF += yF;
    }
  }
  const uint32_t totN = __shfl_sync(FULL, xN, 31), totF = __shfl_sync(FULL, xF, 31);
  __syncwarp();
  if (b.q != &q || b.nN + totN > WBUF || b.nF + totF > WBUF) {
    wb_flush(b, lane);
    if (lane == 0) b.q = &q;
    __syncwarp();
  }
  const uint32_t oN = b.nN, oF = b.nF;
  uint32_t pN = oN + xN - cN, pF = oF + xF - cF;
#pragma unroll
  for (int u = 0; u < U; u++) {
    if (takeN[u]) b.itN[pN++] = item[u];
    if (takeF[u]) b.itF[pF++] = item[u];
  }
  __syncwarp();
  if (lane == 0) {
    b.nN = oN + totN;
    b.nF = oF + totF;
  }
  __syncwarp();
  return cN + cF;
}

// Enqueue of DP state s at `cost`: the near list when the cost is inside the
// current window, the far list otherwise; a flag bit per state and list
// keeps each list free of duplicates (near entries carry the next round's
// parity).  Every lane calls it (want may be false); returns 1 if this lane
// enqueued.
__device__ __forceinline__ uint32_t enqueue_warp(bool want, uint32_t s, uint32_t cost, const QDev& q, uint32_t lane,
                                                 WarpBuf& b) {
  const bool nearq = cost < q.theta_hi;
  bool take = false;
  if (want) {
    const uint32_t bit = dflag_bit(s, nearq ? (q.par ^ 1u) : 2u);
    take = !(atomicOr(&q.dflag[s >> 3], bit) & bit);
  }
  const bool tN[1] = {take && nearq}, tF[1] = {take && !nearq};
  const uint32_t it[1] = {s};
  return append_lists<1>(tN, tF, it, q, lane, b);
}

// Single-entry push for warps whose lanes may serve different queries
// (split and seed tasks): lanes are aggregated per (query, list) with
// __match_any_sync.  which: 0 = near-out list, 1 = far-out list.
__device__ __forceinline__ void push_multi(bool take, uint32_t item, uint32_t which, const QDev& q, uint32_t slot,
                                           uint32_t lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t key = take ? slot * 2u + which : 0xFFFFFFFFu;
  const unsigned m = __match_any_sync(FULL, key);
  const uint32_t leader = (uint32_t)(__ffs(m) - 1);
  uint32_t base = 0;
  if (take && lane == leader) base = atomicAdd(which == 0u ? &q.ctl->n_near : &q.ctl->n_far2, (uint32_t)__popc(m));
  base = __shfl_sync(FULL, base, leader);
  if (take) {
    const uint32_t pos = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
    uint32_t* buf = which == 0u ? q.qbuf[q.out_idx] : q.qbuf[q.far2_idx];
    if (pos < q.cap)
      buf[pos] = item;
    else
      atomicExch(&q.ctl->overflow, 1u);
  }
}

// Hop-bounded queries: the largest distance from vertex u to a group of comp
// over paths of at most b hops (INF32 if one is out of reach), computed by
// one lane for its own u.  Rows for b hops are the snapshot after round b
// while snapshots were taken, else the final rows; for b = 0 only u itself
// counts (distance 0: u is a member).
__device__ __forceinline__ uint32_t hop_budget_one(const QDev& q, uint32_t u, uint32_t comp, uint32_t b) {
  const uint32_t* row = (b >= 1u && b <= q.snap_n) ? q.snap + ((size_t)(b - 1u) * q.nv + u) * ROW
                                                   : q.dist + (size_t)u * ROW;
  const uint4* r4 = reinterpret_cast<const uint4*>(row);
  const uint4 x = __ldcg(r4), y = __ldcg(r4 + 1);
  const uint32_t r[KMAX] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z};
  uint32_t mx = 0;
#pragma unroll
  for (int j = 0; j < KMAX; j++)
    if (j < q.k && ((comp >> j) & 1u)) {
      const uint32_t d = b == 0u ? (r[j] == 0u ? 0u : INF32) : r[j];
      mx = max(mx, d);
    }
  return mx;
}

// ---------------------------------------------------------------------------
// Grow of one DP state (v, p) -- or (v, p, d) with target hop count d+1 --
// along its arcs [a0, a1): target (u, p[, d+1]) at cost c + w(v, u).  GROW_U
// arcs per lane per step, so every lane keeps GROW_U independent chains
// (arc -> target word and bound -> flag) in flight.  A target is lowered
// with a fire-and-forget 64-bit min after a pre-check against its cost and
// the bound check; its state flag gates the list entry.
// ---------------------------------------------------------------------------
#ifndef GSTB_GROW_U
#define GSTB_GROW_U 4
#endif
constexpr int GROW_U = GSTB_GROW_U;
constexpr uint32_t GROW_LOCAL = 32u * GROW_U;  // arcs a state grows itself; the rest go out in chunks

struct GrowCnt {
  uint32_t arcs = 0, upd = 0, enq = 0;
};

__device__ __forceinline__ void grow_arcs(const QDev& q, const GraphDev& g, uint32_t lane, uint32_t v, uint32_t p,
                                          uint32_t comp, uint32_t c, uint32_t best, uint32_t lim, int dnext,
                                          uint32_t a0, uint32_t a1, GrowCnt& cnt, WarpBuf& wb) {
  const int k = q.k;
  const uint32_t nd = (uint32_t)q.nd, thi = q.theta_hi, par = q.par;
  const unsigned short* __restrict__ lbt = q.lbt;
  for (uint32_t base = a0; base < a1; base += 32u * GROW_U) {
    uint2 arc[GROW_U];
    bool ok[GROW_U];
#pragma unroll
    for (int u = 0; u < GROW_U; u++) {
      const uint32_t a = base + (uint32_t)u * 32u + lane;
      ok[u] = a < a1;
      arc[u] = ok[u] ? __ldg(g.adj + a) : make_uint2(0u, 0u);
    }
    // the target's bound first: it rejects most targets (a neighbour of a
    // hub is rarely close to the missing groups), and only the targets it
    // passes need their 8-byte table word (another random sector)
    uint32_t t[GROW_U], cur[GROW_U], lbu[GROW_U], nc[GROW_U];
    bool want[GROW_U];
#pragma unroll
    for (int u = 0; u < GROW_U; u++) {
      ok[u] = ok[u] && arc[u].y <= lim;
      const uint32_t vp = (arc[u].x << k) | p;
      t[u] = dnext < 0 ? vp : vp * nd + (uint32_t)dnext;
      lbu[u] = ok[u] ? (uint32_t)ld_round(lbt + ((size_t)arc[u].x << k) + comp) : 0u;
    }
    bool any = false;
#pragma unroll
    for (int u = 0; u < GROW_U; u++) {
      nc[u] = c + arc[u].y;
      want[u] = ok[u] && lb_ok(nc[u], lbu[u], best);
      any = any || want[u];
      if (ok[u]) cnt.arcs++;
    }
    if (__any_sync(0xFFFFFFFFu, any)) {
#pragma unroll
      for (int u = 0; u < GROW_U; u++) cur[u] = want[u] ? (uint32_t)(ld_cg(q.table + t[u]) >> 32) : 0u;
#pragma unroll
      for (int u = 0; u < GROW_U; u++) want[u] = want[u] && nc[u] < cur[u];
    }
    if (dnext >= 0) {
      // hop-bounded target (u, p, dnext): its missing groups must stay within
      // the D - dnext hops left from u (the test its expansion would apply);
      // a target that fails is never written, flagged or queued
#pragma unroll
      for (int u = 0; u < GROW_U; u++)
        if (want[u]) {
          const uint32_t h = hop_budget_one(q, arc[u].x, comp, (uint32_t)(q.D - dnext));
          want[u] = h != INF32 && (unsigned long long)nc[u] + h <= best;
        }
    }
#pragma unroll
    for (int u = 0; u < GROW_U; u++) {
      if (want[u]) {
        // the pre-check already saw a higher cost: enqueue on it and let the
        // 64-bit min land without waiting for its result (a concurrent lower
        // write also enqueues; the flag keeps the list free of duplicates)
        red_min(q.table + t[u], pack(nc[u], PAR_GROW | v));
        cnt.upd++;
      }
    }
    // near entries are flagged with the next round's parity, far ones with bit 2
    uint32_t old[GROW_U], bit[GROW_U];
#pragma unroll
    for (int u = 0; u < GROW_U; u++) {
      bit[u] = dflag_bit(t[u], nc[u] < thi ? (par ^ 1u) : 2u);
      old[u] = want[u] ? atomicOr(&q.dflag[t[u] >> 3], bit[u]) : bit[u];
    }
    bool tN[GROW_U], tF[GROW_U];
#pragma unroll
    for (int u = 0; u < GROW_U; u++) {
      const bool take = !(old[u] & bit[u]);
      tN[u] = take && nc[u] < thi;
      tF[u] = take && !(nc[u] < thi);
    }
    cnt.enq += append_lists<GROW_U>(tN, tF, t, q, lane, wb);
  }
}

// A warp hands the arcs [a0, a1) of a state's grow to k_heavy in HUB_CHUNK
// pieces.  Entries below the list's capacity are always written (empty
// ranges when the run does not fit), so k_heavy never reads a stale entry.
// Returns false if the run did not fit: the caller then grows those arcs.
constexpr uint32_t CH_GROW = 1u << 31;  // big-list entry is a DP grow chunk
constexpr uint32_t CH_HOP = 1u << 30;   // ... of a hop-bounded state

__device__ __forceinline__ bool push_grow_chunks(RoundDesc* rd, uint32_t slot, bool hop, uint32_t s, uint32_t a0,
                                                 uint32_t a1, uint32_t lane) {
  const uint32_t nch = (a1 - a0 + HUB_CHUNK - 1u) / HUB_CHUNK;
  uint32_t cb = 0;
  if (lane == 0) cb = atomicAdd(&rd->n_big, nch);
  cb = __shfl_sync(0xFFFFFFFFu, cb, 0);
  const bool fits = cb + nch <= rd->big_cap;
  const uint32_t x = slot | CH_GROW | (hop ? CH_HOP : 0u);
  for (uint32_t c = lane; c < nch && cb + c < rd->big_cap; c += 32u) {
    const uint32_t s0 = a0 + c * HUB_CHUNK;
    rd->big[cb + c] = fits ? make_uint4(x, s, s0, min(s0 + HUB_CHUNK, a1)) : make_uint4(slot, 0u, 0u, 0u);
  }
  return fits;
}

// Load the capped group distances of vertex v into every lane's registers.
__device__ __forceinline__ void load_dl(const QDev& q, uint32_t v, uint32_t (&dl)[KMAX],
                                        uint32_t& raw_sum_ok, uint32_t comp,
                                        unsigned long long& raw_sum) {
  const uint4* row = reinterpret_cast<const uint4*>(q.dist + (size_t)v * 8);
  uint4 a = ld_round(row), b = ld_round(row + 1);
  uint32_t r[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  raw_sum = 0;
  raw_sum_ok = 1;
#pragma unroll
  for (int j = 0; j < KMAX; j++) {
    dl[j] = min(r[j], q.cap1);
    if (j < q.k && (comp >> j & 1u)) {
      if (r[j] == INF32) raw_sum_ok = 0;
      raw_sum += r[j];
    }
  }
}

// Slot owning flat item `it` of task type t: largest s with pre[s] <= it.
__device__ __forceinline__ uint32_t find_slot(const uint32_t* __restrict__ pre, int nslots, uint32_t it) {
  int lo = 0, hi = nslots;  // pre[lo] <= it < pre[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (__ldcg(pre + mid) <= it)
      lo = mid;
    else
      hi = mid;
  }
  return (uint32_t)lo;
}

// Same search over a prefix array staged in shared memory.
__device__ __forceinline__ uint32_t find_slot_s(const uint32_t* pre, int nslots, uint32_t it) {
  int lo = 0, hi = nslots;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (pre[mid] <= it)
      lo = mid;
    else
      hi = mid;
  }
  return (uint32_t)lo;
}

// A DP state's vertex row staged for its merges: the costs of its 2^k table
// entries and its 2^k bound-table entries.
struct MergeTile {
  uint32_t cost[1u << KMAX];
  unsigned short lb[1u << KMAX];
};

// ---------------------------------------------------------------------------
// Unbounded DP item (v, p), in two parts.  dp_gate runs on one lane for its
// own item: it takes the item out of the near list, drops it when its cost
// is above the incumbent, updates the incumbent from the complement merge
// and the one-label completion, and applies the bound; dp_expand then grows
// and merges the surviving state with the whole warp.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool dp_gate(const QDev& q, uint32_t s, uint32_t& c_out, uint32_t& best_out,
                                        bool& counted) {
  const int k = q.k;
  const uint32_t K2 = 1u << k, full = (uint32_t)q.full;
  const uint32_t v = s >> k, p = s & (K2 - 1u);
  counted = false;
  atomicAnd(&q.dflag[s >> 3], ~dflag_bit(s, q.par));
  const uint32_t c = (uint32_t)(ld_cg(q.table + s) >> 32);
  uint32_t best = ld_best(q.ctl);
  if (c == INF32 || c > best) return false;
  unsigned long long* row = q.table + (size_t)v * K2;
  if (p == full) {
    if (c < best) atomicMin(&q.ctl->best, c);
    return false;
  }
  const uint32_t comp = full ^ p;
  uint32_t dl[KMAX], sum_ok;
  unsigned long long raw_sum;
  load_dl(q, v, dl, sum_ok, comp, raw_sum);
  // complement merge straight into the full state (DPQ.cu:82-94); a full
  // state of cost equal to best is still recorded: best may come from a
  // bound-only tree (star or one-label) that has no table entry
  const uint32_t cc = (uint32_t)(ld_cg(row + comp) >> 32);
  if (cc != INF32) {
    const unsigned long long m = (unsigned long long)c + cc;
    if (m <= best) {
      atomicMin(row + full, pack((uint32_t)m, PAR_MERGE | p));
      atomicMin(&q.ctl->best_full, (m << 32) | v);
      if (m < best) {
        atomicMin(&q.ctl->best, (uint32_t)m);
        best = (uint32_t)m;
      }
    }
  }
  // one-label completion: T(v,p) plus shortest paths to the missing groups
  // (DPQ.cu:95-107, CPUNONHOP.h:684-699)
  if (sum_ok) {
    const unsigned long long ol = (unsigned long long)c + raw_sum;
    if (ol < best) {
      atomicMin(&q.ctl->best, (uint32_t)ol);
      best = (uint32_t)ol;
    }
  }
  counted = true;
  const uint32_t lbv = ld_round(q.lbt + ((size_t)v << k) + comp);
  c_out = c;
  best_out = best;
  return lb_ok(c, lbv, best);
}

__device__ void dp_expand(const QDev& q, const GraphDev& g, uint32_t s, uint32_t c, uint32_t best, uint32_t lane,
                          RoundDesc* __restrict__ rd, uint32_t slot, WarpStat& ws, WarpBuf& wb, MergeTile* mt) {
  const int k = q.k;
  const uint32_t K2 = 1u << k, full = (uint32_t)q.full;
  const uint32_t v = s >> k, p = s & (K2 - 1u), comp = full ^ p;
  unsigned long long* row = q.table + (size_t)v * K2;
  const unsigned short* lbt = q.lbt;
  GrowCnt gc;
  // grow, only from states of cost <= best/2 (optimal-tree decomposition,
  // CPUNONHOP.h:820; exact for the unbounded problem); a high-degree vertex
  // grows its first GROW_LOCAL arcs here and hands the rest to k_heavy
  if (2ull * c <= best) {
    const uint32_t lim = best - c;
    const uint32_t a0 = __ldg(g.beg + v);
    uint32_t a1 = arcs_upto(g, v, __ldg(g.beg + v + 1), lim);
    if (rd->grow_chunks && a1 - a0 >= rd->hub_min_deg &&
        push_grow_chunks(rd, slot, false, s, a0 + GROW_LOCAL, a1, lane))
      a1 = a0 + GROW_LOCAL;
    grow_arcs(q, g, lane, v, p, comp, c, best, lim, -1, a0, a1, gc, wb);
  }
  // merge with every proper, non-empty subset p2 of the complement
  // (DPQ.cu:140-170; the complement itself went to the full state above).
  // Lane j takes the subsets idx = j, j+32, .. (p2 = the idx+1-th subset of
  // the complement, by bit deposit); a state with many partners first stages
  // its vertex's costs and bound row in shared memory with coalesced loads,
  // so every partner is read from there.  A staged cost can be higher than
  // the table's by then (another warp lowered it): a partner missed that way
  // merges with this state when it is expanded itself, and a target whose
  // cost only looked higher gets a min that changes nothing.
  uint32_t merges = 0;
  {
    const uint32_t nsub = (1u << __popc(comp)) - 2u;
    const bool staged = mt != nullptr && rd->merge_stage != 0u && nsub >= rd->merge_stage;
    if (staged) {
      for (uint32_t i = lane; i < K2; i += 32u) {
        mt->cost[i] = (uint32_t)(ld_cg(row + i) >> 32);
        mt->lb[i] = ld_round(lbt + ((size_t)v << k) + i);
      }
      __syncwarp();
    }
    for (uint32_t b = 0; b < nsub; b += 32) {
      uint32_t idx = b + lane;
      bool want = false;
      uint32_t t = 0, m32 = 0;
      if (idx < nsub) {
        uint32_t p2 = pdep(idx + 1u, comp);
        uint32_t qset = p | p2;
        uint32_t c2 = staged ? mt->cost[p2] : (uint32_t)(ld_cg(row + p2) >> 32);
        uint32_t cq = staged ? mt->cost[qset] : (uint32_t)(ld_cg(row + qset) >> 32);
        if (c2 != INF32) {
          merges++;
          unsigned long long m = (unsigned long long)c + c2;
          // conditional tree merging: 3m <= 2 best (CPUNONHOP.h:941)
          if (3ull * m <= 2ull * best && m < cq) {
            uint32_t lbq = staged ? (uint32_t)mt->lb[full ^ qset] : ld_round(lbt + ((size_t)v << k) + (full ^ qset));
            if (lb_ok((uint32_t)m, lbq, best)) {
              m32 = (uint32_t)m;
              t = (v << k) | qset;
              red_min(q.table + t, pack(m32, PAR_MERGE | p));
              want = true;
              gc.upd++;
            }
          }
        }
      }
      gc.enq += enqueue_warp(want, t, m32, q, lane, wb);
    }
    if (staged) __syncwarp();  // the tile is free for the next state
  }
  const uint32_t sa = warp_sum(gc.arcs), su = warp_sum(gc.upd), se = warp_sum(gc.enq), sm = warp_sum(merges);
  if (lane == 0) {
    ws_add(ws, q.ctl, ST_ARCS, sa);
    ws_add(ws, q.ctl, ST_UPDATES, su);
    ws_add(ws, q.ctl, ST_ENQ, se);
    ws_add(ws, q.ctl, ST_MERGES, sm);
  }
}

// ---------------------------------------------------------------------------
// Hop-bounded DP item (v, p, d): state id ((v << k) | p) * nd + d; gate on
// one lane, expansion by the warp, as for the unbounded items.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool hop_gate(const QDev& q, uint32_t s, uint32_t& c_out, uint32_t& best_out,
                                         bool& counted) {
  const int k = q.k, nd = q.nd, D = q.D;
  const uint32_t K2 = 1u << k, full = (uint32_t)q.full;
  const uint32_t d = s % (uint32_t)nd, vp = s / (uint32_t)nd;
  const uint32_t v = vp >> k, p = vp & (K2 - 1u);
  counted = false;
  atomicAnd(&q.dflag[s >> 3], ~dflag_bit(s, q.par));
  const uint32_t c = (uint32_t)(ld_cg(q.table + s) >> 32);
  const uint32_t best = ld_best(q.ctl);
  if (c == INF32 || c > best) return false;
  // dominance: the same subset at a smaller hop count and no higher cost
  for (uint32_t e = 0; e < d; e++)
    if ((uint32_t)(ld_cg(q.table + (size_t)vp * nd + e) >> 32) <= c) return false;
  if (p == full) {
    if (c < best) atomicMin(&q.ctl->best, c);
    return false;
  }
  const uint32_t comp = full ^ p;
  // In a derivation of a tree of hop diameter <= D from (v, p, d), a group
  // missing from p is reached from v by a path outside the subtree, and that
  // path plus the subtree's height d is a path of the tree: it has at most
  // D - d hops.  So the missing groups must be within D - d hops of v.
  const uint32_t lbh = hop_budget_one(q, v, comp, (uint32_t)D - d);
  if (lbh == INF32 || (unsigned long long)c + lbh > best) return false;
  counted = true;
  const uint32_t lbv = ld_round(q.lbt + ((size_t)v << k) + comp);
  c_out = c;
  best_out = best;
  return lb_ok(c, lbv, best);
}

__device__ void hop_expand(const QDev& q, const GraphDev& g, uint32_t s, uint32_t c, uint32_t best, uint32_t lane,
                           RoundDesc* __restrict__ rd, uint32_t slot, WarpStat& ws, WarpBuf& wb) {
  const int k = q.k, nd = q.nd, D = q.D;
  const uint32_t K2 = 1u << k, full = (uint32_t)q.full;
  const uint32_t d = s % (uint32_t)nd, vp = s / (uint32_t)nd;
  const uint32_t v = vp >> k, p = vp & (K2 - 1u), comp = full ^ p;
  const unsigned short* lbt = q.lbt;
  GrowCnt gc;
  if (d < (uint32_t)D) {  // grow d -> d+1 (CPUHOP.h:192-206)
    const uint32_t lim = best - c;
    const uint32_t a0 = __ldg(g.beg + v);
    uint32_t a1 = arcs_upto(g, v, __ldg(g.beg + v + 1), lim);
    if (rd->grow_chunks && a1 - a0 >= rd->hub_min_deg &&
        push_grow_chunks(rd, slot, true, s, a0 + GROW_LOCAL, a1, lane))
      a1 = a0 + GROW_LOCAL;
    grow_arcs(q, g, lane, v, p, comp, c, best, lim, (int)d + 1, a0, a1, gc, wb);
  }
  // merge with (v, p2, d2), p2 a non-empty subset of the complement,
  // d2 <= D - d, into (v, p|p2, max(d, d2))  (CPUHOP.h:208-227)
  uint32_t merges = 0;
  {
    const uint32_t nsub = (1u << __popc(comp)) - 1u;
    const uint32_t nd2 = (uint32_t)D - d + 1u;
    const uint32_t npairs = nsub * nd2;
    unsigned long long* rowv = q.table + ((size_t)v << k) * nd;
    for (uint32_t b = 0; b < npairs; b += 32) {
      uint32_t idx = b + lane;
      bool want = false;
      uint32_t t = 0, m32 = 0;
      if (idx < npairs) {
        uint32_t p2 = pdep(idx / nd2 + 1u, comp);
        uint32_t d2 = idx % nd2;
        uint32_t c2 = (uint32_t)(ld_cg(rowv + (size_t)p2 * nd + d2) >> 32);
        if (c2 != INF32) {
          merges++;
          unsigned long long m = (unsigned long long)c + c2;
          uint32_t qset = p | p2;
          uint32_t ndd = max(d, d2);
          uint32_t par = PAR_MERGE | p | (d << 8) | (d2 << 11);
          if (m <= best) {
            m32 = (uint32_t)m;
            t = ((v << k) | qset) * (uint32_t)nd + ndd;
            if (qset == full) {
              // recorded at cost == best too: best may come from a tree
              // that has no table entry
              atomicMin(q.table + t, pack(m32, par));
              atomicMin(&q.ctl->best_full, ((unsigned long long)m32 << 32) | (v * 8u + ndd));
              if (m32 < best) atomicMin(&q.ctl->best, m32);
            } else {
              uint32_t lbq = ld_round(lbt + ((size_t)v << k) + (full ^ qset));
              if (lb_ok(m32, lbq, best) && m32 < (uint32_t)(ld_cg(q.table + t) >> 32)) {
                red_min(q.table + t, pack(m32, par));
                want = true;
                gc.upd++;
              }
            }
          }
        }
      }
      gc.enq += enqueue_warp(want, t, m32, q, lane, wb);
    }
  }
  const uint32_t sa = warp_sum(gc.arcs), su = warp_sum(gc.upd), se = warp_sum(gc.enq), sm = warp_sum(merges);
  if (lane == 0) {
    ws_add(ws, q.ctl, ST_ARCS, sa);
    ws_add(ws, q.ctl, ST_UPDATES, su);
    ws_add(ws, q.ctl, ST_ENQ, se);
    ws_add(ws, q.ctl, ST_MERGES, sm);
  }
}

// A DP task: W items (one per lane) of the round's DP or hop-bounded list.
// Each lane runs its item's gates; then the warp expands the surviving
// states one after another.  W is chosen per round by k_control (1 when the
// round has few items, so that each state gets a warp of its own; up to 32
// when it has many, most of which the gates drop).
__device__ void dp_task(const QDev* qd, const uint32_t* __restrict__ pre, int nslots, uint32_t total,
                        uint32_t task, uint32_t W, bool hop, const GraphDev& g, uint32_t lane,
                        RoundDesc* __restrict__ rd, WarpStat& ws, WarpBuf& wb, MergeTile* mt) {
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t it = task * W + lane;
  const bool valid = lane < W && it < total;
  uint32_t slot = 0xFFFFFFFFu, s = 0, c = 0, best = 0;
  bool live = false, counted = false;
  if (valid) {
    slot = find_slot_s(pre, nslots, it);
    const QDev& q = qd[slot];
    s = q.qbuf[q.in_idx][it - pre[slot]];
    live = hop ? hop_gate(q, s, c, best, counted) : dp_gate(q, s, c, best, counted);
  }
  // expanded-state counts, per query of the task
  unsigned cm = __ballot_sync(FULL, counted);
  while (cm) {
    const uint32_t si = __shfl_sync(FULL, slot, __ffs(cm) - 1);
    const unsigned same = __ballot_sync(FULL, counted && slot == si);
    if (lane == 0) ws_add(ws, qd[si].ctl, ST_EXPANDED, __popc(same));
    cm &= ~same;
  }
  unsigned lm = __ballot_sync(FULL, live);
  while (lm) {
    const uint32_t i = __ffs(lm) - 1;
    lm &= lm - 1u;
    const uint32_t si = __shfl_sync(FULL, slot, i), ss = __shfl_sync(FULL, s, i);
    const uint32_t cc = __shfl_sync(FULL, c, i), bb = __shfl_sync(FULL, best, i);
    const QDev& q = qd[si];
    if (hop)
      hop_expand(q, g, ss, cc, bb, lane, rd, si, ws, wb);
    else
      dp_expand(q, g, ss, cc, bb, lane, rd, si, ws, wb, mt);
  }
}

// Next task of a warp.  Each warp's first task is its own index; after that
// the warps take tasks from a shared counter (work stealing), so a warp that
// met cheap tasks keeps taking new ones while one with a long task (a hub
// vertex, a state with many merge partners) is still busy.
__device__ __forceinline__ uint32_t next_task(uint32_t* counter, uint32_t nwarps, uint32_t lane) {
  uint32_t t = 0;
  if (lane == 0) t = nwarps + atomicAdd(counter, 1u);
  return __shfl_sync(0xFFFFFFFFu, t, 0);
}

// ---------------------------------------------------------------------------
// Distance items.  A warp task holds W items (a vertex with the mask of its
// pending groups); W is chosen per round by k_control: 4 when the round has
// few items (short rounds, low latency), up to 32 when it has many (fewer
// per-task overheads).  Lanes 0..W-1 read the items' headers in parallel;
// then the arcs of all items of one query in the task are relaxed as one flat
// list, 32 x SSSP_U arcs per step.  Each lane keeps SSSP_U independent chains
// (arc -> distance row -> pending flag) in flight, and uneven degrees are
// spread over all 32 lanes.
// ---------------------------------------------------------------------------
constexpr uint32_t SSSP_WMAX = 32;   // most items per warp task
#ifndef GSTB_SSSP_U
#define GSTB_SSSP_U 4
#endif
constexpr int SSSP_U = GSTB_SSSP_U;  // arcs per lane per step
constexpr uint32_t HUB_LOCAL = 32;   // arcs of a hub item its own task relaxes

struct alignas(16) RelaxHdr {
  uint32_t d[KMAX];  // group distances at the item's vertex
  uint32_t rm;       // groups to relax from it
  uint32_t lim;      // largest arc weight that can still lower a distance
  uint32_t a0;       // first arc to relax
  uint32_t pad;
};

struct RelaxCnt {
  uint32_t arcs = 0, upd = 0, enq = 0;
};

// Per-warp shared scratch; a warp uses one member at a time: the headers of
// its distance items (or of a hub chunk), its bound rows' capped distances,
// or a DP state's merge tile.
union WarpScratch {
  RelaxHdr hdr[32];
  uint32_t dl[KMAX][32];
  MergeTile mg;
};

__device__ __forceinline__ uint32_t sel8(const uint4& a, const uint4& b, uint32_t i) {
  const uint4& h = i < 4u ? a : b;
  const uint32_t j = i & 3u;
  return j == 0u ? h.x : (j == 1u ? h.y : (j == 2u ? h.z : h.w));
}

// Relax the arcs of the task's items [i0, i1), all of query q.  Lane j holds
// in `x` the inclusive prefix n_0 + ... + n_j of the task's arc counts; item
// i's arcs are [h[i].a0, h[i].a0 + n_i).  Every lane of the warp calls it with
// the same i0, i1.  A lowered distance is written with a fire-and-forget
// atomicMin after a pre-check; the pending-groups flag of the target gates
// its list entry (parity-split flags, so no update is lost); appends are
// aggregated over the whole warp.
__device__ __forceinline__ void relax_flat(const QDev& q, const RelaxHdr* __restrict__ h, uint32_t x, uint32_t i0,
                                           uint32_t i1, uint32_t capb, const GraphDev& g, uint32_t lane,
                                           RelaxCnt& cnt, WarpBuf& wb) {
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t lo_end = __shfl_sync(FULL, x, i0 == 0u ? 0u : i0 - 1u);
  const uint32_t f0 = i0 == 0u ? 0u : lo_end;
  const uint32_t f1 = __shfl_sync(FULL, x, i1 - 1u);
  const uint32_t thi = q.theta_hi, nsh = near_sh(q.par ^ 1u);
  uint32_t* __restrict__ dist = q.dist_nx;  // targets: the rows this round writes

  for (uint32_t base = f0; base < f1; base += 32u * SSSP_U) {
    uint2 arc[SSSP_U];
    uint32_t itm[SSSP_U], lim[SSSP_U];
    bool ok[SSSP_U];
#pragma unroll
    for (int u = 0; u < SSSP_U; u++) {
      const uint32_t f = base + (uint32_t)u * 32u + lane;
      // item of flat position f: the first i in [i0, i1) with x_i > f
      // (binary lifting over the lanes' prefixes)
      uint32_t pos = i0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t cand = pos + step - 1u;
        const uint32_t xc = __shfl_sync(FULL, x, min(cand, 31u));
        if (cand < i1 && xc <= f) pos += step;
      }
      const uint32_t xs = __shfl_sync(FULL, x, pos == 0u ? 0u : min(pos - 1u, 31u));
      const uint32_t start = pos == 0u ? 0u : xs;
      ok[u] = f < f1;
      itm[u] = ok[u] ? pos : i0;
      // the item's weight limit and first arc in one 8-byte shared load
      const uint2 la = *reinterpret_cast<const uint2*>(&h[itm[u]].lim);
      lim[u] = la.x;
      arc[u] = ok[u] ? __ldg(g.adj + la.y + (f - start)) : make_uint2(0u, 0u);
    }
    uint4 ra[SSSP_U], rb[SSSP_U];
#pragma unroll
    for (int u = 0; u < SSSP_U; u++) {
      ok[u] = ok[u] && arc[u].y <= lim[u];
      if (ok[u]) {
        const uint4* row = reinterpret_cast<const uint4*>(dist + (size_t)arc[u].x * 8);
        ra[u] = __ldcg(row);
        rb[u] = __ldcg(row + 1);
      } else {
        ra[u] = rb[u] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    uint32_t nn[SSSP_U], nf[SSSP_U];
#pragma unroll
    for (int u = 0; u < SSSP_U; u++) {
      nn[u] = nf[u] = 0u;
      if (ok[u]) {
        cnt.arcs++;
        // the item's distances and group mask in two 16-byte shared loads
        const uint4* hv = reinterpret_cast<const uint4*>(&h[itm[u]]);
        const uint4 h0 = hv[0], h1 = hv[1];
        const uint32_t rm = h1.w;
        const uint32_t dv[KMAX] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z};
        const uint32_t du[KMAX] = {ra[u].x, ra[u].y, ra[u].z, ra[u].w, rb[u].x, rb[u].y, rb[u].z};
#pragma unroll
        for (int t = 0; t < KMAX; t++) {
          if ((rm >> t) & 1u) {
            const uint32_t dt = dv[t];
            const uint32_t nd = dt + arc[u].y;
            if (nd >= dt && nd <= capb && nd < du[t]) {
              red_min(dist + (size_t)arc[u].x * ROW + t, nd);
              if (nd < thi)
                nn[u] |= 1u << t;
              else
                nf[u] |= 1u << t;
              cnt.upd++;
            }
          }
        }
      }
    }
    // flags: one fire-and-forget OR per target for both lists, skipped when
    // the row just read shows the bits set already.  The list entry is taken
    // when that row showed the list's byte empty.  Within a round the
    // next-parity and far bytes only gain bits, so the first OR to reach a
    // byte comes from a lane that read it empty: every newly pending vertex
    // is appended at least once.  Two lanes that both read it empty append
    // it twice; the consumer's atomicAnd hands the groups to one of them
    // and the other finds none.  No lane waits for an atomic's result.
    uint32_t itv[SSSP_U];
    bool tN[SSSP_U], tF[SSSP_U];
#pragma unroll
    for (int u = 0; u < SSSP_U; u++) {
      const uint32_t bits = (nn[u] << nsh) | (nf[u] << FAR_SH);
      // (exact rounds compare with the written row, the running minimum of
      // the round: it filters repeated relaxations of a target far better
      // than the previous round's row, at the price of a few entries for
      // vertices whose own new value has not been carried across yet)
      const uint32_t fw = rb[u].w;
      if (bits & ~fw) red_or(dist + (size_t)arc[u].x * ROW + FLAGW, bits);
      tN[u] = nn[u] && ((fw >> nsh) & 0xFFu) == 0u;
      tF[u] = nf[u] && ((fw >> FAR_SH) & 0xFFu) == 0u;
      itv[u] = arc[u].x;
    }
    cnt.enq += append_lists<SSSP_U>(tN, tF, itv, q, lane, wb);
  }
}

// Warp-reduce a relaxation's counters into the warp's statistics.
__device__ __forceinline__ void relax_cnt_add(WarpStat& ws, QCtl* c, RelaxCnt cnt, uint32_t items, uint32_t lane) {
  const uint32_t a = warp_sum(cnt.arcs), u = warp_sum(cnt.upd), e = warp_sum(cnt.enq);
  if (lane == 0) {
    ws_add(ws, c, ST_SSSP, items);
    ws_add(ws, c, ST_SSSP_ARCS, a);
    ws_add(ws, c, ST_SSSP_UPDATES, u);
    ws_add(ws, c, ST_SSSP_ENQ, e);
  }
}

__device__ void sssp_task(const QDev* qd, const uint32_t* __restrict__ pre, int nslots,
                          uint32_t total, uint32_t task, uint32_t W, const GraphDev& g, uint32_t lane, WarpStat& ws,
                          RoundDesc* __restrict__ rd, RelaxHdr* __restrict__ sh, WarpBuf& wb) {
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t it = task * W + lane;
  const bool valid = lane < W && it < total;
  const uint32_t slot = valid ? find_slot_s(pre, nslots, it) : 0xFFFFFFFFu;
  uint32_t n = 0, capb = INF32;
  bool active = false;
  if (valid) {
    const QDev& q = qd[slot];
    const int k = q.k;
    const uint32_t v = q.qbuf[q.in_idx][it - pre[slot]];
    // the header's loads depend on v only, so they are all in flight at once;
    // take the groups pending at v for this round's parity
    const uint32_t psh = near_sh(q.par);
    const uint32_t m =
        (atomicAnd(q.dist + (size_t)v * ROW + FLAGW, ~(0xFFu << psh)) >> psh) & 0xFFu;
    const uint4* drow = reinterpret_cast<const uint4*>(q.dist + (size_t)v * ROW);
    const uint4 da = __ldcg(drow), db = __ldcg(drow + 1);
    uint32_t best = ld_best(q.ctl);
    const uint32_t b0 = __ldg(g.beg + v), b1 = __ldg(g.beg + v + 1);
    uint4 wa = make_uint4(b1, b1, b1, b1), wb = wa;
    if (g.wcut != nullptr) {
      const uint4* wr = reinterpret_cast<const uint4*>(g.wcut + (size_t)v * 8);
      wa = __ldg(wr);
      wb = __ldg(wr + 1);
    }
    const uint32_t d[KMAX] = {da.x, da.y, da.z, da.w, db.x, db.y, db.z};
    if (q.dist_nx != q.dist) {
      // exact rounds: the distances that changed last round carry over into
      // the rows this round writes (the other rows hold them already)
      uint32_t* nx = q.dist_nx + (size_t)v * ROW;
#pragma unroll
      for (int t = 0; t < KMAX; t++)
        if (t < k && ((m >> t) & 1u)) red_min(nx + t, d[t]);
    }
    // star bound at v (unbounded queries only): v joined to every group by
    // shortest paths is a feasible tree (one-label completion, CPUNONHOP.h:684-699)
    if (q.D < 0) {
      unsigned long long sum = 0;
      bool fin = true;
#pragma unroll
      for (int t = 0; t < KMAX; t++)
        if (t < k) {
          fin = fin && d[t] != INF32;
          sum += d[t];
        }
      if (fin && sum < best) {
        atomicMin(&q.ctl->best, (uint32_t)sum);
        best = (uint32_t)sum;
      }
    }
    // distances beyond cap(best) cannot lower a bound below best: skip them
    capb = (uint32_t)((unsigned long long)best * q.cap_num / q.cap_den);
    uint32_t rm = 0, dmin = INF32;
#pragma unroll
    for (int t = 0; t < KMAX; t++)
      if (t < k && ((m >> t) & 1u) && d[t] <= capb) {
        rm |= 1u << t;
        dmin = min(dmin, d[t]);
      }
    active = rm != 0;
    uint32_t lim = 0;
    if (active) {
      lim = capb - dmin;
      uint32_t a1 = b1;
      if (g.wcut != nullptr && lim <= 128u) a1 = sel8(wa, wb, lim <= 1u ? 0u : 32u - __clz(lim - 1u));
      n = a1 - b0;
      // hub: hand all but the first HUB_LOCAL arcs to k_heavy in chunks of
      // HUB_CHUNK arcs, one warp each
      if (n >= rd->hub_deg && n - HUB_LOCAL >= rd->hub_min_rest) {
        const uint32_t st0 = b0 + HUB_LOCAL;
        const uint32_t nch = (a1 - st0 + HUB_CHUNK - 1u) / HUB_CHUNK;
        const uint32_t cb = atomicAdd(&rd->n_big, nch);
        const bool fits = cb + nch <= rd->big_cap;
        // entries below the cap are always written (empty ranges when the
        // whole run does not fit) so k_heavy never reads a stale entry
        for (uint32_t c = 0; c < nch && cb + c < rd->big_cap; c++) {
          const uint32_t s0 = st0 + c * HUB_CHUNK;
          rd->big[cb + c] = fits ? make_uint4(slot | (rm << 16), v, s0, min(s0 + HUB_CHUNK, a1))
                                 : make_uint4(slot, v, 0u, 0u);
        }
        if (fits) n = HUB_LOCAL;
      }
    }
    RelaxHdr hd;
#pragma unroll
    for (int t = 0; t < KMAX; t++) hd.d[t] = d[t];
    hd.rm = rm;
    hd.lim = lim;
    hd.a0 = b0;
    hd.pad = 0;
    sh[lane] = hd;
  }
  __syncwarp();
  // valid items are lanes [0, nvalid); split them into runs of one query
  const unsigned vmask = __ballot_sync(FULL, valid);
  if (vmask == 0u) return;
  const uint32_t nvalid = 32u - __clz(vmask);
  uint32_t x = n;  // inclusive prefix of the arc counts over the lanes
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  const uint32_t prev_slot = __shfl_up_sync(FULL, slot, 1);
  unsigned runs = __ballot_sync(FULL, valid && (lane == 0u || prev_slot != slot));
  const unsigned amask = __ballot_sync(FULL, active);
  while (runs) {
    const uint32_t i0 = (uint32_t)(__ffs(runs) - 1);
    runs &= runs - 1u;
    const uint32_t i1 = runs ? (uint32_t)(__ffs(runs) - 1) : nvalid;
    const uint32_t si = __shfl_sync(FULL, slot, i0);
    const bool in_run = lane >= i0 && lane < i1;
    uint32_t cb = in_run ? capb : INF32;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cb = min(cb, __shfl_xor_sync(FULL, cb, o));
    const unsigned rmask = (i1 >= 32u ? 0xFFFFFFFFu : ((1u << i1) - 1u)) & ~((1u << i0) - 1u);
    const uint32_t n_items = __popc(amask & rmask);
    const QDev& q = qd[si];
    RelaxCnt cnt;
    relax_flat(q, sh, x, i0, i1, cb, g, lane, cnt, wb);
    relax_cnt_add(ws, q.ctl, cnt, n_items, lane);
  }
}

// One hub chunk (k_heavy, one warp): relax arcs [first, end) of vertex v for
// the pending groups recorded by k_light.  Same relaxation as sssp_task.
__device__ void hub_chunk(const QDev* qd, const uint4 item, const GraphDev& g, uint32_t lane,
                          RelaxHdr* __restrict__ sh, WarpStat& ws, WarpBuf& wb) {
  const unsigned FULL = 0xFFFFFFFFu;
  if (item.z >= item.w) return;  // filler entry of a chunk run that did not fit
  const uint32_t slot = item.x & 0xFFFFu, v = item.y;
  const QDev& q = qd[slot];
  uint32_t capb = 0, n = 0;
  if (lane == 0) {
    const uint4* drow = reinterpret_cast<const uint4*>(q.dist + (size_t)v * ROW);
    const uint4 da = __ldcg(drow), db = __ldcg(drow + 1);
    const uint32_t best = ld_best(q.ctl);
    const uint32_t d[KMAX] = {da.x, da.y, da.z, da.w, db.x, db.y, db.z};
    capb = (uint32_t)((unsigned long long)best * q.cap_num / q.cap_den);
    uint32_t rm = 0, dmin = INF32;
#pragma unroll
    for (int t = 0; t < KMAX; t++)
      if (((item.x >> (16 + t)) & 1u) && d[t] <= capb) {
        rm |= 1u << t;
        dmin = min(dmin, d[t]);
      }
    RelaxHdr hd;
#pragma unroll
    for (int t = 0; t < KMAX; t++) hd.d[t] = d[t];
    hd.rm = rm;
    hd.lim = rm ? capb - dmin : 0u;
    hd.a0 = item.z;
    hd.pad = 0;
    sh[0] = hd;
    n = rm ? item.w - item.z : 0u;
  }
  __syncwarp();
  capb = __shfl_sync(FULL, capb, 0);
  n = __shfl_sync(FULL, n, 0);
  if (n == 0) return;
  RelaxCnt cnt;
  relax_flat(q, sh, n, 0u, 1u, capb, g, lane, cnt, wb);  // one item: every lane holds its prefix n
  relax_cnt_add(ws, q.ctl, cnt, 0u, lane);
}

// One DP grow chunk (k_heavy, one warp): arcs [first, end) of a state that a
// k_light warp handed over.  The state's current cost is read again (it can
// only have dropped, and a lower cost grows validly too) and the gates of the
// state's own expansion are re-checked.
__device__ void grow_chunk(const QDev* qd, const uint4 item, const GraphDev& g, uint32_t lane,
                           WarpStat& ws, WarpBuf& wb) {
  const unsigned FULL = 0xFFFFFFFFu;
  if (item.z >= item.w) return;  // filler entry of a chunk run that did not fit
  const uint32_t slot = item.x & 0xFFFFu;
  const bool hop = (item.x & CH_HOP) != 0u;
  const QDev& q = qd[slot];
  const int k = q.k;
  const uint32_t K2 = 1u << k, full = (uint32_t)q.full, nd = (uint32_t)q.nd, s = item.y;
  const uint32_t vp = hop ? s / nd : s, d = hop ? s % nd : 0u;
  const uint32_t v = vp >> k, p = vp & (K2 - 1u), comp = full ^ p;
  uint32_t c = 0, best = 0, lbv = 0;
  if (lane == 0) {
    c = (uint32_t)(ld_cg(q.table + s) >> 32);
    best = ld_best(q.ctl);
    lbv = ld_round(q.lbt + ((size_t)v << k) + comp);
  }
  c = __shfl_sync(FULL, c, 0);
  best = __shfl_sync(FULL, best, 0);
  lbv = __shfl_sync(FULL, lbv, 0);
  if (c == INF32 || c > best || !lb_ok(c, lbv, best)) return;
  if (!hop && 2ull * c > best) return;
  GrowCnt gc;
  grow_arcs(q, g, lane, v, p, comp, c, best, best - c, hop ? (int)d + 1 : -1, item.z, item.w, gc, wb);
  const uint32_t a = warp_sum(gc.arcs), u = warp_sum(gc.upd), e = warp_sum(gc.enq);
  if (lane == 0) {
    ws_add(ws, q.ctl, ST_ARCS, a);
    ws_add(ws, q.ctl, ST_UPDATES, u);
    ws_add(ws, q.ctl, ST_ENQ, e);
  }
}

// Near-far split of one far item: cost in [theta_lo, theta_hi) -> near list;
// above -> far-out list; below theta_lo it was already expanded at that cost
// (every new cost is >= the cost of the item that produced it) -> dropped.
// Distance items are vertices with a mask of pending groups; DP items are
// states.  Items moved to the near list carry the parity of the next round.
// The caller pushes `s` to the near-out list if toN and to the far-out list
// if toF (push_multi, warp-aggregated).
__device__ void split_item(const QDev& q, uint32_t s, bool& toN, bool& toF) {
  uint32_t best = ld_cg(&q.ctl->best);
  toN = toF = false;
  if (q.phase == PH_SSSP) {
    uint32_t* fw = q.dist + (size_t)s * ROW + FLAGW;
    const uint32_t capb = (uint32_t)((unsigned long long)best * q.cap_num / q.cap_den);
    const uint32_t fm = (atomicAnd(fw, ~(0xFFu << FAR_SH)) >> FAR_SH) & 0xFFu;
    uint32_t nb = 0, kb = 0;
    for (int t = 0; t < q.k; t++) {
      if (!((fm >> t) & 1u)) continue;
      uint32_t d = ld_cg(q.dist + (size_t)s * ROW + t);
      if (d < q.theta_lo || d == INF32 || d > capb) continue;
      if (d < q.theta_hi)
        nb |= 1u << t;
      else
        kb |= 1u << t;
    }
    // items moved to the near list carry the next round's parity, which a
    // split round does not flip
    const uint32_t psh = near_sh(q.par);
    if (nb | kb) {
      const uint32_t old = atomicOr(fw, (nb << psh) | (kb << FAR_SH));
      toN = nb && ((old >> psh) & 0xFFu) == 0u;
      toF = kb && ((old >> FAR_SH) & 0xFFu) == 0u;
    }
    return;
  }
  uint32_t cost = (uint32_t)(ld_cg(q.table + s) >> 32);
  if (cost < q.theta_lo || cost == INF32 || cost > best) {
    atomicAnd(&q.dflag[s >> 3], ~dflag_bit(s, 2u));
  } else if (cost < q.theta_hi) {
    atomicAnd(&q.dflag[s >> 3], ~dflag_bit(s, 2u));
    uint32_t bit = dflag_bit(s, q.par);
    uint32_t old = atomicOr(&q.dflag[s >> 3], bit);
    toN = !(old & bit);
  } else {
    toF = true;
  }
}

// Member item v*8+j -> distance 0; the vertex enters the first near list
// (the caller pushes v if toN).
__device__ void sseed_item(const QDev& q, uint32_t item, bool& toN) {
  uint32_t v = item >> 3, j = item & 7u;
  q.dist[(size_t)v * ROW + j] = 0;
  const uint32_t psh = near_sh(q.par);
  toN = ((atomicOr(q.dist + (size_t)v * ROW + FLAGW, (1u << j) << psh) >> psh) & 0xFFu) == 0u;
}

// Single append (DP seeding only: once per member state of a query).
__device__ __forceinline__ void push_list(const QDev& q, uint32_t* cnt, uint32_t* buf, uint32_t item) {
  uint32_t pos = atomicAdd(cnt, 1u);
  if (pos < q.cap)
    buf[pos] = item;
  else
    atomicExch(&q.ctl->overflow, 1u);
}

// Cost-0 states: every non-empty subset of a member's mask (DPQ.cu:341-358).
// The member item of the lowest group bit of the mask does the seeding.
__device__ void dseed_item(const QDev& q, uint32_t item) {
  uint32_t v = item >> 3, gi = item & 7u;
  uint32_t m = 0;
  for (int t = 0; t < q.k; t++)
    if (q.dist[(size_t)v * 8 + t] == 0) m |= 1u << t;
  if (m == 0 || (uint32_t)(__ffs(m) - 1) != gi) return;
  for (uint32_t sub = m; sub; sub = (sub - 1u) & m) {
    uint32_t s = q.phase == PH_HOP ? ((v << q.k) | sub) * (uint32_t)q.nd : ((v << q.k) | sub);
    q.table[s] = pack(0u, 0u);
    if (sub == (uint32_t)q.full) {  // v is in every query group: a cost-0 tree
      atomicMin(&q.ctl->best, 0u);
      atomicMin(&q.ctl->best_full, q.phase == PH_HOP ? (unsigned long long)(v * 8u) : (unsigned long long)v);
      continue;
    }
    uint32_t bit = dflag_bit(s, q.par);
    if (!(atomicOr(&q.dflag[s >> 3], bit) & bit)) push_list(q, &q.ctl->n_near, q.qbuf[q.out_idx], s);
  }
}

// One warp per query: group-to-group distances gd[i][j] = min over members of
// group i of the (capped) distance to group j, then the tour tables
//   P[i][S][j]  cheapest visiting order of S starting at i, ending at j
//   T2[i][S]    min_j P[i][S][j]
// (replaces the host DP of DPQ.cu:409-483 / AllPaths, CPUNONHOP.h:269-386).
__device__ void tour_warp(const QDev& q, uint32_t lane) {
  const int k = q.k;
  const uint32_t K2 = 1u << k;
  uint32_t* P = q.tour;
  uint32_t* T2 = q.tour + (size_t)k * K2 * k;
  uint32_t* gd = T2 + (size_t)k * K2;  // [8][8]
  for (uint32_t t = lane; t < 64; t += 32) gd[t] = BIG;
  __syncwarp();
  for (uint32_t t = lane; t < q.n_members; t += 32) {
    uint32_t item = q.members[t];
    uint32_t v = item >> 3, i = item & 7u;
    for (int j = 0; j < k; j++) atomicMin(&gd[i * 8 + j], min(q.dist[(size_t)v * 8 + j], q.cap1));
  }
  __syncwarp();
  // With no feasible tree found yet the distance rounds ran without a cap, so
  // an unreachable pair of groups proves there is no solution at all.
  if (lane == 0 && ld_cg(&q.ctl->best) == INF32) {
    bool cut = false;
    for (int i = 0; i < k; i++)
      for (int j = 0; j < k; j++)
        if (i != j && __ldcg(&gd[i * 8 + j]) >= BIG) cut = true;
    if (cut) q.ctl->infeasible = 1u;
  }
  const uint32_t nP = (uint32_t)k * K2 * (uint32_t)k;
  for (uint32_t t = lane; t < nP; t += 32) P[t] = BIG;
  __syncwarp();
  for (uint32_t i = lane; i < (uint32_t)k; i += 32) P[((size_t)i * K2 + (1u << i)) * k + i] = 0;
  __syncwarp();
  for (int size = 2; size <= k; size++) {
    for (uint32_t t = lane; t < nP; t += 32) {
      uint32_t l = t % k, S = (t / k) % K2, i = t / (k * K2);
      if ((uint32_t)__popc(S) != (uint32_t)size || !(S >> i & 1u) || !(S >> l & 1u) || l == i) continue;
      uint32_t Sp = S ^ (1u << l);
      uint32_t bestv = BIG;
      for (int jj = 0; jj < k; jj++)
        if (Sp >> jj & 1u) bestv = min(bestv, sat_add(P[((size_t)i * K2 + Sp) * k + jj], __ldcg(&gd[jj * 8 + l])));
      P[t] = bestv;
    }
    __syncwarp();
  }
  for (uint32_t t = lane; t < (uint32_t)k * K2; t += 32) {
    uint32_t i = t / K2, S = t % K2;
    uint32_t m = BIG;
    for (int l = 0; l < k; l++) m = min(m, P[((size_t)i * K2 + S) * k + l]);
    T2[t] = m;
  }
  __syncwarp();
}

// Lower-bound table rows: lbt[v][X] = lower_bound_comp(d(v), X) for every
// subset X (the per-vertex one_label_lb table of the reference,
// DPQ.cu:174-224, with the tour bounds of CPUNONHOP.h:436-496), saturated to
// 16 bits, which only lowers a bound.  32 consecutive items, one vertex per
// lane.  All lanes evaluate the same subset X at a time, so the bound's
// loops over the groups of X branch alike in every lane and the tour-table
// reads are one broadcast per warp; each lane packs 8 entries of its row
// into one 16-byte store.  Items of different
// queries in one task are handled run by run.
// lower_bound_comp for a subset X that every lane of the warp evaluates at
// the same time: the loops run over the groups of X only, and lane `lane`'s
// capped distances are read from shared memory (sdl[j][lane]), where a
// group index that varies inside the loop costs no local memory.  Same value
// as lower_bound_comp, with less work:
//   - each unordered pair {i, j} is visited once with the cheaper of the two
//     orders P[i][X][j], P[j][X][i] (the ordered pairs (i, j) and (j, i) give
//     d_i + P[i][X][j] + d_j and d_j + P[j][X][i] + d_i); a pair (i, i) only
//     exists for X = {i}, where every bound is d_i;
//   - each term is a sum of three values <= 2^30, which cannot overflow 32
//     bits, and saturation at BIG and the halving are monotone, so both are
//     applied once to the minimum (lb1) or maximum (lb2) instead of per term.
__device__ __forceinline__ uint32_t lower_bound_uniform(const uint32_t (*sdl)[32], uint32_t lane, int k, uint32_t X,
                                                        const uint32_t* __restrict__ P,
                                                        const uint32_t* __restrict__ T2) {
  const uint32_t K2 = 1u << k;
  if ((X & (X - 1u)) == 0u) return sdl[__ffs(X) - 1][lane];  // a single group
  uint32_t lb0 = 0, mind = BIG;
  for (uint32_t m = X; m; m &= m - 1u) {
    const uint32_t d = sdl[__ffs(m) - 1][lane];
    lb0 = max(lb0, d);
    mind = min(mind, d);
  }
  uint32_t m1 = 0xFFFFFFFFu, m2 = 0;
  for (uint32_t mi = X; mi; mi &= mi - 1u) {
    const uint32_t i = __ffs(mi) - 1;
    const uint32_t di = sdl[i][lane];
    const uint32_t* Pi = P + ((size_t)i * K2 + X) * k;
    for (uint32_t mj = mi & (mi - 1u); mj; mj &= mj - 1u) {  // the groups of X above i
      const uint32_t j = __ffs(mj) - 1;
      const uint32_t pij = min(ld_round(Pi + j), ld_round(P + ((size_t)j * K2 + X) * k + i));
      m1 = min(m1, di + pij + sdl[j][lane]);
    }
    m2 = max(m2, di + ld_round(T2 + (size_t)i * K2 + X) + mind);
  }
  const uint32_t lb1 = (min(m1, BIG) + 1u) >> 1;
  const uint32_t lb2 = (min(m2, BIG) + 1u) >> 1;
  return max(lb0, max(lb1, lb2));
}

__device__ void lbt_rows32(const QDev* qd, const uint32_t* __restrict__ pre, int nslots, uint32_t n_lb,
                           uint32_t task, uint32_t lane, uint32_t (*sdl)[32]) {
  const unsigned FULL = 0xFFFFFFFFu;
  const uint32_t it = task * 32u + lane;
  const bool valid = it < n_lb;
  const uint32_t slot = valid ? find_slot_s(pre, nslots, it) : 0xFFFFFFFFu;
  const uint32_t prev = __shfl_up_sync(FULL, slot, 1);
  unsigned runs = __ballot_sync(FULL, valid && (lane == 0u || prev != slot));
  while (runs) {
    const uint32_t i0 = (uint32_t)(__ffs(runs) - 1);
    runs &= runs - 1u;
    const uint32_t si = __shfl_sync(FULL, slot, i0);
    const bool mine = valid && slot == si;
    const QDev& q = qd[si];
    const int k = q.k;
    const uint32_t K2 = 1u << k;
    const uint32_t* P = q.tour;
    const uint32_t* T2 = q.tour + (size_t)k * K2 * k;
    const uint32_t v = mine ? q.lb_off + (it - pre[si]) : 0u;
    {
      uint4 a = make_uint4(0u, 0u, 0u, 0u), b = a;
      if (mine) {
        const uint4* row = reinterpret_cast<const uint4*>(q.dist + (size_t)v * ROW);
        a = ld_round(row);
        b = ld_round(row + 1);
      }
      const uint32_t r[KMAX] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z};
#pragma unroll
      for (int j = 0; j < KMAX; j++) sdl[j][lane] = min(r[j], q.cap1);
    }
    __syncwarp();
    unsigned short* out = q.lbt + ((size_t)v << k);
    for (uint32_t x0 = 0; x0 < K2; x0 += 8u) {
      uint32_t pk[4];
#pragma unroll
      for (int h = 0; h < 4; h++) {
        uint32_t two = 0;
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const uint32_t X = x0 + 2u * h + e;
          uint32_t lb = 0;
          if (X != 0u && X < K2) lb = lower_bound_uniform(sdl, lane, k, X, P, T2);
          const uint32_t ent = lb >= BIG ? LB_INF : min(lb, LB_INF - 1u);
          two |= ent << (16 * e);
        }
        pk[h] = two;
      }
      if (mine) {
        if (K2 >= 8u) {
          *reinterpret_cast<uint4*>(out + x0) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        } else {
          for (uint32_t X = 0; X < K2; X++) out[X] = (unsigned short)(pk[X >> 1] >> (16 * (X & 1u)));
        }
      }
    }
    __syncwarp();  // the next run reuses the distance stage
  }
}

// Weight of arc (a -> b): the warp scans a's weight-sorted adjacency, 32
// arcs per step (hub lists hold tens of thousands of arcs).  Every lane calls
// it with the same a and b.
__device__ uint32_t arc_weight_warp(const GraphDev& g, uint32_t a, uint32_t b, uint32_t lane) {
  const uint32_t x0 = __ldg(g.beg + a), x1 = __ldg(g.beg + a + 1);
  for (uint32_t base = x0; base < x1; base += 32u) {
    const uint32_t x = base + lane;
    uint32_t w = INF32;
    if (x < x1) {
      const uint2 arc = __ldg(g.adj + x);
      if (arc.x == b) w = arc.y;
    }
    const unsigned hit = __ballot_sync(0xFFFFFFFFu, w != INF32);
    if (hit) return __shfl_sync(0xFFFFFFFFu, w, __ffs(hit) - 1);
  }
  return INF32;
}

// Follow parent words from the best full state, emitting (u, v, w) edges;
// qbuf[0] serves as the explicit stack.  Run by one warp: every lane walks
// the same states (lane 0 alone writes), and the arc weights are looked up
// by the whole warp.
__device__ void extract_warp(const QDev& q, const GraphDev& g, uint32_t lane) {
  QCtl* ctl = q.ctl;
  const unsigned long long bf = __ldcg(&ctl->best_full);
  if (bf == INF64) {
    if (lane == 0) {
      ctl->status = 1;
      ctl->n_edges = 0;
    }
    return;
  }
  const int k = q.k, nd = q.nd;
  const bool hop = q.phase == PH_HOP;
  const uint32_t payload = (uint32_t)bf;
  const uint32_t root = hop ? payload >> 3 : payload;
  const uint32_t rd = hop ? (payload & 7u) : 0u;
  uint32_t* stack = q.qbuf[0];
  uint32_t sp = 0;
  const uint32_t full = (uint32_t)q.full;
  if (lane == 0) stack[0] = hop ? ((root << k) | full) * (uint32_t)nd + rd : ((root << k) | full);
  sp = 1;
  __syncwarp();
  uint32_t ne = 0, steps = 0, status = 0;
  const uint32_t max_steps = 4u * g.V + 64u;
  while (sp > 0) {
    if (++steps > max_steps || sp + 2 > q.cap) {
      status = 2;
      break;
    }
    const uint32_t s = __ldcg(stack + --sp);
    __syncwarp();  // every lane has read the top before lane 0 overwrites it
    const uint32_t d = hop ? s % (uint32_t)nd : 0u;
    const uint32_t vp = hop ? s / (uint32_t)nd : s;
    const uint32_t v = vp >> k, p = vp & ((1u << k) - 1u);
    const unsigned long long e = __ldcg(q.table + s);
    if ((uint32_t)(e >> 32) == INF32) {
      status = 2;
      break;
    }
    const uint32_t par = (uint32_t)e;
    const uint32_t type = par >> 30;
    if (type == 1u) {
      const uint32_t u = par & 0x3FFFFFFFu;
      const uint32_t w = arc_weight_warp(g, v, u, lane);
      if (lane == 0 && ne < q.max_edges) {
        q.out_edges[3 * ne] = u;
        q.out_edges[3 * ne + 1] = v;
        q.out_edges[3 * ne + 2] = w;
      }
      ne++;
      if (hop && d == 0) {
        status = 2;
        break;
      }
      if (lane == 0) stack[sp] = hop ? ((u << k) | p) * (uint32_t)nd + d - 1 : ((u << k) | p);
      sp++;
    } else if (type == 2u) {
      const uint32_t p1 = par & 0xFFu, p2 = p ^ p1;
      if (p1 == 0 || p2 == 0 || (p1 & ~p) != 0) {
        status = 2;
        break;
      }
      if (lane == 0) {
        if (hop) {
          const uint32_t d1 = (par >> 8) & 7u, d2 = (par >> 11) & 7u;
          stack[sp] = ((v << k) | p1) * (uint32_t)nd + d1;
          stack[sp + 1] = ((v << k) | p2) * (uint32_t)nd + d2;
        } else {
          stack[sp] = (v << k) | p1;
          stack[sp + 1] = (v << k) | p2;
        }
      }
      sp += 2;
    } else if (type != 0u) {
      status = 2;
      break;
    }
    __syncwarp();  // lane 0's pushes are visible to the next pop
  }
  if (lane == 0) {
    ctl->status = status;
    ctl->n_edges = ne;
    ctl->root = root;
  }
}

// ---------------------------------------------------------------------------
// Workspace initialisation of an admitted query, one launch: the state table
// to INF (all ones), both distance-row buffers to "unknown" (words 0..6 all
// ones) with no group pending (word 7 zero), and the state flags to zero.
// 16-byte stores, grid-stride.  (Replaces several memsets per query, one of
// them a 2D memset over V rows of 4 bytes.)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_init_workspace(uint4* __restrict__ table, size_t table_vec,
                                                        uint4* __restrict__ dist, uint4* __restrict__ dist2,
                                                        uint32_t nv, uint4* __restrict__ dflag, size_t dflag_vec) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint4 ones = make_uint4(INF32, INF32, INF32, INF32);
  const uint4 tail = make_uint4(INF32, INF32, INF32, 0u);
  for (size_t i = tid; i < table_vec; i += stride) table[i] = ones;
  for (size_t v = tid; v < nv; v += stride) {
    dist[2 * v] = ones;
    dist[2 * v + 1] = tail;
    if (dist2 != nullptr) {
      dist2[2 * v] = ones;
      dist2[2 * v + 1] = tail;
    }
  }
  for (size_t i = tid; i < dflag_vec; i += stride) dflag[i] = make_uint4(0u, 0u, 0u, 0u);
}

// ---------------------------------------------------------------------------
// Control: one thread per slot.  Absorbs the previous round's counters,
// decides this round's action, and publishes per-type item counts as
// exclusive prefix sums over slots (pre[t][0..nslots]).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void absorb(QDev& q, QCtl& c) {
  if (c.cancel) {  // the host withdrew the request
    q.st = J_DONE;
    c.final_status = 12;  // GST_CANCELLED
    c.done = 1;
    return;
  }
  if (c.overflow) {
    q.st = J_DONE;
    c.final_status = 6;  // GST_QUEUE_OVERFLOW
    c.done = 1;
    return;
  }
  int t;
  q.snap_h = 0;  // a snapshot scheduled last round has been copied
  switch (q.act) {
    case A_SSEED:
      t = q.in_idx; q.in_idx = q.out_idx; q.out_idx = t;
      q.n_in = c.n_near;
      q.n_far = 0;
      q.st = J_SSSP;
      break;
    case A_WORK:
      t = q.in_idx; q.in_idx = q.out_idx; q.out_idx = t;
      q.n_in = c.n_near;
      q.n_far = c.n_far;
      q.par ^= 1u;  // producers of the round flagged the next items with the other parity
      if (q.st == J_SSSP) {
        q.hops++;
        if (q.dist_nx != q.dist) {  // exact rounds: the rows just written become the current ones
          uint32_t* x = q.dist;
          q.dist = q.dist_nx;
          q.dist_nx = x;
        }
        if (q.hops == q.center_h + 1u) q.center_done = 1u;  // the pass ran during this round
        // rows after round b bound the paths of at most b hops: copy them
        // while the next round runs (a value it lowers in the meantime is
        // still a valid bound)
        if (q.D >= 0 && q.hops < (uint32_t)q.D) q.snap_h = q.hops;
      }
      break;
    case A_SPLIT:
      t = q.in_idx; q.in_idx = q.out_idx; q.out_idx = t;
      t = q.far_idx; q.far_idx = q.far2_idx; q.far2_idx = t;
      q.n_in = c.n_near;
      q.n_far = c.n_far2;
      break;
    case A_TOUR:
      q.st = c.infeasible ? J_EXTRACT : J_LB;  // disconnected groups: straight to "no solution"
      break;
    case A_LB:
      // the bound table is filled in chunks of LB_CHUNK entries per round
      q.lb_off += min(q.nv - q.lb_off, LB_CHUNK);
      if (q.lb_off >= q.nv) q.st = J_DPSEED;
      break;
    case A_DSEED:
      t = q.in_idx; q.in_idx = q.out_idx; q.out_idx = t;
      q.n_in = c.n_near;
      q.n_far = 0;
      q.st = J_DP;
      break;
    case A_EXTRACT:
      q.st = J_DONE;
      c.final_status = c.status == 1 ? 1u : (c.status != 0 ? 8u : 0u);  // NO_SOLUTION / INTERNAL / OK
      c.done = 1;
      break;
    default:
      break;
  }
  if (q.act != A_NONE) c.stat[ST_ROUNDS]++;
  q.act = A_NONE;
}

// End of a hop-bounded query's distance rounds.  Every tree of hop diameter
// <= D has a vertex with all its vertices within ceil(D/2) hops (a centre of
// the tree), so when the exact rows of that many hops showed no vertex with
// every group in reach, the query has no solution.
__device__ __forceinline__ void hop_rounds_done(QDev& q, QCtl& c) {
  if (q.center_h != 0u && q.center_done && c.center == 0u && c.best == INF32) c.infeasible = 1u;
  q.dist_nx = q.dist;
}

__device__ __forceinline__ void decide(QDev& q, QCtl& c) {
  for (int guard = 0; guard < 8; guard++) {
    switch (q.st) {
      case J_INIT:
        q.phase = PH_SSSP;
        q.theta_lo = 0;
        // a hop-bounded query runs its distance rounds as Bellman-Ford rounds
        // (one window holding everything): after D rounds every path of at
        // most D hops has been relaxed
        q.theta_hi = q.D >= 0 ? INF32 : q.delta_sssp;
        q.delta = q.delta_sssp;
        q.hops = 0;
        c.n_near = 0;
        q.act = A_SSEED;
        return;
      case J_SSSP:
      case J_DP: {
        if (q.st == J_SSSP && q.D >= 0 && q.hops >= (uint32_t)q.D) {
          // hop-bounded distances: d_j(v) <= the cheapest path of at most D
          // hops from group j to v, INF if there is none.  Every path of the
          // final tree has at most D hops, so these are valid lower bounds,
          // and an unreached vertex cannot join a group
          q.cap1 = BIG;
          q.snap_n = min(q.hops, (uint32_t)q.D - 1u);
          hop_rounds_done(q, c);
          q.st = J_TOUR;
          continue;
        }
        if (q.st == J_DP && q.phase == PH_DP && q.ratio_num != 0u && c.best_full != INF64) {
          // Progressive exit (CPUNONHOP.h:730-755, in exact integer
          // arithmetic).  Every state of cost below lo (theta_lo, or theta_hi
          // once the window's near list is empty) has been expanded at its
          // final cost.  The optimum's derivation has no state costlier than
          // the optimum, so an optimum below lo would already be recorded:
          // opt >= min(best_full, lo).  Stop once best_full <= ratio * lo.
          const unsigned long long lo = q.n_in > 0 ? q.theta_lo : q.theta_hi;
          const unsigned long long bf = c.best_full >> 32;
          if (bf * q.ratio_den <= lo * q.ratio_num) {
            c.early = 1u;
            c.lb_exit = (uint32_t)(bf < lo ? bf : lo);
            q.st = J_EXTRACT;
            continue;
          }
        }
        if (q.n_in > 0) {
          c.n_near = 0;
          c.n_far = q.n_far;
          q.act = A_WORK;
          return;
        }
        uint32_t next_lo = q.theta_hi;
        // distance rounds only matter up to cap(best); DP rounds up to best
        unsigned long long limit = c.best;
        if (q.st == J_SSSP && c.best != INF32) limit = (unsigned long long)c.best * q.cap_num / q.cap_den;
        bool exhausted = q.n_far == 0 || next_lo > limit;
        if (!exhausted) {
          q.theta_lo = next_lo;
          q.theta_hi = next_lo + q.delta;
          c.n_near = 0;
          c.n_far2 = 0;
          q.act = A_SPLIT;
          return;
        }
        if (q.st == J_SSSP) {
          // a hop-bounded query whose rounds converged before D: rows for
          // more hops than the snapshots taken are the final distances
          if (q.D >= 0) {
            q.snap_n = min(q.hops, q.D > 0 ? (uint32_t)q.D - 1u : 0u);
            hop_rounds_done(q, c);
          }
          // every distance below theta_hi is exact and every distance <=
          // cap(best) was discovered; unknown ones are >= min(theta_hi, cap+1)
          unsigned long long b1 = c.best == INF32 ? (unsigned long long)INF32 : limit + 1;
          unsigned long long cap1 = q.n_far == 0 ? b1 : (q.theta_hi < b1 ? q.theta_hi : b1);
          q.cap1 = (uint32_t)(cap1 < BIG ? cap1 : BIG);
          q.st = J_TOUR;
          continue;
        }
        q.st = J_EXTRACT;
        continue;
      }
      case J_TOUR:
        q.act = A_TOUR;
        return;
      case J_LB:
        q.act = A_LB;
        return;
      case J_DPSEED:
        q.phase = q.D < 0 ? PH_DP : PH_HOP;
        q.theta_lo = 0;
        q.theta_hi = q.delta_dp;
        q.delta = q.delta_dp;
        q.n_in = 0;
        q.n_far = 0;
        c.n_near = 0;
        c.n_far = 0;
        q.act = A_DSEED;
        return;
      case J_EXTRACT:
        q.act = A_EXTRACT;
        return;
      default:
        q.act = A_NONE;
        return;
    }
  }
}

// Shared memory of one control step.
struct CtlSmem {
  uint32_t wsum[32][NT];  // per-warp inclusive totals, then their scan
  uint32_t carry[NT];     // items of the slots in earlier chunks
  uint32_t live_cnt, used_hi;
};

// One control step over slots [0, nslots) by all threads of one block
// (blockDim.x a multiple of 32, at most 1024).  Slots go in chunks of
// blockDim.x; the per-type prefixes carry from one chunk to the next, so any
// block size gives the same prefixes.
__device__ void control_step(QDev* qd, QCtl* ctl, int nslots, RoundDesc* rd, uint32_t* pre, CtlSmem& sm) {
  const int tid = threadIdx.x, B = blockDim.x;
  const uint32_t lane = tid & 31, wid = tid >> 5, nw = (uint32_t)B >> 5;
  if (tid == 0) sm.live_cnt = sm.used_hi = 0;
  if (tid < NT) sm.carry[tid] = 0;
  __syncthreads();
  for (int base = 0; base <= nslots; base += B) {
    const int s = base + tid;
    uint32_t cnt[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) cnt[t] = 0;
    // the state alone first: most slots are free when the scan covers them all
    const int32_t st0 = s < nslots ? qd[s].st : J_FREE;
    if (st0 != J_FREE) atomicMax(&sm.used_hi, (uint32_t)s + 1u);
    if (st0 != J_FREE && st0 != J_DONE) {
      QDev q = qd[s];
      QCtl& c = ctl[s];
      absorb(q, c);
      if (q.st != J_DONE) decide(q, c);
      switch (q.act) {
        case A_SSEED: cnt[T_SSEED] = q.n_members; break;
        case A_DSEED: cnt[T_DSEED] = q.n_members; break;
        case A_SPLIT: cnt[T_SPLIT] = q.n_far; break;
        case A_TOUR: cnt[T_TOUR] = 1; break;
        case A_LB: cnt[T_LB] = min(q.nv - q.lb_off, LB_CHUNK); break;
        case A_EXTRACT: cnt[T_EXTRACT] = 1; break;
        case A_WORK:
          cnt[q.phase == PH_SSSP ? T_SSSP : (q.phase == PH_DP ? T_DP : T_HOP)] = q.n_in;
          break;
        default: break;
      }
      if (q.snap_h) cnt[T_SNAP] = q.nv;  // copy the distance rows of round snap_h
      if (q.st != J_DONE) atomicAdd(&sm.live_cnt, 1u);
      qd[s] = q;
    }
    // exclusive scan over the chunk's slots, per task type
    uint32_t incl[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) {
      uint32_t x = cnt[t];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
      }
      incl[t] = x;
      if (lane == 31) sm.wsum[wid][t] = x;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
      for (int t = 0; t < NT; t++) {
        uint32_t x = lane < nw ? sm.wsum[lane][t] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
          if (lane >= (uint32_t)o) x += y;
        }
        sm.wsum[lane][t] = x;  // inclusive over warps
      }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < NT; t++) {
      uint32_t before = sm.carry[t] + (wid ? sm.wsum[wid - 1][t] : 0u) + incl[t] - cnt[t];
      if (s <= nslots) pre[t * (MAX_SLOTS + 1) + s] = before;
    }
    __syncthreads();  // carry and wsum read by every thread
    if (tid < NT) sm.carry[tid] += sm.wsum[nw - 1][tid];
    __syncthreads();
  }
  if (tid == 0) {
    // distance items per warp task: 4 while that leaves at most two tasks per
    // light warp, more (up to sssp_wmax) in rounds with many items
    uint32_t w = 4;
    const unsigned long long n_sssp = sm.carry[T_SSSP];
    while (w < min(rd->sssp_wmax, SSSP_WMAX) && n_sssp > 2ull * w * rd->light_warps) w <<= 1;
    rd->sssp_w = w;
    // DP states per warp task: 1 while that leaves at most two tasks per
    // light warp (every state gets a warp), more (up to dp_wmax) in rounds
    // with many states
    uint32_t wd = 1;
    const unsigned long long n_dp = (unsigned long long)sm.carry[T_DP] + sm.carry[T_HOP];
    while (wd < rd->dp_wmax && n_dp > 2ull * wd * rd->light_warps) wd <<= 1;
    rd->dp_w = wd;
    const uint32_t per_task[NT] = {32, 32, 32, 1, 1, w, wd, wd, 32, 32};
    uint32_t off = 0;
    for (int t = 0; t < NT; t++) {
      uint32_t tot = sm.carry[t];
      rd->items[t] = tot;
      if (t == T_LB) {
        rd->light_tasks = off;
        off = 0;
      }
      rd->task_off[t] = off;
      off += (tot + per_task[t] - 1) / per_task[t];
    }
    rd->task_off[NT] = off;
    rd->heavy_tasks = off;
    rd->n_live = sm.live_cnt;
    rd->nslots = sm.used_hi;  // slots the round kernels search (all later ones are free)
    rd->n_big = 0;
    rd->next_light = 0;
    rd->next_heavy = 0;
    // hub chunking pays off only when the round is too small to fill the GPU
    const uint32_t n_items = rd->items[T_SSSP] + rd->items[T_DP] + rd->items[T_HOP];
    rd->hub_on = (rd->big != nullptr && n_items < rd->hub_max_items) ? 1u : 0u;
    // distance items: every hub in small rounds; in larger ones (a single
    // query's dense rounds) only the biggest hubs, whose one warp would
    // otherwise finish long after the rest: at least hub_big_deg arcs and
    // more than 1/hub_share_div of a warp's share of the round's arcs
    uint32_t big_deg = rd->hub_big_deg;
    if (rd->hub_share_div != 0u) {
      const unsigned long long share =
          (unsigned long long)n_items * rd->avg_deg / max(1u, rd->light_warps) / rd->hub_share_div;
      big_deg = (uint32_t)max((unsigned long long)big_deg, min(share, (unsigned long long)INF32 - 1ull));
    }
    rd->hub_deg = rd->hub_on ? rd->hub_min_deg
                             : ((rd->big != nullptr && n_items < rd->hub_max_items2) ? big_deg : INF32);
    // DP tasks that hold several states hand their hub grows out in every
    // round: a task with a few hub states would otherwise grow them one
    // after another on one warp
    rd->grow_chunks = (rd->big != nullptr && (rd->hub_on || wd > 1u)) ? 1u : 0u;
  }
}

__global__ void __launch_bounds__(1024) k_control(QDev* __restrict__ qd, QCtl* __restrict__ ctl, int nslots,
                                                  RoundDesc* __restrict__ rd, uint32_t* __restrict__ pre) {
  __shared__ CtlSmem sm;
  control_step(qd, ctl, nslots, rd, pre, sm);
}

// ---------------------------------------------------------------------------
// Round work, one warp task at a time.  The separate round kernels (k_light,
// k_heavy) and the persistent one (k_rounds) run the same tasks.
// ---------------------------------------------------------------------------

// Light task `task` (types T_SPLIT .. T_HOP: splits, seeds, tour tables,
// extraction, distance items, DP states).  s_pre / s_dp / s_hop: the per-slot
// prefixes of the distance, DP and hop items, staged in shared memory.
__device__ __forceinline__ void light_task(const QDev* qd, RoundDesc* rd, const uint32_t* pre,
                                           const uint32_t* s_pre, const uint32_t* s_dp, const uint32_t* s_hop,
                                           int nslots, const GraphDev& g, uint32_t task, uint32_t lane,
                                           WarpStat& ws, WarpBuf& wb, WarpScratch& sc) {
  int t = 0;
  while (t < T_HOP && task >= __ldcg(&rd->task_off[t + 1])) t++;
  const uint32_t local = task - __ldcg(&rd->task_off[t]);
  const uint32_t* P = pre + t * (MAX_SLOTS + 1);
  const uint32_t total = __ldcg(&rd->items[t]);
  if (t == T_SSSP) {
    sssp_task(qd, s_pre, nslots, total, local, __ldcg(&rd->sssp_w), g, lane, ws, rd, sc.hdr, wb);
  } else if (t == T_DP || t == T_HOP) {
    dp_task(qd, t == T_DP ? s_dp : s_hop, nslots, total, local, __ldcg(&rd->dp_w), t == T_HOP, g, lane, rd, ws, wb,
            &sc.mg);
  } else if (t == T_TOUR) {
    tour_warp(qd[find_slot(P, nslots, local)], lane);
  } else if (t == T_EXTRACT) {
    extract_warp(qd[find_slot(P, nslots, local)], g, lane);
  } else {
    const uint32_t it = local * 32u + lane;
    bool toN = false, toF = false;
    uint32_t slot = 0, item = 0;
    if (it < total) {
      slot = find_slot(P, nslots, it);
      const QDev& q = qd[slot];
      const uint32_t idx = it - __ldcg(P + slot);
      if (t == T_SPLIT) {
        item = q.qbuf[q.far_idx][idx];
        split_item(q, item, toN, toF);
      } else if (t == T_SSEED) {
        const uint32_t m = __ldg(q.members + idx);
        item = m >> 3;
        sseed_item(q, m, toN);
      } else {
        dseed_item(q, __ldg(q.members + idx));
      }
    }
    push_multi(toN, item, 0u, qd[slot], slot, lane);
    push_multi(toF, item, 1u, qd[slot], slot, lane);
  }
}

// Heavy task `ht` that does not depend on the round's light tasks: bound-table
// rows (one vertex per lane) and snapshot rows of hop-bounded queries.
__device__ __forceinline__ void heavy_static_task(const QDev* qd, const uint32_t* pre, const uint32_t* s_lb,
                                                  int nslots, uint32_t ht, uint32_t snap0, uint32_t n_lb,
                                                  uint32_t n_snap, uint32_t lane, uint32_t (*sdl)[32]) {
  if (ht < snap0) {
    lbt_rows32(qd, s_lb, nslots, n_lb, ht, lane, sdl);
    return;
  }
  // snapshot of a hop-bounded query's distance rows, one row per lane
  const uint32_t it = (ht - snap0) * 32u + lane;
  if (it < n_snap) {
    const uint32_t* P = pre + T_SNAP * (MAX_SLOTS + 1);
    const uint32_t slot = find_slot(P, nslots, it);
    const QDev& qs = qd[slot];
    const uint32_t v = it - __ldcg(P + slot);
    const uint4* src = reinterpret_cast<const uint4*>(qs.dist + (size_t)v * ROW);
    uint4* dst = reinterpret_cast<uint4*>(qs.snap + ((size_t)(qs.snap_h - 1u) * qs.nv + v) * ROW);
    const uint4 a = __ldcg(src), b = __ldcg(src + 1);
    dst[0] = a;
    dst[1] = b;
    if (qs.snap_h == qs.star_h || qs.snap_h == qs.center_h) {
      // the rows are the exact distances over paths of at most snap_h hops
      const uint32_t r[KMAX] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z};
      bool all = true;
      unsigned long long sum = 0;
#pragma unroll
      for (int t = 0; t < KMAX; t++)
        if (t < qs.k) {
          all = all && r[t] != INF32;
          sum += r[t];
        }
      if (all && qs.snap_h == qs.center_h && __ldca(&qs.ctl->center) == 0u) atomicExch(&qs.ctl->center, 1u);
      // v joined to every group by its cheapest path of at most star_h
      // hops: a breadth-first tree from v inside their union has depth <=
      // star_h, so diameter <= 2 * star_h <= D, at cost <= sum
      if (all && qs.snap_h == qs.star_h && sum < ld_best(qs.ctl)) atomicMin(&qs.ctl->best, (uint32_t)sum);
    }
  }
}

// Arc chunk `i` that a light task handed over this round (hub vertex of a
// distance item, or a high-degree DP state's grow).
__device__ __forceinline__ void chunk_task(const QDev* qd, const RoundDesc* rd, const GraphDev& g, uint32_t i,
                                           uint32_t lane, RelaxHdr* hub, WarpStat& ws, WarpBuf& wb) {
  const uint4 it = __ldcg(rd->big + i);
  if (it.x & CH_GROW)
    grow_chunk(qd, it, g, lane, ws, wb);
  else
    hub_chunk(qd, it, g, lane, hub, ws, wb);
}

// Light round kernel: the round's light tasks.  NW warps per block (4 or
// 8); the occupancy bound keeps 24 warps per SM at 80 registers.
#ifndef GSTB_LIGHT_MIN_BLOCKS
#define GSTB_LIGHT_MIN_BLOCKS 3  // blocks of 8 warps
#endif
template <int NW>
__global__ void __launch_bounds__(NW * 32, GSTB_LIGHT_MIN_BLOCKS * 8 / NW)
    k_light(const QDev* __restrict__ qd, RoundDesc* __restrict__ rd, const uint32_t* __restrict__ pre, int nslots,
            GraphDev g) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t ntasks = __ldcg(&rd->light_tasks);
  nslots = min(nslots, (int)__ldcg(&rd->nslots));
  // prefixes over slots of the item types with many items, staged once per block
  __shared__ uint32_t s_pre[MAX_SLOTS + 1], s_dp[MAX_SLOTS + 1], s_hop[MAX_SLOTS + 1];
  __shared__ WarpScratch s_sc[NW];
  __shared__ WarpStat s_ws[NW];
  __shared__ WarpBuf s_wb[NW];
  WarpStat& ws = s_ws[threadIdx.x >> 5];
  WarpBuf& wb = s_wb[threadIdx.x >> 5];
  if (lane == 0) {
    ws_init(ws);
    wb_init(wb);
  }
  for (int i = threadIdx.x; i <= nslots; i += blockDim.x) {
    s_pre[i] = __ldcg(pre + T_SSSP * (MAX_SLOTS + 1) + i);
    s_dp[i] = __ldcg(pre + T_DP * (MAX_SLOTS + 1) + i);
    s_hop[i] = __ldcg(pre + T_HOP * (MAX_SLOTS + 1) + i);
  }
  __syncthreads();
#if GSTB_STEAL
  for (uint32_t task = warp; task < ntasks; task = next_task(&rd->next_light, nwarps, lane))
#else
  for (uint32_t task = warp; task < ntasks; task += nwarps)
#endif
    light_task(qd, rd, pre, s_pre, s_dp, s_hop, nslots, g, task, lane, ws, wb, s_sc[threadIdx.x >> 5]);
  wb_flush(wb, lane);
  if (lane == 0) ws_flush(ws);
}

// Heavy round kernel: the arc chunks k_light handed over this round, then
// bound-table rows and snapshot rows.
template <int NW>
__global__ void __launch_bounds__(NW * 32, 24 / NW)
    k_heavy(const QDev* __restrict__ qd, RoundDesc* __restrict__ rd, const uint32_t* __restrict__ pre, int nslots,
            GraphDev g) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nbig = rd->big ? min(__ldcg(&rd->n_big), rd->big_cap) : 0u;
  const uint32_t ntasks = __ldcg(&rd->heavy_tasks) + nbig;
  nslots = min(nslots, (int)__ldcg(&rd->nslots));
  __shared__ uint32_t s_lb[MAX_SLOTS + 1];
  __shared__ RelaxHdr s_hub[NW];
  __shared__ uint32_t s_dl[NW][KMAX][32];  // bound rows: each lane's capped distances
  __shared__ WarpStat s_ws[NW];
  __shared__ WarpBuf s_wb[NW];
  WarpStat& ws = s_ws[threadIdx.x >> 5];
  WarpBuf& wb = s_wb[threadIdx.x >> 5];
  if (lane == 0) {
    ws_init(ws);
    wb_init(wb);
  }
  for (int i = threadIdx.x; i <= nslots; i += blockDim.x) s_lb[i] = __ldcg(pre + T_LB * (MAX_SLOTS + 1) + i);
  __syncthreads();
  const uint32_t n_lb = __ldcg(&rd->items[T_LB]), n_snap = __ldcg(&rd->items[T_SNAP]);
  const uint32_t snap0 = __ldcg(&rd->task_off[T_SNAP]);  // heavy tasks before the snapshot rows
#if GSTB_STEAL
  for (uint32_t task = warp; task < ntasks; task = next_task(&rd->next_heavy, nwarps, lane)) {
#else
  for (uint32_t task = warp; task < ntasks; task += nwarps) {
#endif
    if (task < nbig)
      chunk_task(qd, rd, g, task, lane, &s_hub[threadIdx.x >> 5], ws, wb);
    else
      heavy_static_task(qd, pre, s_lb, nslots, task - nbig, snap0, n_lb, n_snap, lane, s_dl[threadIdx.x >> 5]);
  }
  wb_flush(wb, lane);
  if (lane == 0) ws_flush(ws);
}

// ---------------------------------------------------------------------------
// Persistent round loop: R rounds in one cooperative launch (every block
// resident at once).  Block 0 runs the first control step; the last block to
// finish a round's work runs the next one.  A round is
//   wait for its control step (epoch) -> light tasks and the static heavy
//   tasks (bound rows, snapshots), taken by warp striding -> every block done
//   with those (phase1: the arc chunks the light tasks handed over are all
//   written; skipped in rounds that hand out none) -> the chunks -> arrive;
//   the last block to arrive runs the next control step and publishes it.
// Every wait is bounded by pc->timeout_ns (and an iteration limit): when one
// expires the launch sets pc->err and every block returns, the host fails
// the admitted queries with GST_DEVICE_TIMEOUT and the context stays usable.
// ---------------------------------------------------------------------------
// The waits poll with relaxed loads (read at L2, leaving the SM's L1 alone)
// and order what follows with one fence once the flag is seen: an acquire at
// every poll would invalidate the L1 of an SM whose other blocks are still
// working from it.
__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// One thread: wait until *flag >= target, then fence (the acquire).  False
// when the launch has failed (another wait expired) or this one expires.
__device__ bool wait_geq(const uint32_t* flag, uint32_t target, PersistCtl* pc, uint32_t where) {
  const unsigned long long t0 = global_ns(), lim = pc->timeout_ns;
  uint32_t ns = 32;
  for (uint32_t it = 0; it < (1u << 25); it++) {
    if (ld_relaxed_gpu(flag) >= target) {
      __threadfence();
      return true;
    }
    if (ld_relaxed_gpu(&pc->err)) return false;
    if (global_ns() - t0 > lim) break;
    if (it >= 64u) {  // a short wait polls back to back, a long one backs off to 1 us
      __nanosleep(ns);
      if (ns < 1024u) ns <<= 1;
    }
  }
  atomicCAS(&pc->err_where, 0u, where);
  atomicExch(&pc->err, 1u);
  return false;
}

// Publish control step `e` (after its writes).  One thread.
__device__ __forceinline__ void publish(PersistCtl* pc, uint32_t e) {
  __threadfence();
  if (!pc->hold) st_release_gpu(&pc->epoch, e);
}

template <int NW>
struct RoundSmem {
  uint32_t pre_sssp[MAX_SLOTS + 1], pre_dp[MAX_SLOTS + 1], pre_hop[MAX_SLOTS + 1], pre_lb[MAX_SLOTS + 1];
  WarpScratch w[NW];
  WarpStat ws[NW];
  WarpBuf wb[NW];
  CtlSmem ctl;
  uint32_t ok, last;
};

template <int NW>
__global__ void __launch_bounds__(NW * 32, 24 / NW)
    k_rounds(QDev* qd, QCtl* ctl, int nslots_ctl, RoundDesc* rd, uint32_t* pre, GraphDev g, uint32_t R,
             PersistCtl* pc) {
  __shared__ RoundSmem<NW> sm;
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  const uint32_t warp = blockIdx.x * (blockDim.x >> 5) + wib;
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  WarpStat& ws = sm.ws[wib];
  WarpBuf& wb = sm.wb[wib];
  uint32_t p1 = 0;  // rounds with a chunk phase so far (the same in every block)
  if (blockIdx.x == 0) {
    control_step(qd, ctl, nslots_ctl, rd, pre, sm.ctl);
    __syncthreads();
    if (threadIdx.x == 0) publish(pc, 1u);
  }
  for (uint32_t r = 0; r < R; r++) {
    if (threadIdx.x == 0) sm.ok = wait_geq(&pc->epoch, r + 1u, pc, 1u) ? 1u : 0u;
    __syncthreads();
    if (!sm.ok) return;
    // a round with no live query does nothing, nor do the rest: every block
    // reads the same count, so every block leaves here together
    if (__ldcg(&rd->n_live) == 0u) return;
    const int nslots = min(nslots_ctl, (int)__ldcg(&rd->nslots));
    for (int i = threadIdx.x; i <= nslots; i += blockDim.x) {
      sm.pre_sssp[i] = __ldcg(pre + T_SSSP * (MAX_SLOTS + 1) + i);
      sm.pre_dp[i] = __ldcg(pre + T_DP * (MAX_SLOTS + 1) + i);
      sm.pre_hop[i] = __ldcg(pre + T_HOP * (MAX_SLOTS + 1) + i);
      sm.pre_lb[i] = __ldcg(pre + T_LB * (MAX_SLOTS + 1) + i);
    }
    if (lane == 0) {
      ws_init(ws);
      wb_init(wb);
    }
    __syncthreads();
    const uint32_t ntl = __ldcg(&rd->light_tasks), nth = __ldcg(&rd->heavy_tasks);
    const uint32_t n_lb = __ldcg(&rd->items[T_LB]), n_snap = __ldcg(&rd->items[T_SNAP]);
    const uint32_t snap0 = __ldcg(&rd->task_off[T_SNAP]);
    // light tasks, then the static heavy ones, as one list dealt out over
    // the warps (two lists dealt out one after the other would leave the
    // warps with the heaviest light tasks also the first heavy ones)
    for (uint32_t task = warp; task < ntl + nth; task += nwarps) {
      if (task < ntl)
        light_task(qd, rd, pre, sm.pre_sssp, sm.pre_dp, sm.pre_hop, nslots, g, task, lane, ws, wb, sm.w[wib]);
      else
        heavy_static_task(qd, pre, sm.pre_lb, nslots, task - ntl, snap0, n_lb, n_snap, lane, sm.w[wib].dl);
    }
    // phase 1 done in this block: its chunk entries are written.  Rounds
    // that hand out no chunks (every block reads the same flags) skip the
    // grid-wide wait for the others
    if (rd->big != nullptr && (__ldcg(&rd->hub_deg) != INF32 || __ldcg(&rd->grow_chunks) != 0u)) {
      p1++;
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&pc->phase1, 1u);
        sm.ok = wait_geq(&pc->phase1, p1 * gridDim.x, pc, 2u) ? 1u : 0u;
      }
    }
    __syncthreads();
    if (sm.ok) {
      const uint32_t nbig = rd->big ? min(__ldcg(&rd->n_big), rd->big_cap) : 0u;
      for (uint32_t i = warp; i < nbig; i += nwarps) chunk_task(qd, rd, g, i, lane, &sm.w[wib].hdr[0], ws, wb);
    }
    wb_flush(wb, lane);
    if (lane == 0) ws_flush(ws);
    __syncthreads();
    if (!sm.ok) return;
    if (threadIdx.x == 0) {
      __threadfence();
      const uint32_t old = atomicAdd(&pc->arrive, 1u);
      sm.last = old == (r + 1u) * gridDim.x - 1u ? 1u : 0u;
      if (sm.last) {
        __threadfence();  // every block's round work is visible from here on
        pc->rounds = r + 1u;
      }
    }
    __syncthreads();
    if (sm.last && r + 1u < R) {
      control_step(qd, ctl, nslots_ctl, rd, pre, sm.ctl);
      __syncthreads();
      if (threadIdx.x == 0) publish(pc, r + 2u);
    }
    __syncthreads();  // sm.ok and sm.last are rewritten next round
  }
}

// Host side: the round kernels of one block size, 128 or 256 threads (null
// for any other; 512-thread blocks would need more than the 48 KB of static
// shared memory a block can hold: each warp stages its appends in 2 KB).
const void* light_kernel(int threads) {
  return threads == 128 ? (const void*)k_light<4> : threads == 256 ? (const void*)k_light<8> : nullptr;
}
const void* heavy_kernel(int threads) {
  return threads == 128 ? (const void*)k_heavy<4> : threads == 256 ? (const void*)k_heavy<8> : nullptr;
}
const void* rounds_kernel(int threads) {
  return threads == 128 ? (const void*)k_rounds<4> : threads == 256 ? (const void*)k_rounds<8> : nullptr;
}

}  // namespace gstb
