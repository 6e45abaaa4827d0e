// Device-side data layout and helpers of the gstb engine (sm_100a).
//
// HBM layout of one query (all arrays owned by the engine):
//   table  u64 [V][2^k][nd]   packed  cost << 32 | parent   (nd = D+1, or 1 unbounded)
//                              parent: 00 seed | 01 grow (30-bit predecessor vertex)
//                                      | 10 merge (p1 : 8 bits, d1 : 3, d2 : 3)
//                              INF = all ones (memset 0xFF); a 64-bit atomicMin keeps
//                              cost and parent consistent (no torn parents, unlike the
//                              reference's separate stores at DPQ.cu:117-121).
//   dist   u32 [V][8]          one 32-byte sector per vertex: words 0..6 the
//                               shortest distance from query group j to v,
//                               word 7 the groups of v pending in the near list
//                               (bits 0-7 and 8-15: the two round parities) and
//                               in the far list (bits 16-23).  A relaxation
//                               reads the target's distances and flags with one
//                               sector load and updates both in that sector.
//   dflag  u32 [ceil(V*2^k*nd/8)]   4 bits per state: in-near (two round
//                                   parities), in-far
//   qbuf   u32 [4][cap]        near-in, near-out, far, far-out work lists of state ids
//   tour   u32 [k][2^k][k] + [k][2^k] + [8][8]  tour tables P, T2 and group distances
//   lbt    u16 [V][2^k]        lower bound of completing (v, X) to every group
//   snap   u32 [D-1][V][8]     hop-bounded queries: the distance rows after
//                               Bellman-Ford round b (b = 1..D-1), i.e. lower
//                               bounds of the cheapest paths of at most b hops
#pragma once
#include <cstdint>

namespace gstb {

constexpr uint32_t INF32 = 0xFFFFFFFFu;
constexpr unsigned long long INF64 = 0xFFFFFFFFFFFFFFFFull;
constexpr uint32_t BIG = 1u << 30;  // saturation value inside lower-bound sums
constexpr uint32_t PAR_GROW = 0x40000000u;
constexpr uint32_t PAR_MERGE = 0x80000000u;
constexpr int KMAX = 7;        // query groups at most (word 7 of a distance row holds flags)
constexpr int ROW = 8;         // words per distance row
constexpr int FLAGW = 7;       // the pending-flags word of a row
constexpr uint32_t FAR_SH = 16;  // far-list byte of the flags word
__device__ __forceinline__ uint32_t near_sh(uint32_t par) { return par * 8u; }  // near-list byte of a parity
constexpr int DMAX = 7;

// Job state machine (advanced on the device by k_control once per round).
enum JobState : int32_t { J_FREE = 0, J_INIT, J_SSSP, J_TOUR, J_LB, J_DPSEED, J_DP, J_EXTRACT, J_DONE };
enum Action : int32_t { A_NONE = 0, A_SSEED, A_WORK, A_SPLIT, A_TOUR, A_LB, A_DSEED, A_EXTRACT };

// Task types of one round.  Light kernel: split, seeds, tour, extract,
// distance items and DP states; heavy kernel: the arc chunks the light kernel
// handed over, then lower-bound table rows.
enum TaskType : int32_t { T_SPLIT = 0, T_SSEED, T_DSEED, T_TOUR, T_EXTRACT, T_SSSP, T_DP, T_HOP, T_LB, T_SNAP, NT };
constexpr int MAX_SLOTS = 1024;

// Round-wide work description written by k_control.
struct RoundDesc {
  uint32_t items[NT];     // items per task type
  uint32_t task_off[NT + 1];  // warp-task offsets (light types, then heavy types restart at 0)
  uint32_t light_tasks, heavy_tasks;
  uint32_t n_live;        // slots whose job is not finished
  uint32_t n_big;         // arc chunks queued by k_light for k_heavy this round
  // arc chunks: distance items {slot | groups << 16, vertex, first arc, end arc},
  // DP grow chunks {slot | 1 << 31 (| 1 << 30 hop-bounded), state, first arc,
  // end arc}; set once by the host (null / 0 disables chunking)
  uint4* big;
  uint32_t big_cap;
  uint32_t hub_min_deg;   // only items with at least this many arcs under their limit are chunked
  uint32_t hub_min_rest;  // ... and only when at least this many arcs remain under the limit
  uint32_t hub_max_items; // chunk only in rounds with fewer distance items (latency-bound rounds)
  uint32_t hub_on;        // set by k_control for the current round
  // larger rounds: items of at least hub_big_deg arcs are still chunked in
  // rounds with fewer than hub_max_items2 distance items (0: never)
  uint32_t hub_max_items2, hub_big_deg;
  // ... and only when they exceed 1/hub_share_div of a warp's share of the
  // round's arcs (items x avg_deg / light_warps; 0: no such test)
  uint32_t hub_share_div, avg_deg;
  uint32_t hub_deg;       // this round's chunking threshold for distance items (INF32: none; k_control)
  uint32_t grow_chunks;   // DP grows hand hub arcs out this round (set by k_control)
  uint32_t sssp_w;        // distance items per warp task this round (set by k_control)
  uint32_t dp_w;          // DP states per warp task this round (set by k_control)
  uint32_t dp_wmax;       // largest DP task width (set by the host)
  uint32_t sssp_wmax;     // largest distance task width, at most SSSP_WMAX (set by the host)
  uint32_t merge_stage;   // a DP state with at least this many merge partners stages its row (0: never; host)
  uint32_t light_warps;   // warps of one k_light launch (set by the host)
  uint32_t nslots;        // 1 + the highest slot in use this round (set by k_control)
  // work stealing: a warp that finished its first task takes the next one
  // from these counters (zeroed by k_control every round)
  uint32_t next_light, next_heavy;
};
// State of one persistent round launch (k_rounds), written by the host
// before each launch (the counters zero).
// The polled word and the two arrival counters sit in cache lines of their
// own, so that polling blocks do not queue on the counters' atomics.
struct PersistCtl {
  alignas(128) uint32_t epoch;  // control steps published (round r's work waits for epoch >= r + 1)
  alignas(128) uint32_t arrive; // blocks that finished their round work, summed over rounds
  alignas(128) uint32_t phase1; // blocks done with the light and static heavy tasks, summed over chunk rounds
  alignas(128) uint32_t err;    // 1: a bounded wait expired, the launch stopped
  uint32_t err_where;  // the first wait that expired: 1 control step, 2 light tasks
  uint32_t rounds;   // rounds completed
  uint32_t hold;     // 1: control steps are not published (makes the waits expire; a test of them)
  uint32_t pad;
  unsigned long long timeout_ns;  // limit of every wait
};
#ifndef GSTB_HUB_CHUNK
#define GSTB_HUB_CHUNK 256
#endif
constexpr uint32_t HUB_CHUNK = GSTB_HUB_CHUNK;  // arcs per chunk (one warp)
constexpr uint32_t LB_CHUNK = 1u << 22; // bound-table rows (vertices) per query per round

enum Phase : int32_t {
  PH_IDLE = 0,
  PH_SSSP = 1,
  PH_DP = 2,   // unbounded DPBF
  PH_HOP = 3,  // hop-bounded DPBF
};

// Statistics slots (match GST_STAT_* in gstb.h).
enum {
  ST_EXPANDED = 0,
  ST_SSSP = 1,
  ST_ARCS = 2,
  ST_UPDATES = 3,
  ST_ENQ = 4,
  ST_ROUNDS = 5,
  ST_MERGES = 6,
  ST_SSSP_ARCS = 8,
  ST_SSSP_UPDATES = 9,
  ST_SSSP_ENQ = 10,
};

// Written by kernels, read back by the host after every round.  The fields
// sit in separate 32-byte sectors by access pattern: the incumbent is read by
// every item, the list counters take one atomic per warp step, the statistics
// are added once per warp and query, the rest is written once.
struct alignas(64) QCtl {
  // sector 0: the incumbent
  uint32_t best;     // best feasible cost known (upper bound)
  uint32_t root;
  unsigned long long best_full;  // min over full states of cost << 32 | payload
  uint32_t infeasible;  // the query groups are not connected
  uint32_t center;   // hop-bounded: some vertex has every group within ceil(D/2) hops
  uint32_t pad0[2];
  // sector 1: list append counters
  uint32_t n_near;   // append counter of the near-out list
  uint32_t n_far;    // append counter of the far list
  uint32_t n_far2;   // append counter of the far-out list (split rounds)
  uint32_t overflow; // a list exceeded its capacity
  uint32_t pad1[4];
  // sectors 2-4: statistics
  unsigned long long stat[12];
  // sector 5: completion
  uint32_t n_edges;  // extraction: number of tree edges
  uint32_t status;   // extraction: 0 ok, 1 no solution, 2 cycle / inconsistency
  uint32_t done;     // job finished (set by k_control)
  uint32_t final_status;  // gst_status of the finished job
  uint32_t cancel;   // set by the host: end the job at the next round (GST_CANCELLED)
  uint32_t early;    // progressive mode: the DP stopped early (1) ...
  uint32_t lb_exit;  // ... with this lower bound on the optimum proven
  uint32_t pad2[1];
};

// Per-query descriptor; the host rewrites it before each round.
struct QDev {
  unsigned long long* table;
  uint32_t* dist;
  uint32_t* dflag;
  uint32_t* qbuf[4];
  uint32_t* tour;
  unsigned short* lbt;      // [V][2^k] lower bound per (vertex, uncovered set)
  const uint32_t* members;  // distance items v*8+j of every query-group member
  uint32_t* out_edges;      // extraction output (u, v, w) triples
  QCtl* ctl;
  uint32_t cap;
  uint32_t nv;              // number of vertices
  uint32_t n_members;
  uint32_t max_edges;
  int32_t k, D, nd, full;
  uint32_t WT;       // 2^k * nd entries per vertex
  int32_t phase;
  // round fields
  int32_t in_idx, out_idx, far_idx, far2_idx;
  uint32_t n_in;     // items in qbuf[in_idx]
  uint32_t n_far;    // items in qbuf[far_idx] (split input)
  uint32_t theta_lo, theta_hi;  // current near window [lo, hi)
  uint32_t cap1;     // distances >= cap1 are only known to be >= cap1
  uint32_t cap_num, cap_den;  // distance rounds stop at best * cap_num / cap_den
  // state machine
  int32_t st, act;
  uint32_t delta, delta_sssp, delta_dp;
  uint32_t par;      // parity of the items in (or entering) the near list
  uint32_t lb_off;   // bound-table rows (vertices) already computed
  uint32_t hops;     // distance rounds done (hop-bounded queries stop after D)
  uint32_t snap_h;   // distance round whose rows k_heavy copies to snap this round (0: none)
  uint32_t snap_n;   // snapshots taken (rows for b hops: snap[b-1] if b <= snap_n, else dist)
  uint32_t pad_s;
  uint32_t* snap;    // [D-1][V][8] (hop-bounded queries)
  // Distance rows written by a distance round.  Unbounded queries relax in
  // place (dist_nx == dist).  Hop-bounded queries run exact (Jacobi)
  // Bellman-Ford rounds over two row buffers: round b reads dist (the exact
  // distances over paths of at most b-1 hops) and writes dist_nx, and
  // k_control swaps the two after the round.
  uint32_t* dist_nx;
  // Hop-bounded queries (D >= 2): the round whose exact rows give the
  // incumbent (star_h = floor(D/2): a vertex with every group within star_h
  // hops spans a tree of diameter <= D) and the round whose rows decide
  // feasibility (center_h = ceil(D/2): every tree of diameter <= D has a
  // vertex with every group within center_h hops).  0: none.
  uint32_t star_h, center_h;
  uint32_t center_done;  // the feasibility pass has run
  // progressive mode: return the best recorded tree once its cost is at most
  // ratio_num / ratio_den times the proven lower bound (ratio_num 0: exact)
  uint32_t ratio_num, ratio_den;
};

struct GraphDev {
  const uint32_t* beg;   // [V+1]
  const uint2* adj;      // [arcs] {neighbour, weight}, each list sorted by (weight, neighbour)
  uint32_t V;
  const uint32_t* wcut;  // [V][8]: first arc of v with weight > 2^b (b = 0..7), or null
};

// Upper bound on the end of the arcs of v whose weight is <= lim (the list is
// sorted by weight): one load of the bucket index instead of a search.
__device__ __forceinline__ uint32_t arcs_upto(const GraphDev& g, uint32_t v, uint32_t a1, uint32_t lim) {
  if (g.wcut == nullptr || lim > 128u) return a1;
  uint32_t b = lim <= 1u ? 0u : 32u - __clz(lim - 1u);  // smallest b with 2^b >= lim
  return __ldg(g.wcut + (size_t)v * 8 + b);
}

// DP state flags: 4 bits per state, 8 states per word.  Bits 0 and 1 mark
// "in the near list" for the two round parities, bit 2 "in the far list".
__device__ __forceinline__ uint32_t dflag_bit(uint32_t s, uint32_t b) { return 1u << (4u * (s & 7u) + b); }

__device__ __forceinline__ unsigned long long pack(uint32_t cost, uint32_t par) {
  return ((unsigned long long)cost << 32) | par;
}

// Fire-and-forget reductions (PTX red): the issuing warp never waits for them.
__device__ __forceinline__ void red_min(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.min.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_min(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.min.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_or(uint32_t* p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Loads of data that a launch may itself have written in an earlier round
// (distance rows, bound and tour tables): cached in L1, but as ordinary weak
// loads, which the fences between rounds order.  The non-coherent read-only
// path (__ldg) is kept for data that no launch writes (the graph, member lists).
template <class T>
__device__ __forceinline__ T ld_round(const T* p) {
  return __ldca(p);
}
__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) { return __ldcg(p); }
// The incumbent through L1: a value cached earlier in the same launch can be
// higher than the current one, which only weakens pruning (every use of best
// is an upper bound), and it spares the incumbent's L2 sector a read per item.
__device__ __forceinline__ uint32_t ld_best(const QCtl* c) { return __ldca(&c->best); }
__device__ __forceinline__ unsigned long long ld_cg(const unsigned long long* p) { return __ldcg(p); }

// Software parallel-bit-deposit of the low bits of x into the set bits of mask.
__device__ __forceinline__ uint32_t pdep(uint32_t x, uint32_t mask) {
  uint32_t r = 0;
  while (mask) {
    uint32_t low = mask & (0u - mask);
    if (x & 1u) r |= low;
    x >>= 1;
    mask ^= low;
  }
  return r;
}

__device__ __forceinline__ uint32_t sat_add(uint32_t a, uint32_t b) {
  uint32_t s = a + b;
  return (s < a || s > BIG) ? BIG : s;
}

// Lower bound on the cost of connecting a vertex (with group distances dl[],
// already capped) to every group of `comp`:
//   one-label  max_j dl_j                                   (DPQ.cu:182-188)
//   tour lb1   min_{i,j} ceil((dl_i + P[i][comp][j] + dl_j)/2)   (CPUNONHOP.h:448-466)
//   tour lb2   max_i ceil((dl_i + T2[i][comp] + min_j dl_j)/2)   (CPUNONHOP.h:468-472)
// P[i][S][j] = cheapest order of visiting the groups of S starting at i and
// ending at j with group-to-group distances as step costs; T2 = min_j P.
__device__ __forceinline__ uint32_t lower_bound_comp(const uint32_t (&dl)[KMAX], int k,
                                                     uint32_t comp, const uint32_t* __restrict__ P,
                                                     const uint32_t* __restrict__ T2) {
  if (comp == 0) return 0;
  const uint32_t K2 = 1u << k;
  uint32_t lb0 = 0, mind = BIG;
#pragma unroll
  for (int j = 0; j < KMAX; j++)
    if (j < k && (comp >> j & 1u)) {
      lb0 = max(lb0, dl[j]);
      mind = min(mind, dl[j]);
    }
  uint32_t lb1 = BIG, lb2 = 0;
#pragma unroll
  for (int i = 0; i < KMAX; i++) {
    if (i < k && (comp >> i & 1u)) {
      const uint32_t* Pi = P + ((size_t)i * K2 + comp) * k;
#pragma unroll
      for (int j = 0; j < KMAX; j++)
        if (j < k && (comp >> j & 1u)) {
          uint32_t t = sat_add(sat_add(dl[i], ld_round(Pi + j)), dl[j]);
          lb1 = min(lb1, (t + 1) >> 1);
        }
      uint32_t t2 = sat_add(sat_add(dl[i], ld_round(T2 + (size_t)i * K2 + comp)), mind);
      lb2 = max(lb2, (t2 + 1) >> 1);
    }
  }
  return max(lb0, max(lb1 >= BIG ? BIG : lb1, lb2));
}

}  // namespace gstb
