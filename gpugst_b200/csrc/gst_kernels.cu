// CUDA kernels of the gstb engine, sm_100a.
//
// Hot path of one query (the reference's DPBF_GPU, code/GPUGST/src/DPQ.cu:275-624,
// and DPBF_gpu, code/D-GPUGST/src/DPQ.cu:149-269, re-designed):
//   k_sssp_seed   group members -> distance items at 0        (DPQ.cu:359-368)
//   k_work        one frontier round, warp per item:
//                   distance item : multi-source relax of one (vertex, group)
//                                   (replaces dis0_init_1, DPQ.cu:241-271)
//                   DP item       : best update from complement / one-label
//                                   completion, lower-bound prune, grow along
//                                   the weight-sorted adjacency, merge with
//                                   every disjoint subset at the vertex
//                                   (replaces Relax, DPQ.cu:73-172 and
//                                   D-GPUGST/src/DPQ.cu:62-126)
//   k_split       near-far bucketing: moves far items whose cost entered the
//                 new window to the near list
//   k_tour        group-to-group distances and tour tables (host DP at
//                 DPQ.cu:409-483, re-done on device by one CTA)
//   k_dp_seed     cost-0 states of every subset of a member's group mask
//                 (DPQ.cu:341-358)
//   k_extract     follow parents from the best full state into a tree
//                 (the reference's extraction, CPUNONHOP.h:390-432 /
//                 CPUHOP.h:234-259, which its GPU path leaves commented out)
#include "gst_device.cuh"

namespace gstb {

// ---------------------------------------------------------------------------
// Warp-aggregated enqueue.  Every lane of the warp calls it (want may be
// false).  A state is inserted into the near list when its cost is inside the
// current window and into the far list otherwise; a 2-bit flag per state keeps
// each list free of duplicates.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void enqueue_warp(bool want, uint32_t s, uint32_t cost, const QDev& q,
                                             uint32_t* flags, uint32_t lane) {
  bool nearq = cost < q.theta_hi;
  bool take = false;
  if (want) {
    uint32_t bit = 1u << (2u * (s & 15u) + (nearq ? 0u : 1u));
    uint32_t old = atomicOr(&flags[s >> 4], bit);
    take = !(old & bit);
  }
  const unsigned FULL = 0xFFFFFFFFu;
#pragma unroll
  for (int which = 0; which < 2; which++) {
    bool mine = take && ((which == 0) == nearq);
    unsigned m = __ballot_sync(FULL, mine);
    if (m == 0) continue;
    uint32_t leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) {
      uint32_t* cnt = which == 0 ? &q.ctl->n_near : &q.ctl->n_far;
      base = atomicAdd(cnt, (uint32_t)__popc(m));
    }
    base = __shfl_sync(FULL, base, leader);
    if (mine) {
      uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
      uint32_t* buf = which == 0 ? q.qbuf[q.out_idx] : q.qbuf[q.far_idx];
      if (pos < q.cap)
        buf[pos] = s;
      else
        atomicExch(&q.ctl->overflow, 1u);
    }
  }
  unsigned cntm = __popc(__ballot_sync(FULL, take));
  if (lane == 0 && cntm) atomicAdd(&q.ctl->stat[ST_ENQ], (unsigned long long)cntm);
}

// Load the capped group distances of vertex v into every lane's registers.
__device__ __forceinline__ void load_dl(const QDev& q, uint32_t v, uint32_t (&dl)[KMAX],
                                        uint32_t& raw_sum_ok, uint32_t comp,
                                        unsigned long long& raw_sum) {
  const uint4* row = reinterpret_cast<const uint4*>(q.dist + (size_t)v * 8);
  uint4 a = __ldg(row), b = __ldg(row + 1);
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

// ---------------------------------------------------------------------------
// Distance item: relax (v, group j) along arcs whose weight keeps the new
// distance within the best known cost.
// ---------------------------------------------------------------------------
__device__ void sssp_item(const QDev& q, const GraphDev& g, uint32_t s, uint32_t lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  uint32_t v = s >> 3, j = s & 7u;
  if (lane == 0) atomicAnd(&q.sflag[s >> 4], ~(1u << (2u * (s & 15u))));
  __syncwarp();
  uint32_t d = __shfl_sync(FULL, ld_cg(q.dist + s), 0);
  uint32_t best = __shfl_sync(FULL, ld_cg(&q.ctl->best), 0);
  if (d == INF32 || d > best) return;
  // star bound: v joined to every group by its shortest paths (one-label
  // completion of the empty tree at v, CPUNONHOP.h:684-699).  Not a valid
  // bound under a hop limit, so only for unbounded queries.
  if (q.D < 0) {
    uint32_t dj = lane < (uint32_t)q.k ? ld_cg(q.dist + (size_t)v * 8 + lane) : 0u;
    unsigned ok = __all_sync(FULL, dj != INF32);
    unsigned long long sum = dj;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
    if (ok && lane == 0 && sum < best) atomicMin(&q.ctl->best, (uint32_t)sum);
  }
  best = __shfl_sync(FULL, ld_cg(&q.ctl->best), 0);
  if (d > best) return;
  uint32_t lim = best - d;
  uint32_t a0 = __ldg(g.beg + v), a1 = __ldg(g.beg + v + 1);
  uint32_t scanned = 0, upd = 0;
  for (uint32_t base = a0; base < a1; base += 32) {
    uint32_t a = base + lane;
    bool in = a < a1;
    uint2 arc = in ? __ldg(g.adj + a) : make_uint2(0, 0xFFFFFFFFu);
    bool over = arc.y > lim;
    bool want = false;
    uint32_t it = 0, nd = 0;
    if (in && !over) {
      scanned++;
      nd = d + arc.y;
      it = arc.x * 8u + j;
      if (nd < ld_cg(q.dist + it)) {
        uint32_t old = atomicMin(q.dist + it, nd);
        want = nd < old;
        upd += want;
      }
    }
    enqueue_warp(want, it, nd, q, q.sflag, lane);
    if (__any_sync(FULL, over)) break;  // adjacency is sorted by weight
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    scanned += __shfl_xor_sync(FULL, scanned, o);
    upd += __shfl_xor_sync(FULL, upd, o);
  }
  if (lane == 0) {
    atomicAdd(&q.ctl->stat[ST_SSSP], 1ull);
    atomicAdd(&q.ctl->stat[ST_ARCS], (unsigned long long)scanned);
    atomicAdd(&q.ctl->stat[ST_UPDATES], (unsigned long long)upd);
  }
}

// ---------------------------------------------------------------------------
// Unbounded DP item (v, p).
// ---------------------------------------------------------------------------
__device__ void dp_item(const QDev& q, const GraphDev& g, uint32_t s, uint32_t lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  const int k = q.k;
  const uint32_t K2 = 1u << k, full = (uint32_t)q.full;
  const uint32_t v = s >> k, p = s & (K2 - 1u);
  if (lane == 0) atomicAnd(&q.dflag[s >> 4], ~(1u << (2u * (s & 15u))));
  __syncwarp();
  uint32_t c = __shfl_sync(FULL, (uint32_t)(ld_cg(q.table + s) >> 32), 0);
  uint32_t best = __shfl_sync(FULL, ld_cg(&q.ctl->best), 0);
  if (c == INF32 || c > best) return;
  unsigned long long* row = q.table + (size_t)v * K2;
  if (p == full) {
    if (lane == 0) atomicMin(&q.ctl->best, c);
    return;
  }
  const uint32_t comp = full ^ p;
  const uint32_t* P = q.tour;
  const uint32_t* T2 = q.tour + (size_t)k * K2 * k;
  uint32_t dl[KMAX], sum_ok;
  unsigned long long raw_sum;
  load_dl(q, v, dl, sum_ok, comp, raw_sum);
  if (lane == 0) {
    // complement merge straight into the full state (DPQ.cu:82-94)
    uint32_t cc = (uint32_t)(ld_cg(row + comp) >> 32);
    if (cc != INF32) {
      unsigned long long m = (unsigned long long)c + cc;
      if (m < INF32) {
        atomicMin(row + full, pack((uint32_t)m, PAR_MERGE | p));
        atomicMin(&q.ctl->best, (uint32_t)m);
        atomicMin(&q.ctl->best_full, (m << 32) | v);
      }
    }
    // one-label completion: T(v,p) plus shortest paths to the missing groups
    // (DPQ.cu:95-107, CPUNONHOP.h:684-699)
    if (sum_ok) {
      unsigned long long ol = (unsigned long long)c + raw_sum;
      if (ol < INF32) atomicMin(&q.ctl->best, (uint32_t)ol);
    }
    atomicAdd(&q.ctl->stat[ST_EXPANDED], 1ull);
  }
  __syncwarp();
  best = __shfl_sync(FULL, ld_cg(&q.ctl->best), 0);
  uint32_t lbv = lower_bound_comp(dl, k, comp, P, T2);
  if ((unsigned long long)c + lbv > best) return;

  uint32_t scanned = 0, upd = 0;
  // grow, only from states of cost <= best/2 (optimal-tree decomposition,
  // CPUNONHOP.h:820; exact for the unbounded problem, see DESIGN)
  if (2ull * c <= best) {
    uint32_t lim = best - c;
    uint32_t a0 = __ldg(g.beg + v), a1 = __ldg(g.beg + v + 1);
    for (uint32_t base = a0; base < a1; base += 32) {
      uint32_t a = base + lane;
      bool in = a < a1;
      uint2 arc = in ? __ldg(g.adj + a) : make_uint2(0, 0xFFFFFFFFu);
      bool over = arc.y > lim;
      bool want = false;
      uint32_t t = 0, nc = 0;
      if (in && !over) {
        scanned++;
        nc = c + arc.y;
        t = (arc.x << k) | p;
        if (nc < (uint32_t)(ld_cg(q.table + t) >> 32)) {
          uint32_t dlu[KMAX], okb;
          unsigned long long rs;
          load_dl(q, arc.x, dlu, okb, comp, rs);
          uint32_t lbu = lower_bound_comp(dlu, k, comp, P, T2);
          if ((unsigned long long)nc + lbu <= best) {
            unsigned long long old = atomicMin(q.table + t, pack(nc, PAR_GROW | v));
            want = (uint32_t)(old >> 32) > nc;
            upd += want;
          }
        }
      }
      enqueue_warp(want, t, nc, q, q.dflag, lane);
      if (__any_sync(FULL, over)) break;
    }
  }
  // merge with every proper, non-empty subset p2 of the complement
  // (DPQ.cu:140-170; the complement itself went to the full state above)
  {
    const uint32_t nsub = (1u << __popc(comp)) - 2u;
    uint32_t merges = 0;
    for (uint32_t b = 0; b < nsub; b += 32) {
      uint32_t idx = b + lane;
      bool want = false;
      uint32_t t = 0, m32 = 0;
      if (idx < nsub) {
        uint32_t p2 = pdep(idx + 1u, comp);
        uint32_t c2 = (uint32_t)(ld_cg(row + p2) >> 32);
        if (c2 != INF32) {
          merges++;
          unsigned long long m = (unsigned long long)c + c2;
          uint32_t qset = p | p2;
          // conditional tree merging: 3m <= 2 best (CPUNONHOP.h:941)
          if (3ull * m <= 2ull * best) {
            uint32_t lbq = lower_bound_comp(dl, k, full ^ qset, P, T2);
            if (m + lbq <= best) {
              m32 = (uint32_t)m;
              t = (v << k) | qset;
              unsigned long long old = atomicMin(q.table + t, pack(m32, PAR_MERGE | p));
              want = (uint32_t)(old >> 32) > m32;
              upd += want;
            }
          }
        }
      }
      enqueue_warp(want, t, m32, q, q.dflag, lane);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) merges += __shfl_xor_sync(FULL, merges, o);
    if (lane == 0 && merges) atomicAdd(&q.ctl->stat[ST_MERGES], (unsigned long long)merges);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    scanned += __shfl_xor_sync(FULL, scanned, o);
    upd += __shfl_xor_sync(FULL, upd, o);
  }
  if (lane == 0) {
    atomicAdd(&q.ctl->stat[ST_ARCS], (unsigned long long)scanned);
    atomicAdd(&q.ctl->stat[ST_UPDATES], (unsigned long long)upd);
  }
}

// ---------------------------------------------------------------------------
// Hop-bounded DP item (v, p, d): state id ((v << k) | p) * nd + d.
// ---------------------------------------------------------------------------
__device__ void hop_item(const QDev& q, const GraphDev& g, uint32_t s, uint32_t lane) {
  const unsigned FULL = 0xFFFFFFFFu;
  const int k = q.k, nd = q.nd, D = q.D;
  const uint32_t K2 = 1u << k, full = (uint32_t)q.full;
  const uint32_t d = s % (uint32_t)nd, vp = s / (uint32_t)nd;
  const uint32_t v = vp >> k, p = vp & (K2 - 1u);
  if (lane == 0) atomicAnd(&q.dflag[s >> 4], ~(1u << (2u * (s & 15u))));
  __syncwarp();
  uint32_t c = __shfl_sync(FULL, (uint32_t)(ld_cg(q.table + s) >> 32), 0);
  uint32_t best = __shfl_sync(FULL, ld_cg(&q.ctl->best), 0);
  if (c == INF32 || c > best) return;
  // dominance: the same subset at a smaller hop count and no higher cost
  {
    bool dom = false;
    if (lane < d) dom = (uint32_t)(ld_cg(q.table + (size_t)vp * nd + lane) >> 32) <= c;
    if (__any_sync(FULL, dom)) return;
  }
  if (p == full) {
    if (lane == 0) atomicMin(&q.ctl->best, c);
    return;
  }
  const uint32_t comp = full ^ p;
  const uint32_t* P = q.tour;
  const uint32_t* T2 = q.tour + (size_t)k * K2 * k;
  uint32_t dl[KMAX], sum_ok;
  unsigned long long raw_sum;
  load_dl(q, v, dl, sum_ok, comp, raw_sum);
  if (lane == 0) atomicAdd(&q.ctl->stat[ST_EXPANDED], 1ull);
  uint32_t lbv = lower_bound_comp(dl, k, comp, P, T2);
  if ((unsigned long long)c + lbv > best) return;
  uint32_t scanned = 0, upd = 0;
  if (d < (uint32_t)D) {  // grow d -> d+1 (CPUHOP.h:192-206)
    uint32_t lim = best - c;
    uint32_t a0 = __ldg(g.beg + v), a1 = __ldg(g.beg + v + 1);
    for (uint32_t base = a0; base < a1; base += 32) {
      uint32_t a = base + lane;
      bool in = a < a1;
      uint2 arc = in ? __ldg(g.adj + a) : make_uint2(0, 0xFFFFFFFFu);
      bool over = arc.y > lim;
      bool want = false;
      uint32_t t = 0, nc = 0;
      if (in && !over) {
        scanned++;
        nc = c + arc.y;
        t = ((arc.x << k) | p) * (uint32_t)nd + d + 1;
        if (nc < (uint32_t)(ld_cg(q.table + t) >> 32)) {
          uint32_t dlu[KMAX], okb;
          unsigned long long rs;
          load_dl(q, arc.x, dlu, okb, comp, rs);
          uint32_t lbu = lower_bound_comp(dlu, k, comp, P, T2);
          if ((unsigned long long)nc + lbu <= best) {
            unsigned long long old = atomicMin(q.table + t, pack(nc, PAR_GROW | v));
            want = (uint32_t)(old >> 32) > nc;
            upd += want;
          }
        }
      }
      enqueue_warp(want, t, nc, q, q.dflag, lane);
      if (__any_sync(FULL, over)) break;
    }
  }
  // merge with (v, p2, d2), p2 a non-empty subset of the complement,
  // d2 <= D - d, into (v, p|p2, max(d, d2))  (CPUHOP.h:208-227)
  {
    const uint32_t nsub = (1u << __popc(comp)) - 1u;
    const uint32_t nd2 = (uint32_t)D - d + 1u;
    const uint32_t npairs = nsub * nd2;
    unsigned long long* rowv = q.table + ((size_t)v << k) * nd;
    uint32_t merges = 0;
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
          if (m < INF32) {
            m32 = (uint32_t)m;
            t = ((v << k) | qset) * (uint32_t)nd + ndd;
            if (qset == full) {
              atomicMin(q.table + t, pack(m32, par));
              atomicMin(&q.ctl->best, m32);
              atomicMin(&q.ctl->best_full, ((unsigned long long)m32 << 32) | (v * 8u + ndd));
            } else {
              uint32_t lbq = lower_bound_comp(dl, k, full ^ qset, P, T2);
              if (m + lbq <= best) {
                unsigned long long old = atomicMin(q.table + t, pack(m32, par));
                want = (uint32_t)(old >> 32) > m32;
                upd += want;
              }
            }
          }
        }
      }
      enqueue_warp(want, t, m32, q, q.dflag, lane);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) merges += __shfl_xor_sync(FULL, merges, o);
    if (lane == 0 && merges) atomicAdd(&q.ctl->stat[ST_MERGES], (unsigned long long)merges);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    scanned += __shfl_xor_sync(FULL, scanned, o);
    upd += __shfl_xor_sync(FULL, upd, o);
  }
  if (lane == 0) {
    atomicAdd(&q.ctl->stat[ST_ARCS], (unsigned long long)scanned);
    atomicAdd(&q.ctl->stat[ST_UPDATES], (unsigned long long)upd);
  }
}

// Find the job owning flat work index `it` (prefix is exclusive, size njobs+1).
__device__ __forceinline__ int find_job(const uint32_t* __restrict__ prefix, int njobs, uint32_t it) {
  int lo = 0, hi = njobs;  // prefix[lo] <= it < prefix[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (__ldg(prefix + mid) <= it)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(256) k_work(const QDev* __restrict__ qd, const uint32_t* __restrict__ jobs,
                                              const uint32_t* __restrict__ prefix, int njobs,
                                              uint32_t total, GraphDev g) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t it = warp; it < total; it += nwarps) {
    int j = find_job(prefix, njobs, it);
    const QDev& q = qd[__ldg(jobs + j)];
    uint32_t s = q.qbuf[q.in_idx][it - __ldg(prefix + j)];
    if (q.phase == PH_SSSP)
      sssp_item(q, g, s, lane);
    else if (q.phase == PH_DP)
      dp_item(q, g, s, lane);
    else
      hop_item(q, g, s, lane);
  }
}

// Near-far split: far items whose cost is in [theta_lo, theta_hi) move to the
// near list; costs above stay; costs below theta_lo were already expanded at
// that cost (every new cost is >= the cost of the item that produced it).
__global__ void __launch_bounds__(256) k_split(const QDev* __restrict__ qd, const uint32_t* __restrict__ jobs,
                                               const uint32_t* __restrict__ prefix, int njobs,
                                               uint32_t total) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < total; it += stride) {
    int j = find_job(prefix, njobs, it);
    const QDev& q = qd[__ldg(jobs + j)];
    uint32_t s = q.qbuf[q.far_idx][it - __ldg(prefix + j)];
    uint32_t* flags = q.phase == PH_SSSP ? q.sflag : q.dflag;
    uint32_t cost = q.phase == PH_SSSP ? ld_cg(q.dist + s) : (uint32_t)(ld_cg(q.table + s) >> 32);
    uint32_t best = ld_cg(&q.ctl->best);
    uint32_t sh = 2u * (s & 15u);
    if (cost < q.theta_lo || cost == INF32 || cost > best) {
      atomicAnd(&flags[s >> 4], ~(2u << sh));
    } else if (cost < q.theta_hi) {
      atomicAnd(&flags[s >> 4], ~(2u << sh));
      uint32_t old = atomicOr(&flags[s >> 4], 1u << sh);
      if (!(old & (1u << sh))) {
        uint32_t pos = atomicAdd(&q.ctl->n_near, 1u);
        if (pos < q.cap)
          q.qbuf[q.out_idx][pos] = s;
        else
          atomicExch(&q.ctl->overflow, 1u);
      }
    } else {
      uint32_t pos = atomicAdd(&q.ctl->n_far2, 1u);
      if (pos < q.cap)
        q.qbuf[q.far2_idx][pos] = s;
      else
        atomicExch(&q.ctl->overflow, 1u);
    }
  }
}

// Members -> distance items at distance 0, all in the first near list.
__global__ void k_sssp_seed(const QDev* __restrict__ qd, const uint32_t* __restrict__ jobs,
                            const uint32_t* __restrict__ prefix, int njobs, uint32_t total) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < total; it += stride) {
    int j = find_job(prefix, njobs, it);
    const QDev& q = qd[__ldg(jobs + j)];
    uint32_t s = __ldg(q.members + (it - __ldg(prefix + j)));
    q.dist[s] = 0;
    uint32_t old = atomicOr(&q.sflag[s >> 4], 1u << (2u * (s & 15u)));
    if (!(old & (1u << (2u * (s & 15u))))) {
      uint32_t pos = atomicAdd(&q.ctl->n_near, 1u);
      if (pos < q.cap)
        q.qbuf[q.out_idx][pos] = s;
      else
        atomicExch(&q.ctl->overflow, 1u);
    }
  }
}

// Cost-0 states: every non-empty subset of a member's mask (DPQ.cu:341-358).
// The member item of the lowest group bit of the mask does the seeding.
__global__ void k_dp_seed(const QDev* __restrict__ qd, const uint32_t* __restrict__ jobs,
                          const uint32_t* __restrict__ prefix, int njobs, uint32_t total) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < total; it += stride) {
    int j = find_job(prefix, njobs, it);
    const QDev& q = qd[__ldg(jobs + j)];
    uint32_t item = __ldg(q.members + (it - __ldg(prefix + j)));
    uint32_t v = item >> 3, gi = item & 7u;
    uint32_t m = 0;
    for (int t = 0; t < q.k; t++)
      if (q.dist[(size_t)v * 8 + t] == 0) m |= 1u << t;
    if (m == 0 || (uint32_t)(__ffs(m) - 1) != gi) continue;
    for (uint32_t sub = m; sub; sub = (sub - 1u) & m) {
      uint32_t s = q.phase == PH_HOP ? ((v << q.k) | sub) * (uint32_t)q.nd : ((v << q.k) | sub);
      q.table[s] = pack(0u, 0u);
      if (sub == (uint32_t)q.full) {  // v is in every query group: a cost-0 tree
        atomicMin(&q.ctl->best, 0u);
        atomicMin(&q.ctl->best_full, q.phase == PH_HOP ? (unsigned long long)(v * 8u) : (unsigned long long)v);
        continue;
      }
      uint32_t old = atomicOr(&q.dflag[s >> 4], 1u << (2u * (s & 15u)));
      if (!(old & (1u << (2u * (s & 15u))))) {
        uint32_t pos = atomicAdd(&q.ctl->n_near, 1u);
        if (pos < q.cap)
          q.qbuf[q.out_idx][pos] = s;
        else
          atomicExch(&q.ctl->overflow, 1u);
      }
    }
  }
}

// One CTA per query: group-to-group distances gd[i][j] = min over members of
// group i of the (capped) distance to group j, then the tour tables
//   P[i][S][j]  cheapest visiting order of S starting at i, ending at j
//   T2[i][S]    min_j P[i][S][j]
// (replaces the host DP of DPQ.cu:409-483 / AllPaths, CPUNONHOP.h:269-386).
__global__ void __launch_bounds__(256) k_tour(const QDev* __restrict__ qd, const uint32_t* __restrict__ jobs) {
  const QDev& q = qd[jobs[blockIdx.x]];
  const int k = q.k;
  const uint32_t K2 = 1u << k;
  __shared__ uint32_t gd[KMAX][KMAX];
  for (int t = threadIdx.x; t < KMAX * KMAX; t += blockDim.x) gd[t / KMAX][t % KMAX] = BIG;
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < q.n_members; t += blockDim.x) {
    uint32_t item = q.members[t];
    uint32_t v = item >> 3, i = item & 7u;
    for (int j = 0; j < k; j++) {
      uint32_t dj = min(q.dist[(size_t)v * 8 + j], q.cap1);
      atomicMin(&gd[i][j], dj);
    }
  }
  __syncthreads();
  uint32_t* P = q.tour;
  uint32_t* T2 = q.tour + (size_t)k * K2 * k;
  const uint32_t nP = (uint32_t)k * K2 * (uint32_t)k;
  for (uint32_t t = threadIdx.x; t < nP; t += blockDim.x) P[t] = BIG;
  __syncthreads();
  for (int i = threadIdx.x; i < k; i += blockDim.x) P[((size_t)i * K2 + (1u << i)) * k + i] = 0;
  __syncthreads();
  for (int size = 2; size <= k; size++) {
    // entries (i, S, l) with |S| = size, i in S, l in S \ {i}
    for (uint32_t t = threadIdx.x; t < nP; t += blockDim.x) {
      uint32_t l = t % k, S = (t / k) % K2, i = t / (k * K2);
      if ((uint32_t)__popc(S) != (uint32_t)size || !(S >> i & 1u) || !(S >> l & 1u) || l == i) continue;
      uint32_t Sp = S ^ (1u << l);
      uint32_t bestv = BIG;
      for (int jj = 0; jj < k; jj++)
        if (Sp >> jj & 1u) bestv = min(bestv, sat_add(P[((size_t)i * K2 + Sp) * k + jj], gd[jj][l]));
      P[t] = bestv;
    }
    __syncthreads();
  }
  for (uint32_t t = threadIdx.x; t < (uint32_t)k * K2; t += blockDim.x) {
    uint32_t i = t / K2, S = t % K2;
    uint32_t m = BIG;
    for (int l = 0; l < k; l++) m = min(m, P[((size_t)i * K2 + S) * k + l]);
    T2[t] = m;
  }
}

// Weight of arc (a -> b): linear scan of a's weight-sorted adjacency.
__device__ uint32_t arc_weight(const GraphDev& g, uint32_t a, uint32_t b) {
  for (uint32_t x = g.beg[a]; x < g.beg[a + 1]; x++) {
    uint2 arc = g.adj[x];
    if (arc.x == b) return arc.y;
  }
  return INF32;
}

// One thread per query: follow parent words from the best full state,
// emitting (u, v, w) edges; qbuf[0] serves as the explicit stack.
__global__ void k_extract(const QDev* __restrict__ qd, const uint32_t* __restrict__ jobs, int njobs,
                          GraphDev g) {
  int jj = blockIdx.x * blockDim.x + threadIdx.x;
  if (jj >= njobs) return;
  const QDev& q = qd[jobs[jj]];
  QCtl* ctl = q.ctl;
  unsigned long long bf = ctl->best_full;
  if (bf == INF64) {
    ctl->status = 1;
    ctl->n_edges = 0;
    return;
  }
  const int k = q.k, nd = q.nd;
  const bool hop = q.phase == PH_HOP;
  uint32_t payload = (uint32_t)bf;
  uint32_t root = hop ? payload >> 3 : payload;
  uint32_t rd = hop ? (payload & 7u) : 0u;
  uint32_t* stack = q.qbuf[0];
  uint32_t sp = 0;
  uint32_t full = (uint32_t)q.full;
  stack[sp++] = hop ? ((root << k) | full) * (uint32_t)nd + rd : ((root << k) | full);
  uint32_t ne = 0;
  uint32_t steps = 0;
  const uint32_t max_steps = 4u * g.V + 64u;
  uint32_t status = 0;
  while (sp > 0) {
    if (++steps > max_steps || sp + 2 > q.cap) {
      status = 2;
      break;
    }
    uint32_t s = stack[--sp];
    uint32_t d = hop ? s % (uint32_t)nd : 0u;
    uint32_t vp = hop ? s / (uint32_t)nd : s;
    uint32_t v = vp >> k, p = vp & ((1u << k) - 1u);
    unsigned long long e = q.table[s];
    if ((uint32_t)(e >> 32) == INF32) {
      status = 2;
      break;
    }
    uint32_t par = (uint32_t)e;
    uint32_t type = par >> 30;
    if (type == 1u) {
      uint32_t u = par & 0x3FFFFFFFu;
      if (ne < q.max_edges) {
        q.out_edges[3 * ne] = u;
        q.out_edges[3 * ne + 1] = v;
        q.out_edges[3 * ne + 2] = arc_weight(g, v, u);
      }
      ne++;
      if (hop) {
        if (d == 0) {
          status = 2;
          break;
        }
        stack[sp++] = ((u << k) | p) * (uint32_t)nd + d - 1;
      } else {
        stack[sp++] = (u << k) | p;
      }
    } else if (type == 2u) {
      uint32_t p1 = par & 0xFFu, p2 = p ^ p1;
      if (p1 == 0 || p2 == 0 || (p1 & ~p) != 0) {
        status = 2;
        break;
      }
      if (hop) {
        uint32_t d1 = (par >> 8) & 7u, d2 = (par >> 11) & 7u;
        stack[sp++] = ((v << k) | p1) * (uint32_t)nd + d1;
        stack[sp++] = ((v << k) | p2) * (uint32_t)nd + d2;
      } else {
        stack[sp++] = (v << k) | p1;
        stack[sp++] = (v << k) | p2;
      }
    } else if (type != 0u) {
      status = 2;
      break;
    }
  }
  ctl->status = status;
  ctl->n_edges = ne;
  ctl->root = root;
}

}  // namespace gstb
