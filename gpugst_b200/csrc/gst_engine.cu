// Host side of the gstb engine: graph / group index residency, the round
// driver shared by the single-query, batched and serving paths, and the C ABI
// declared in include/gstb.h.
//
// One "round" = one launch of each kernel that has work, for every admitted
// query at once, followed by a single read-back of the per-query control
// blocks.  A query walks through
//   INIT -> SSSP (near-far rounds) -> TOUR -> DP seed -> DP (near-far rounds)
//        -> EXTRACT -> DONE
// The reference instead synchronises the host after every Bellman-Ford /
// Relax launch of a single query (DPQ.cu:378-404, 512-544).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <shared_mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/gstb.h"
#include "gst_device.cuh"

namespace gstb {
__global__ void k_control(QDev*, QCtl*, int, RoundDesc*, uint32_t*);
// the round kernels of a block size (128 or 256 threads; null otherwise)
const void* light_kernel(int threads);
const void* heavy_kernel(int threads);
const void* rounds_kernel(int threads);
__global__ void k_init_workspace(uint4*, size_t, uint4*, uint4*, uint32_t, uint4*, size_t);
}  // namespace gstb

using namespace gstb;

#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) {                              \
      last_cuda_error() = e_;                             \
      return GST_CUDA_ERROR;                              \
    }                                                     \
  } while (0)

// Last CUDA error met by any thread of the library (the serving loop runs on
// its own thread), reported by gst_last_cuda_error.
static std::atomic<cudaError_t>& last_cuda_error() {
  static std::atomic<cudaError_t> e{cudaSuccess};
  return e;
}

struct gst_graph {
  uint32_t V = 0;
  uint64_t arcs = 0;
  uint32_t* d_beg = nullptr;
  uint2* d_adj = nullptr;
  uint32_t* d_wcut = nullptr;  // per vertex: first arc with weight > 2^b, b = 0..7
  // group index (host copy; member lists of a query are built on the host).
  // gst_groups_set replaces it under grp_mu held exclusively; every reader
  // (query preparation in all entry points) holds it shared
  std::vector<uint64_t> grp_ptr;
  std::vector<uint32_t> grp_v;
  std::shared_mutex grp_mu;
  int device = 0;
  int num_sms = 148;
  size_t total_mem = 0;  // the device's memory (bytes)
  // launch parameters (defaults and GSTB_* overrides at creation, gst_tuning_set
  // or gst_autotune later); every Runner of the graph reads them
  gst_tuning tune{};
  // persistent round driver for gst_query / gst_query_batch (created lazily)
  void* runner = nullptr;
  std::mutex mu;
  std::atomic<uint64_t> launches{0};
  // fault injection (gst_debug_fail_allocs): workspace allocations still to fail
  std::atomic<int> fail_allocs{0};
  // test hook of the persistent launch (gst_debug_hold_rounds)
  std::atomic<uint32_t> hold_rounds{0}, wait_ms{0};
  bool profile = false;
  bool prof_persistent = false;  // the profiled rounds ran as persistent launches
  double prof_light_ms = 0, prof_heavy_ms = 0;
  uint64_t prof_rounds = 0;
  uint64_t prof_stats[GST_NSTATS] = {0};
};

namespace {

bool has_groups(gst_graph* g) {
  std::shared_lock<std::shared_mutex> lock(g->grp_mu);
  return !g->grp_ptr.empty();
}

uint32_t floor_pow2(uint32_t x) { return x ? 1u << (31 - __builtin_clz(x)) : 0u; }

uint32_t env_u32(const char* name, uint32_t def) {
  const char* s = getenv(name);
  if (!s || !*s) return def;
  return (uint32_t)strtoul(s, nullptr, 10);
}

struct Job {
  // request
  uint32_t groups[KMAX];
  int k = 0, D = -1;
  uint64_t tag = 0;
  uint32_t ratio_num = 0;     // progressive mode: ratio * 1024 (0: exact)
  gst_result* res = nullptr;  // caller result (may be null: serve copies out)
  // derived
  int nd = 1;
  uint32_t WT = 0, full = 0;
  size_t table_bytes = 0, bytes = 0;
  std::vector<uint32_t> members;
  // device workspace
  char* mem = nullptr;
  QDev qd{};
  QCtl ctl{};
  int slot = -1;
  int64_t first_block = 0;  // first round block that runs this job
  uint64_t cap_req = 0;      // frontier capacity after an overflow retry (0 = default)
  uint32_t retries = 0;      // runs repeated after GST_QUEUE_OVERFLOW
  gst_status status = GST_OK;
  bool rejected = false;  // failed validation before admission
  bool cancelled = false; // withdrawn while waiting for a rerun
  bool done = false;
  bool early_done = false;   // fill_result has settled the progressive answer
  uint32_t lower_bound = 0;  // proven lower bound on the optimum
  // results
  int32_t cost = -1;
  uint32_t root = 0;
  std::vector<uint32_t> edges;
  std::chrono::steady_clock::time_point t_submit, t_admit, t_done;
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Progressive-mode ratios are rationals num / RATIO_DEN.
constexpr uint32_t RATIO_DEN = 1024;
uint32_t ratio_to_num(double ratio) {
  if (!(ratio > 1.0)) return 0;  // exact (also NaN)
  return (uint32_t)std::floor(std::min(ratio, 1.0e6) * RATIO_DEN);  // rounded down: never looser than asked
}

// Minimum spanning forest (Kruskal) of an edge multiset given as (u, v, w)
// triples; duplicates collapse.  A progressive answer's derivation may reuse
// edges across subtrees or close cycles (its sub-states can have been lowered
// after it was recorded); its edges stay connected, so the spanning tree
// covers the same vertices, hence the same groups, at no greater cost (the
// reference post-processes its incumbent the same way,
// graph_hash_of_mixed_weighted_MST_postprocessing_no_whole_graph).
void spanning_tree(std::vector<uint32_t>& e) {
  const size_t n = e.size() / 3;
  std::vector<size_t> ord(n);
  for (size_t i = 0; i < n; i++) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return e[3 * a + 2] < e[3 * b + 2]; });
  std::unordered_map<uint32_t, uint32_t> id;
  std::vector<uint32_t> par;
  auto node = [&](uint32_t v) {
    auto it = id.find(v);
    if (it != id.end()) return it->second;
    uint32_t x = (uint32_t)par.size();
    id[v] = x;
    par.push_back(x);
    return x;
  };
  std::function<uint32_t(uint32_t)> find = [&](uint32_t x) { return par[x] == x ? x : par[x] = find(par[x]); };
  std::vector<uint32_t> out;
  for (size_t i : ord) {
    uint32_t a = find(node(e[3 * i])), b = find(node(e[3 * i + 1]));
    if (a == b) continue;
    par[a] = b;
    out.insert(out.end(), {e[3 * i], e[3 * i + 1], e[3 * i + 2]});
  }
  e.swap(out);
}

// Device workspace arena of one Runner: chunks from cudaMalloc, carved by
// best fit with coalescing.  Admission never waits on the driver's allocator
// (a stream-ordered pool that had to grow stalled the serving loop for up to
// half a second).  A block is reusable as soon as it is freed: every kernel,
// copy and memset that touches a workspace runs on the Runner's one stream, so
// work enqueued for the next owner is ordered after the last use.
class Arena {
 public:
  ~Arena() { release(); }

  // Counter of injected failures (gst_debug_fail_allocs): while it is
  // positive, each workspace allocation fails as if the device were full.
  void set_fail_counter(std::atomic<int>* c) { fail_ = c; }

  void* alloc(size_t n) {
    if (fail_) {
      int f = fail_->load();
      while (f > 0 && !fail_->compare_exchange_weak(f, f - 1)) {
      }
      if (f > 0) return nullptr;
    }
    n = align_up(std::max<size_t>(n, 1), 256);
    auto it = by_size_.lower_bound(n);
    if (it == by_size_.end()) {
      // A growth of this size already failed and no memory went back to the
      // device since (a workspace freed inside the arena gives it none):
      // while this arena's queries run, waiting for their blocks to coalesce
      // is cheaper than another failing cudaMalloc on every admission
      // attempt, which held the host for up to 130 ms each time while the GPU
      // ran out of launched rounds.  With nothing in use, growth is retried
      // (with a trim), so a request never waits on itself.
      if (n >= grow_failed_ && in_use_ != 0) return nullptr;
      if (!grow(n)) {
        grow_failed_ = n;
        return nullptr;
      }
      it = by_size_.lower_bound(n);
      if (it == by_size_.end()) return nullptr;
    }
    char* p = it->second;
    const size_t sz = it->first;
    by_size_.erase(it);
    free_.erase(p);
    free_total_ -= sz;
    if (sz > n) insert_free(p + n, sz - n);
    used_[p] = n;
    in_use_ += n;
    return p;
  }

  void free(void* vp) {
    char* p = static_cast<char*>(vp);
    auto u = used_.find(p);
    if (u == used_.end()) return;
    size_t n = u->second;
    used_.erase(u);
    in_use_ -= n;
    const char* base = chunk_base(p);
    // merge with the free neighbours inside the same chunk
    auto nx = free_.find(p + n);
    if (nx != free_.end() && chunk_base(nx->first) == base) {
      n += nx->second;
      erase_free(nx->first, nx->second);
    }
    auto pv = free_.lower_bound(p);
    if (pv != free_.begin()) {
      --pv;
      if (pv->first + pv->second == p && chunk_base(pv->first) == base) {
        char* q = pv->first;
        n += pv->second;
        erase_free(q, pv->second);
        p = q;
      }
    }
    insert_free(p, n);
  }

  // Make at least n bytes free with one allocation instead of several growth
  // steps later (called before a batch or when a serving loop opens).
  bool reserve(size_t n) {
    if (free_total_ >= n) return true;
    return grow(align_up(n - free_total_, 256), true);
  }

  size_t free_bytes() const { return free_total_; }
  // Give back every wholly free chunk when more than `keep` bytes are held
  // (after a batch, so that its memory does not starve other engines).
  void release_above(size_t keep) {
    if (held_ > keep) trim();
  }

  void release() {
    for (auto& c : chunks_) cudaFree(c.first);
    chunks_.clear();
    free_.clear();
    by_size_.clear();
    used_.clear();
    held_ = in_use_ = free_total_ = 0;
  }


 private:
  // Give chunks that are entirely free back to the driver (a request larger
  // than every free block can then get one allocation of its own).
  void trim() {
    grow_failed_ = SIZE_MAX;  // the device gets memory back
    for (auto it = chunks_.begin(); it != chunks_.end();) {
      auto f = free_.find(it->first);
      if (f != free_.end() && f->second == it->second) {
        erase_free(f->first, f->second);
        cudaFree(it->first);
        held_ -= it->second;
        it = chunks_.erase(it);
      } else {
        ++it;
      }
    }
  }

  bool grow(size_t n, bool exact = false) {
    // chunks double from 64 MB up to GSTB_ARENA_MB (default 1 GB)
    const size_t step = (size_t)env_u32("GSTB_ARENA_MB", 1024) << 20;
    void* p = nullptr;
    size_t sz = exact ? n : std::max(n, std::min(step, std::max<size_t>(held_, 64ull << 20)));
    if (cudaMalloc(&p, sz) != cudaSuccess) {
      cudaGetLastError();
      sz = n;
      if (cudaMalloc(&p, sz) != cudaSuccess) {
        cudaGetLastError();
        // free chunks may be what the device is missing; give them back only
        // when no workspace is in use (cudaFree synchronises the device)
        if (in_use_ != 0) return false;
        trim();
        if (cudaMalloc(&p, sz) != cudaSuccess) {
          cudaGetLastError();
          return false;
        }
      }
    }
    chunks_[static_cast<char*>(p)] = sz;
    held_ += sz;
    insert_free(static_cast<char*>(p), sz);
    return true;
  }

  const char* chunk_base(const char* p) const {
    auto it = chunks_.upper_bound(const_cast<char*>(p));
    return it == chunks_.begin() ? nullptr : std::prev(it)->first;
  }

  void insert_free(char* p, size_t n) {
    free_[p] = n;
    by_size_.emplace(n, p);
    free_total_ += n;
  }

  void erase_free(char* p, size_t n) {
    free_.erase(p);
    free_total_ -= n;
    auto r = by_size_.equal_range(n);
    for (auto it = r.first; it != r.second; ++it)
      if (it->second == p) {
        by_size_.erase(it);
        break;
      }
  }

  std::map<char*, size_t> chunks_;        // base -> size
  std::map<char*, size_t> free_;          // free block -> size
  std::multimap<size_t, char*> by_size_;  // size -> free block
  std::unordered_map<char*, size_t> used_;
  size_t held_ = 0, in_use_ = 0, free_total_ = 0;
  size_t grow_failed_ = SIZE_MAX;  // smallest growth that failed since memory last went back to the device
  std::atomic<int>* fail_ = nullptr;
};

// Workspace layout of one query (see gst_device.cuh).
struct Layout {
  size_t table, dist, dist2, dflag, qbuf, tour, lbt, snap, members, edges, total;
  uint32_t cap;
};

// cap_req > 0 asks for a frontier-list capacity of that many items (a query
// retried after GST_QUEUE_OVERFLOW); 0 takes the default.
Layout layout_for(const gst_graph* g, int k, int D, size_t n_members, uint32_t max_edges, uint64_t cap_req = 0) {
  const int nd = D < 0 ? 1 : D + 1;
  Layout L{};
  uint64_t WT = (uint64_t)(1u << k) * nd;
  uint64_t states = (uint64_t)g->V * WT;
  uint64_t caplim = env_u32("GSTB_QUEUE_CAP", 1u << 25);
  // distance lists hold each vertex at most once per list (cap >= V never
  // overflows there); DP lists start at a quarter of the states and grow by
  // rerunning the query if a frontier outgrows them
  uint64_t cap = std::min<uint64_t>(std::max<uint64_t>(states / 4, (uint64_t)g->V + 1024), caplim);
  if (cap_req) cap = cap_req;
  cap = std::max<uint64_t>(cap, 1024);
  L.cap = (uint32_t)cap;
  size_t o = 0;
  L.table = o; o = align_up(o + states * 8, 256);
  L.dist = o; o = align_up(o + (size_t)g->V * 8 * 4, 256);
  // hop-bounded queries: the second row buffer of the exact distance rounds
  L.dist2 = o; o = align_up(o + (D >= 0 ? (size_t)g->V * 8 * 4 : 0), 256);
  L.dflag = o; o = align_up(o + ((states + 7) / 8) * 4, 256);
  L.qbuf = o; o = align_up(o + 4 * cap * 4, 256);
  L.tour = o; o = align_up(o + ((size_t)k * (1u << k) * k + (size_t)k * (1u << k) + 64) * 4, 256);
  L.lbt = o; o = align_up(o + (size_t)g->V * (1u << k) * 2, 256);
  // hop-bounded queries: distance rows after Bellman-Ford rounds 1..D-1
  L.snap = o; o = align_up(o + (nd >= 3 ? (size_t)(nd - 2) * g->V * ROW * 4 : 0), 256);
  L.members = o; o = align_up(o + std::max<size_t>(n_members, 1) * 4, 256);
  L.edges = o; o = align_up(o + (size_t)std::max<uint32_t>(max_edges, 1) * 12, 256);
  L.total = o;
  return L;
}

// ---------------------------------------------------------------------------
// Round driver.  Queries occupy slots of device-resident descriptors; every
// round is k_control -> k_light -> k_heavy, all reading their work from device
// memory, so the host launches several rounds back to back and synchronises
// only to admit new queries and retire finished ones.
// ---------------------------------------------------------------------------
class Runner {
 public:
  explicit Runner(gst_graph* g) : g_(g) {}
  ~Runner() { release(); }

  gst_status init() {
    arena_.set_fail_counter(&g_->fail_allocs);
    CK(cudaSetDevice(g_->device));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (auto& e : ev_) CK(cudaEventCreate(&e));
    for (auto& e : ev_blk_) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_fin_, cudaEventDisableTiming));
    for (auto& hh : ev_prof_)
      for (auto& e : hh) CK(cudaEventCreate(&e));
    delta_sssp_ = g_->tune.delta_sssp;
    delta_dp_ = g_->tune.delta_dp;
    cap_num_ = g_->tune.cap_pct;
    cap_den_ = 100;
    max_edges_dev_ = env_u32("GSTB_MAX_TREE_EDGES", 1u << 16);
    rounds_per_sync_ = g_->tune.rounds_per_launch;
    trace_ms_ = (double)env_u32("GSTB_TRACE_MS", 0);  // report host iterations slower than this
    wait_ms_default_ = std::max(1u, env_u32("GSTB_WAIT_MS", 30000));  // limit of a persistent launch's waits
    max_slots_ = std::min<uint32_t>(MAX_SLOTS - 1, std::max(1u, env_u32("GSTB_MAX_SLOTS", MAX_SLOTS - 1)));
    CK(cudaMalloc(&d_qd_, MAX_SLOTS * sizeof(QDev)));
    CK(cudaMalloc(&d_ctl_, MAX_SLOTS * sizeof(QCtl)));
    CK(cudaMalloc(&d_rd_, sizeof(RoundDesc)));
    {
      gst_status gs = setup_grids();
      if (gs != GST_OK) return gs;
    }
    {
      // hub arc chunk list (k_light -> k_heavy within a round)
      big_cap_ = std::max(1u << 12, env_u32("GSTB_HUB_CHUNKS", 1u << 22));
      CK(cudaMalloc(&d_big_, (size_t)big_cap_ * sizeof(uint4)));
      RoundDesc rd;
      memset(&rd, 0, sizeof(rd));
      rd.big = env_u32("GSTB_HUB_SPLIT", 1) ? d_big_ : nullptr;
      rd.big_cap = big_cap_;
      rd.hub_min_deg = g_->tune.hub_min_deg;
      rd.hub_min_rest = env_u32("GSTB_HUB_MIN_REST", 128);
      rd.hub_max_items = env_u32("GSTB_HUB_MAX_ITEMS", 1000000);
      rd.hub_max_items2 = env_u32("GSTB_HUB_MAX_ITEMS2", 8000000);
      rd.hub_big_deg = std::max(32u, env_u32("GSTB_HUB_BIG_DEG", 1024));
      rd.hub_share_div = env_u32("GSTB_HUB_SHARE_DIV", 16);
      rd.avg_deg = (uint32_t)std::max<uint64_t>(1, (g_->arcs + g_->V - 1) / std::max<uint32_t>(1, g_->V));
      // task widths are sized for the warps resident at once
      rd.light_warps = light_warps();
      rd.sssp_w = 4;
      rd.dp_wmax = g_->tune.dp_wmax;
      rd.sssp_wmax = g_->tune.sssp_wmax;
      rd.merge_stage = g_->tune.merge_stage;
      CK(cudaMemcpy(d_rd_, &rd, sizeof(rd), cudaMemcpyHostToDevice));
    }
    CK(cudaMalloc(&d_pre_, (size_t)NT * (MAX_SLOTS + 1) * 4));
    CK(cudaMemset(d_qd_, 0, MAX_SLOTS * sizeof(QDev)));
    CK(cudaMemset(d_ctl_, 0, MAX_SLOTS * sizeof(QCtl)));
    CK(cudaMallocHost(&h_ctl_, 2 * MAX_SLOTS * sizeof(QCtl)));
    CK(cudaMallocHost(&h_rd_, sizeof(RoundDesc)));
    CK(cudaMallocHost(&h_qd_, sizeof(QDev)));
    CK(cudaMallocHost(&h_one_, sizeof(uint32_t)));
    CK(cudaMalloc(&d_pc_, sizeof(PersistCtl)));
    CK(cudaMallocHost(&h_pc_, 4 * sizeof(PersistCtl)));  // launch templates, then read-backs, per block half
    memset(h_pc_, 0, 4 * sizeof(PersistCtl));
    if (env_u32("GSTB_TRACE_ROUNDS", 0)) CK(cudaMallocHost(&h_rdtrace_, 2 * 64 * sizeof(RoundDesc)));
    *h_one_ = 1u;
    // pinned staging for admissions (descriptors + member lists) and for the
    // tree read-back of retired jobs: copies from pinned memory stay
    // asynchronous, pageable ones would synchronise the stream each time
    stage_cap_ = (size_t)env_u32("GSTB_STAGE_MB", 32) << 20;
    CK(cudaMallocHost(&h_stage_, stage_cap_));
    edge_stage_cap_ = (size_t)env_u32("GSTB_EDGE_STAGE_MB", 16) << 20;
    CK(cudaMallocHost(&h_edge_stage_, edge_stage_cap_));
    memset(h_qd_, 0, sizeof(QDev));  // the zero descriptor that frees a slot
    slots_.assign(max_slots_, nullptr);
    if (env_u32("GSTB_ROUND_GRAPH", 1)) {
      gst_status gs = build_round_graph();
      if (gs != GST_OK) return gs;
    }
    return GST_OK;
  }

  // Grids of the round kernels for the graph's block size: every SM filled
  // to the occupancy limit of each kernel.
  gst_status setup_grids() {
    const int T = (int)g_->tune.block_threads;
    kl_ = light_kernel(T);
    kh_ = heavy_kernel(T);
    kr_ = rounds_kernel(T);
    if (!kl_ || !kh_ || !kr_) return GST_BAD_INPUT;
    threads_ = (uint32_t)T;
    int bl = 0, bh = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bl, kl_, T, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bh, kh_, T, 0));
    light_grid_ = (unsigned)g_->num_sms * (unsigned)std::max(1, bl);
    heavy_grid_ = (unsigned)g_->num_sms * (unsigned)std::max(1, bh);
    resident_light_warps_ = light_grid_ * ((unsigned)T / 32);
    // GSTB_GRID_WAVES > 1 launches that many resident waves of blocks: a
    // block that runs out of tasks early exits and a waiting block takes
    // its place on the SM
    const unsigned waves = std::min(8u, std::max(1u, env_u32("GSTB_GRID_WAVES", 1)));
    light_grid_ *= waves;
    heavy_grid_ *= waves;
    // the persistent round launch: one resident wave, every block at once
    int br = 0, coop = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&br, kr_, T, 0));
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, g_->device));
    rounds_grid_ = coop ? (unsigned)g_->num_sms * (unsigned)std::max(0, br) : 0u;
    persist_ = rounds_grid_ > 0 && g_->tune.persistent;
    return GST_OK;
  }

  // Warps of one round launch: the task widths are sized for them.
  uint32_t light_warps() const { return persist_ ? rounds_grid_ * (threads_ / 32) : resident_light_warps_; }

  // k_light / k_heavy of the graph's block size on the runner's stream.
  cudaError_t launch_light(const GraphDev& gd, int ns) {
    GraphDev g = gd;
    void* args[] = {&d_qd_, &d_rd_, &d_pre_, &ns, &g};
    return cudaLaunchKernel(kl_, dim3(light_grid_), dim3(threads_), args, 0, stream_);
  }
  cudaError_t launch_heavy(const GraphDev& gd, int ns) {
    GraphDev g = gd;
    void* args[] = {&d_qd_, &d_rd_, &d_pre_, &ns, &g};
    return cudaLaunchKernel(kh_, dim3(heavy_grid_), dim3(threads_), args, 0, stream_);
  }

  void release() {
    for (Job* j : slots_)
      if (j) free_job(j);
    slots_.clear();
    if (d_qd_) cudaFree(d_qd_);
    if (d_ctl_) cudaFree(d_ctl_);
    if (d_rd_) cudaFree(d_rd_);
    if (d_big_) cudaFree(d_big_);
    d_big_ = nullptr;
    if (d_pre_) cudaFree(d_pre_);
    if (h_ctl_) cudaFreeHost(h_ctl_);
    if (h_rd_) cudaFreeHost(h_rd_);
    if (h_qd_) cudaFreeHost(h_qd_);
    if (h_one_) cudaFreeHost(h_one_);
    if (h_pc_) cudaFreeHost(h_pc_);
    h_pc_ = nullptr;
    if (d_pc_) cudaFree(d_pc_);
    d_pc_ = nullptr;
    if (h_rdtrace_) cudaFreeHost(h_rdtrace_);
    h_rdtrace_ = nullptr;
    h_one_ = nullptr;
    if (h_stage_) cudaFreeHost(h_stage_);
    if (h_edge_stage_) cudaFreeHost(h_edge_stage_);
    h_stage_ = nullptr;
    h_edge_stage_ = nullptr;
    for (auto& e : ev_)
      if (e) cudaEventDestroy(e);
    for (auto& e : ev_blk_)
      if (e) cudaEventDestroy(e);
    if (ev_fin_) cudaEventDestroy(ev_fin_);
    for (auto& hh : ev_prof_)
      for (auto& e : hh)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamSynchronize(stream_);
    if (round_graph_) cudaGraphExecDestroy(round_graph_);
    round_graph_ = nullptr;
    arena_.release();
    if (stream_) cudaStreamDestroy(stream_);
    d_qd_ = nullptr;
    d_ctl_ = nullptr;
    d_rd_ = nullptr;
    d_pre_ = nullptr;
    h_ctl_ = nullptr;
    h_rd_ = nullptr;
    h_qd_ = nullptr;
    stream_ = nullptr;
  }

  // Prepare a job (validation, member list, sizes).  Does not allocate.
  gst_status prepare(Job* j) {
    if (j->k < 1 || j->k > KMAX) return GST_BAD_INPUT;
    if (j->D > DMAX) return GST_BAD_INPUT;
    std::shared_lock<std::shared_mutex> glock(g_->grp_mu);
    if (g_->grp_ptr.empty()) return GST_BAD_INPUT;
    const uint32_t ng = (uint32_t)(g_->grp_ptr.size() - 1);
    for (int i = 0; i < j->k; i++)
      if (j->groups[i] >= ng) return GST_BAD_INPUT;
    for (int a = 0; a < j->k; a++)
      for (int b = a + 1; b < j->k; b++)
        if (j->groups[a] == j->groups[b]) return GST_BAD_INPUT;
    j->nd = j->D < 0 ? 1 : j->D + 1;
    j->WT = (1u << j->k) * (uint32_t)j->nd;
    j->full = (1u << j->k) - 1u;
    if ((uint64_t)g_->V * j->WT >= (1ull << 32) || g_->V >= (1u << 29)) return GST_BAD_INPUT;
    j->members.clear();
    for (int i = 0; i < j->k; i++) {
      uint32_t gi = j->groups[i];
      if (g_->grp_ptr[gi + 1] == g_->grp_ptr[gi]) return GST_NO_SOLUTION;  // empty group
      for (uint64_t t = g_->grp_ptr[gi]; t < g_->grp_ptr[gi + 1]; t++)
        j->members.push_back(g_->grp_v[t] * 8u + (uint32_t)i);
    }
    Layout L = layout_for(g_, j->k, j->D, j->members.size(), max_edges_dev_, j->cap_req);
    j->table_bytes = (size_t)g_->V * j->WT * 8;
    j->bytes = L.total;
    return GST_OK;
  }

  bool has_free_slot() const { return n_used_ < max_slots_; }
  bool reserve(size_t bytes) { return arena_.reserve(bytes); }
  bool has_free(size_t bytes) const { return arena_.free_bytes() >= bytes; }
  void release_arena_above(size_t keep) { arena_.release_above(keep); }

  // Take the graph's launch parameters (between calls: nothing in flight).
  gst_status apply_tuning() {
    delta_sssp_ = g_->tune.delta_sssp;
    delta_dp_ = g_->tune.delta_dp;
    cap_num_ = g_->tune.cap_pct;
    cap_den_ = 100;
    const uint32_t hub = g_->tune.hub_min_deg, dpw = g_->tune.dp_wmax, ssw = g_->tune.sssp_wmax;
    const uint32_t mst = g_->tune.merge_stage;
    const bool regrid = g_->tune.block_threads != threads_;
    if (regrid) {
      gst_status gs = setup_grids();
      if (gs != GST_OK) return gs;
    }
    persist_ = rounds_grid_ > 0 && g_->tune.persistent;
    const uint32_t lw = light_warps();
    CK(cudaMemcpyAsync(&d_rd_->hub_min_deg, &hub, sizeof(hub), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(&d_rd_->dp_wmax, &dpw, sizeof(dpw), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(&d_rd_->sssp_wmax, &ssw, sizeof(ssw), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(&d_rd_->merge_stage, &mst, sizeof(mst), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(&d_rd_->light_warps, &lw, sizeof(lw), cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    if (g_->tune.rounds_per_launch != rounds_per_sync_ || regrid) {
      rounds_per_sync_ = g_->tune.rounds_per_launch;
      if (round_graph_) {
        cudaGraphExecDestroy(round_graph_);
        round_graph_ = nullptr;
        gst_status gs = build_round_graph();
        if (gs != GST_OK) return gs;
      }
    }
    return GST_OK;
  }
  size_t live() const { return n_used_; }

  // Allocate the workspace, initialise it and install the job in a free
  // slot; false if no slot or no device memory is available.
  bool admit(Job* j) {
    if (n_used_ >= max_slots_) return false;
    const size_t need = align_up(sizeof(QDev), 64) + align_up(sizeof(QCtl), 64) + align_up(j->members.size() * 4, 64);
    const int sh = (int)(next_block_ & 1);  // staging half of the block this job starts in
    if (stage_off_[sh] + need > stage_cap_ / 2) return false;  // staging full until that block has run
    void* p = arena_.alloc(j->bytes);
    if (p == nullptr) return false;
    int slot = -1;
    for (uint32_t s = 0; s < max_slots_; s++)
      if (!slots_[s]) {
        slot = (int)s;
        break;
      }
    j->mem = (char*)p;
    j->slot = slot;
    Layout L = layout_for(g_, j->k, j->D, j->members.size(), max_edges_dev_, j->cap_req);
    QDev& q = j->qd;
    memset(&q, 0, sizeof(q));
    q.table = (unsigned long long*)(j->mem + L.table);
    q.dist = (uint32_t*)(j->mem + L.dist);
    q.dist_nx = j->D >= 0 ? (uint32_t*)(j->mem + L.dist2) : q.dist;
    q.dflag = (uint32_t*)(j->mem + L.dflag);
    for (int b = 0; b < 4; b++) q.qbuf[b] = (uint32_t*)(j->mem + L.qbuf) + (size_t)b * L.cap;
    q.tour = (uint32_t*)(j->mem + L.tour);
    q.lbt = (unsigned short*)(j->mem + L.lbt);
    q.snap = (uint32_t*)(j->mem + L.snap);
    q.nv = g_->V;
    q.members = (const uint32_t*)(j->mem + L.members);
    q.out_edges = (uint32_t*)(j->mem + L.edges);
    q.ctl = d_ctl_ + slot;
    q.cap = L.cap;
    q.n_members = (uint32_t)j->members.size();
    q.max_edges = max_edges_dev_;
    q.k = j->k;
    q.D = j->D;
    q.nd = j->nd;
    q.full = (int)j->full;
    q.WT = j->WT;
    q.phase = PH_SSSP;
    // hop-bounded queries read an unreached distance as "no path within the
    // hops left": their distance rounds may only skip what exceeds the
    // incumbent itself (capping them at cap_pct% of it, with unknown entries
    // read as "above the cap", admitted 6.6x more DP states on the 3M-vertex
    // mix through the weaker hop-budget bound)
    q.cap_num = j->D >= 0 ? 1u : cap_num_;
    q.cap_den = j->D >= 0 ? 1u : cap_den_;
    q.star_h = j->D >= 2 ? (uint32_t)j->D / 2u : 0u;
    q.center_h = j->D >= 2 ? ((uint32_t)j->D + 1u) / 2u : 0u;
    q.in_idx = 0;
    q.out_idx = 1;
    q.far_idx = 2;
    q.far2_idx = 3;
    q.st = J_INIT;
    q.act = A_NONE;
    q.delta_sssp = delta_sssp_;
    q.delta_dp = delta_dp_;
    q.ratio_num = j->D < 0 ? j->ratio_num : 0u;
    q.ratio_den = RATIO_DEN;
    memset(&j->ctl, 0, sizeof(j->ctl));
    j->ctl.best = INF32;
    j->ctl.best_full = INF64;
    // state table INF, distances unknown with no group pending, no state
    // flag set: one launch (the byte counts are multiples of 16: the table
    // holds an even number of 8-byte words, the flags span is 256-aligned)
    k_init_workspace<<<(unsigned)g_->num_sms * 8u, 256, 0, stream_>>>(
        reinterpret_cast<uint4*>(q.table), (size_t)g_->V * j->WT * 8 / 16, reinterpret_cast<uint4*>(q.dist),
        q.dist_nx != q.dist ? reinterpret_cast<uint4*>(q.dist_nx) : nullptr, g_->V,
        reinterpret_cast<uint4*>(q.dflag), (L.qbuf - L.dflag) / 16);
    g_->launches++;
    // stage the member list and both descriptors in pinned memory; it is not
    // reused before the stream synchronises at the end of the next round block
    char* st = h_stage_ + (size_t)sh * (stage_cap_ / 2) + stage_off_[sh];
    memcpy(st, &q, sizeof(QDev));
    char* stc = st + align_up(sizeof(QDev), 64);
    memcpy(stc, &j->ctl, sizeof(QCtl));
    char* stm = stc + align_up(sizeof(QCtl), 64);
    memcpy(stm, j->members.data(), j->members.size() * 4);
    stage_off_[sh] += need;
    j->first_block = next_block_;
    cudaMemcpyAsync((void*)q.members, stm, j->members.size() * 4, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(d_qd_ + slot, st, sizeof(QDev), cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(d_ctl_ + slot, stc, sizeof(QCtl), cudaMemcpyHostToDevice, stream_);
    slots_[slot] = j;
    n_used_++;
    nslots_hi_ = std::max<uint32_t>(nslots_hi_, (uint32_t)slot + 1);
    j->t_admit = std::chrono::steady_clock::now();
    return true;
  }

  void free_job(Job* j) {
    if (j->mem) arena_.free(j->mem);
    j->mem = nullptr;
  }

  // Withdraw the admitted job with this tag: its control block's cancel flag
  // is set stream-ordered after the block in flight, and k_control ends the
  // job at its next round with GST_CANCELLED.  False if no admitted job has
  // the tag (the caller checks its pending queue).
  bool cancel_tag(uint64_t tag) {
    for (Job* j : retry_)
      if (j->tag == tag) {
        j->cancelled = true;  // reported as cancelled instead of being rerun
        return true;
      }
    for (uint32_t s = 0; s < slots_.size(); s++) {
      Job* j = slots_[s];
      if (j && j->tag == tag) {
        if (cudaMemcpyAsync(&d_ctl_[s].cancel, h_one_, sizeof(uint32_t), cudaMemcpyHostToDevice, stream_) !=
            cudaSuccess) {
          last_cuda_error() = cudaGetLastError();
          return false;
        }
        return true;
      }
    }
    return false;
  }

  double last_call_ms() const { return last_call_ms_; }
  double trace_ms() const { return trace_ms_; }

  // Run rounds until no admitted job is left and admit_more() adds none.
  // `on_done` is called for every finished job (after its results are copied).
  //
  // Round blocks are pipelined: block b+1 is launched before the host looks
  // at block b's control blocks, so the GPU keeps working while the host
  // retires finished queries and stages new ones.  Everything the host
  // enqueues (admissions, tree copies, slot clears, frees) is stream-ordered
  // after the block in flight; staging buffers alternate between two halves.
  template <class AdmitFn, class DoneFn>
  gst_status run(AdmitFn&& admit_more, DoneFn&& on_done) {
    CK(cudaEventRecord(ev_[0], stream_));
    int64_t inflight = -1;  // id of the block launched but not yet examined
    std::vector<Job*> fin;  // retired jobs whose tree copies are in flight
    std::vector<size_t> fin_off;
    int fin_half = 0;
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
    double sum_admit = 0, sum_launch = 0, sum_fin = 0, sum_blk = 0, sum_all = 0;
    int iters = 0;
    for (;;) {
      const clk::time_point t_it = clk::now();
      double t_admit = 0, t_launch = 0, t_fin = 0, t_blk = 0;
      // queries retried with larger frontier lists go first
      while (!retry_.empty() && has_free_slot()) {
        Job* j = retry_.front();
        if (j->cancelled) {
          j->status = GST_CANCELLED;
          j->done = true;
          j->t_done = std::chrono::steady_clock::now();
          retry_.pop_front();
          on_done(j);
          continue;
        }
        if (!admit(j)) {
          if (n_used_ > 0) break;  // wait for memory
          j->status = GST_OOM;     // does not fit even alone
          j->done = true;
          j->t_done = std::chrono::steady_clock::now();
          retry_.pop_front();
          on_done(j);
          continue;
        }
        retry_.pop_front();
      }
      admit_more();
      if (trace_ms_ > 0) t_admit = ms_since(t_it);
      int64_t launched = -1;
      if (n_used_ > 0) {
        gst_status st = launch_block(rounds_per_sync_);
        if (st != GST_OK) return st;
        launched = next_block_++;
      }
      if (trace_ms_ > 0) t_launch = ms_since(t_it);
      if (!fin.empty()) {
        CK(cudaEventSynchronize(ev_fin_));
        finalize(fin, fin_off, fin_half, on_done);
      }
      if (trace_ms_ > 0) t_fin = ms_since(t_it);
      if (inflight >= 0) {
        const int h = (int)(inflight & 1);
        CK(cudaEventSynchronize(ev_blk_[h]));
        if (trace_ms_ > 0) t_blk = ms_since(t_it);
        stage_off_[h] = 0;  // admissions staged for this block have been copied
        if (g_->profile) accumulate_profile(h);
        gst_status st = detect_done(inflight, fin, fin_off);
        if (st != GST_OK) return st;
        fin_half = h;
        if (!fin.empty()) CK(cudaEventRecord(ev_fin_, stream_));
      }
      if (trace_ms_ > 0) {
        const double t_all = ms_since(t_it);
        sum_admit += t_admit;
        sum_launch += t_launch - t_admit;
        sum_fin += t_fin - t_launch;
        sum_blk += t_blk > 0 ? t_blk - t_fin : 0.0;
        sum_all += t_all;
        iters++;
        if (t_all >= trace_ms_)
          fprintf(stderr,
                  "gstb: slow host iteration %.2f ms (admit %.2f, launch %.2f, finalize %.2f, block wait %.2f; "
                  "%u queries in slots)\n",
                  t_all, t_admit, t_launch - t_admit, t_fin - t_launch, t_blk > 0 ? t_blk - t_fin : 0.0, n_used_);
      }
      inflight = launched;
      if (inflight < 0 && n_used_ == 0 && fin.empty() && retry_.empty()) break;
    }
    CK(cudaEventRecord(ev_[1], stream_));
    CK(cudaEventSynchronize(ev_[1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    last_call_ms_ = ms;
    if (trace_ms_ > 0 && sum_all >= trace_ms_)
      fprintf(stderr,
              "gstb: run of %d host iterations: %.2f ms (admit %.2f, launch %.2f, finalize %.2f, block wait %.2f, "
              "rest %.2f)\n",
              iters, sum_all, sum_admit, sum_launch, sum_fin, sum_blk,
              sum_all - sum_admit - sum_launch - sum_fin - sum_blk);
    return GST_OK;
  }

 private:
  // A block of rounds_per_sync_ rounds as one CUDA graph.  Its arguments are
  // static: k_control scans every slot and publishes the bound the round
  // kernels search, so the graph serves any set of admitted queries.
  gst_status build_round_graph() {
    GraphDev gd{g_->d_beg, g_->d_adj, g_->V, g_->d_wcut};
    cudaGraph_t gr = nullptr;
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaSuccess;
    for (uint32_t r = 0; r < rounds_per_sync_; r++) {
      k_control<<<1, 1024, 0, stream_>>>(d_qd_, d_ctl_, (int)max_slots_, d_rd_, d_pre_);
      if (le == cudaSuccess) le = launch_light(gd, MAX_SLOTS);
      if (le == cudaSuccess) le = launch_heavy(gd, MAX_SLOTS);
    }
    if (le == cudaSuccess) le = cudaGetLastError();
    const cudaError_t ce = cudaStreamEndCapture(stream_, &gr);  // always leave capture mode
    CK(le);
    CK(ce);
    const cudaError_t ie = cudaGraphInstantiate(&round_graph_, gr, 0);
    cudaGraphDestroy(gr);
    CK(ie);
    return GST_OK;
  }

  gst_status launch_block(uint32_t R) {
    const int h = (int)(next_block_ & 1);
    const bool prof = g_->profile;
    blk_persist_[h] = persist_ && !(prof && h_rdtrace_);  // the per-round trace needs separate launches
    if (blk_persist_[h]) {
      // the block's rounds as one persistent launch; its state is reset from
      // this half's pinned template (rewritten only after the block of two
      // launches ago was examined, so never under a copy in flight)
      PersistCtl& tp = h_pc_[h];
      memset(&tp, 0, sizeof(tp));
      const uint32_t wm = g_->wait_ms.load();
      tp.timeout_ns = (unsigned long long)(wm ? wm : wait_ms_default_) * 1000000ull;
      tp.hold = g_->hold_rounds.load();
      CK(cudaMemcpyAsync(d_pc_, &tp, sizeof(PersistCtl), cudaMemcpyHostToDevice, stream_));
      GraphDev gd{g_->d_beg, g_->d_adj, g_->V, g_->d_wcut};
      // the control steps scan the slots in use: admissions happen only
      // between launches, so none above the highest one starts during it
      int nsc = (int)std::max<uint32_t>(1u, nslots_hi_);
      uint32_t R32 = R;
      PersistCtl* pc = d_pc_;
      void* args[] = {&d_qd_, &d_ctl_, &nsc, &d_rd_, &d_pre_, &gd, &R32, &pc};
      if (prof) CK(cudaEventRecord(ev_prof_[h][0], stream_));
      CK(cudaLaunchCooperativeKernel(kr_, dim3(rounds_grid_), dim3(threads_), args, 0, stream_));
      if (prof) CK(cudaEventRecord(ev_prof_[h][1], stream_));
      CK(cudaMemcpyAsync(h_pc_ + 2 + h, d_pc_, sizeof(PersistCtl), cudaMemcpyDeviceToHost, stream_));
      const int ns = (int)nslots_hi_;
      prof_rounds_[h] = prof ? R : 0;
      g_->launches += 1;
      blk_slots_[h] = (uint32_t)ns;
      CK(cudaMemcpyAsync(h_ctl_ + (size_t)h * MAX_SLOTS, d_ctl_, (size_t)ns * sizeof(QCtl), cudaMemcpyDeviceToHost,
                         stream_));
      CK(cudaEventRecord(ev_blk_[h], stream_));
      return GST_OK;
    }
    if (round_graph_ && R == rounds_per_sync_ && !prof) {
      CK(cudaGraphLaunch(round_graph_, stream_));
    } else {
      // profiled blocks time every kernel with events between the launches
      GraphDev gd{g_->d_beg, g_->d_adj, g_->V, g_->d_wcut};
      const int ns = (int)nslots_hi_;
      cudaEvent_t* pe = ev_prof_[h];
      for (uint32_t r = 0; r < R; r++) {
        k_control<<<1, 1024, 0, stream_>>>(d_qd_, d_ctl_, ns, d_rd_, d_pre_);
        if (prof) CK(cudaEventRecord(pe[3 * r], stream_));
        CK(launch_light(gd, ns));
        if (prof) CK(cudaEventRecord(pe[3 * r + 1], stream_));
        CK(launch_heavy(gd, ns));
        if (prof) CK(cudaEventRecord(pe[3 * r + 2], stream_));
        if (prof && h_rdtrace_)  // the round's work counts, for the per-round trace
          CK(cudaMemcpyAsync(h_rdtrace_ + (size_t)h * 64 + r, d_rd_, sizeof(RoundDesc), cudaMemcpyDeviceToHost,
                             stream_));
      }
    }
    const int ns = (int)nslots_hi_;
    CK(cudaGetLastError());
    prof_rounds_[h] = prof ? R : 0;
    g_->launches += 3ull * R;
    blk_slots_[h] = (uint32_t)ns;
    CK(cudaMemcpyAsync(h_ctl_ + (size_t)h * MAX_SLOTS, d_ctl_, (size_t)ns * sizeof(QCtl), cudaMemcpyDeviceToHost,
                       stream_));
    CK(cudaEventRecord(ev_blk_[h], stream_));
    return GST_OK;
  }

  void accumulate_profile(int h) {
    if (blk_persist_[h]) {
      // one launch for the block: its time goes to the round kernel (light),
      // its rounds are those it ran with a live query
      if (prof_rounds_[h]) {
        float a = 0;
        cudaEventElapsedTime(&a, ev_prof_[h][0], ev_prof_[h][1]);
        g_->prof_light_ms += a;
        g_->prof_rounds += h_pc_[2 + h].rounds;
        g_->prof_persistent = true;
      }
      return;
    }
    for (uint32_t r = 0; r < prof_rounds_[h]; r++) {
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, ev_prof_[h][3 * r], ev_prof_[h][3 * r + 1]);
      cudaEventElapsedTime(&b, ev_prof_[h][3 * r + 1], ev_prof_[h][3 * r + 2]);
      if (h_rdtrace_) {
        // GSTB_TRACE_ROUNDS: one line per profiled round: kernel times and
        // the work of each task type (k_light: split, distance seed, DP seed,
        // tour, extract, distance items, DP states, hop states; k_heavy:
        // bound rows, snapshot rows; plus the arc chunks handed over)
        const RoundDesc& d = h_rdtrace_[(size_t)h * 64 + r];
        fprintf(stderr,
                "gstb round %llu: light %.3f ms heavy %.3f ms | live %u | split %u sseed %u dseed %u tour %u "
                "extract %u sssp %u (w %u) dp %u hop %u | lb %u snap %u | chunks %u%s\n",
                (unsigned long long)g_->prof_rounds, a, b, d.n_live, d.items[T_SPLIT], d.items[T_SSEED],
                d.items[T_DSEED], d.items[T_TOUR], d.items[T_EXTRACT], d.items[T_SSSP], d.sssp_w, d.items[T_DP],
                d.items[T_HOP], d.items[T_LB], d.items[T_SNAP], d.n_big, d.hub_on ? " (chunking)" : "");
      }
      g_->prof_light_ms += a;
      g_->prof_heavy_ms += b;
      g_->prof_rounds++;
    }
  }

  // Jobs that block `blk` saw finish: queue their tree copies, free their
  // workspace and slot (all stream-ordered after the block in flight).
  gst_status detect_done(int64_t blk, std::vector<Job*>& fin, std::vector<size_t>& fin_off) {
    const int h = (int)(blk & 1);
    const QCtl* snap = h_ctl_ + (size_t)h * MAX_SLOTS;
    char* estage = h_edge_stage_ + (size_t)h * (edge_stage_cap_ / 2);
    size_t off = 0;
    // a persistent launch whose bounded wait expired left its queries' rounds
    // unfinished: every query of the block that had not finished fails
    const bool expired = blk_persist_[h] && h_pc_[2 + h].err != 0u;
    if (expired) timeouts_++;
    for (uint32_t s = 0; s < blk_slots_[h]; s++) {
      Job* j = slots_[s];
      if (!j || j->first_block > blk) continue;
      if (!snap[s].done && !expired) continue;
      j->ctl = snap[s];
      j->status = snap[s].done ? (gst_status)j->ctl.final_status : GST_DEVICE_TIMEOUT;
      size_t my = (size_t)-1;
      if (j->status == GST_OK) {
        j->cost = (int32_t)(j->ctl.best_full >> 32);
        j->root = j->ctl.root;
        uint32_t ne = std::min(j->ctl.n_edges, max_edges_dev_);
        j->edges.resize((size_t)ne * 3);
        if (ne) {
          if (off + (size_t)ne * 12 <= edge_stage_cap_ / 2) {
            CK(cudaMemcpyAsync(estage + off, j->qd.out_edges, (size_t)ne * 12, cudaMemcpyDeviceToHost, stream_));
            my = off;
            off += align_up((size_t)ne * 12, 16);
          } else {  // rare: a huge tree, copy it synchronously
            CK(cudaMemcpy(j->edges.data(), j->qd.out_edges, (size_t)ne * 12, cudaMemcpyDeviceToHost));
          }
        }
      }
      // free the slot: a zeroed descriptor is J_FREE for k_control (pinned
      // source, so the copy stays asynchronous)
      CK(cudaMemcpyAsync(d_qd_ + s, h_qd_, sizeof(QDev), cudaMemcpyHostToDevice, stream_));
      free_job(j);
      slots_[s] = nullptr;
      n_used_--;
      fin.push_back(j);
      fin_off.push_back(my);
    }
    while (nslots_hi_ > 0 && !slots_[nslots_hi_ - 1]) nslots_hi_--;
    return GST_OK;
  }

  template <class DoneFn>
  void finalize(std::vector<Job*>& fin, std::vector<size_t>& fin_off, int half, DoneFn&& on_done) {
    const char* estage = h_edge_stage_ + (size_t)half * (edge_stage_cap_ / 2);
    auto now = std::chrono::steady_clock::now();
    for (size_t i = 0; i < fin.size(); i++) {
      Job* j = fin[i];
      // lists of one entry per state cannot overflow; list indices are 32-bit
      const uint64_t cap_max = std::min<uint64_t>((uint64_t)g_->V * j->WT, 1ull << 31);
      if (j->status == GST_QUEUE_OVERFLOW && (uint64_t)j->qd.cap < cap_max) {
        // a frontier outgrew its list: run the query again with 4x the capacity
        j->cap_req = std::min<uint64_t>(cap_max, (uint64_t)j->qd.cap * 4);
        j->retries++;
        Layout L = layout_for(g_, j->k, j->D, j->members.size(), max_edges_dev_, j->cap_req);
        j->bytes = L.total;
        j->status = GST_OK;
        j->edges.clear();
        retry_.push_back(j);
        continue;
      }
      if (j->status == GST_OK && !j->edges.empty() && fin_off[i] != (size_t)-1)
        memcpy(j->edges.data(), estage + fin_off[i], j->edges.size() * 4);
      j->t_done = now;
      j->done = true;
      on_done(j);
    }
    fin.clear();
    fin_off.clear();
  }

  gst_graph* g_;
  Arena arena_;
  std::deque<Job*> retry_;  // queries to run again with larger frontier lists
  cudaStream_t stream_ = nullptr;
  std::vector<Job*> slots_;
  uint32_t n_used_ = 0, nslots_hi_ = 0, max_slots_ = MAX_SLOTS - 1;
  QDev* d_qd_ = nullptr;
  QCtl* d_ctl_ = nullptr;
  RoundDesc* d_rd_ = nullptr;
  uint4* d_big_ = nullptr;
  uint32_t big_cap_ = 0;
  uint32_t* d_pre_ = nullptr;
  QCtl* h_ctl_ = nullptr;
  RoundDesc* h_rd_ = nullptr;
  QDev* h_qd_ = nullptr;
  uint32_t* h_one_ = nullptr;  // pinned 1, the source of cancel flags
  char* h_stage_ = nullptr;
  char* h_edge_stage_ = nullptr;
  size_t stage_cap_ = 0, stage_off_[2] = {0, 0}, edge_stage_cap_ = 0;
  int64_t next_block_ = 0;
  uint32_t blk_slots_[2] = {0, 0}, prof_rounds_[2] = {0, 0};
  bool persist_ = false, blk_persist_[2] = {false, false};
  unsigned rounds_grid_ = 0;  // blocks of the persistent launch (0: cooperative launch unavailable)
  PersistCtl* d_pc_ = nullptr;
  PersistCtl* h_pc_ = nullptr;  // pinned [4]: launch templates, then read-backs, per block half
  uint32_t wait_ms_default_ = 30000;
  uint64_t timeouts_ = 0;
  cudaEvent_t ev_blk_[2] = {nullptr, nullptr}, ev_fin_ = nullptr;
  cudaEvent_t ev_prof_[2][3 * 64] = {};
  RoundDesc* h_rdtrace_ = nullptr;  // pinned [2][64] round descriptors (GSTB_TRACE_ROUNDS)
  uint32_t delta_sssp_ = 8, delta_dp_ = 2, max_edges_dev_ = 1u << 16;
  uint32_t cap_num_ = 1, cap_den_ = 2, rounds_per_sync_ = 6;
  cudaEvent_t ev_[2] = {};
  unsigned light_grid_ = 148 * 4, heavy_grid_ = 148 * 2, resident_light_warps_ = 148 * 4 * 8;
  uint32_t threads_ = 256;  // threads per block of the round kernels
  const void* kl_ = nullptr;
  const void* kh_ = nullptr;
  const void* kr_ = nullptr;
  double last_call_ms_ = 0;
  double trace_ms_ = 0;
  cudaGraphExec_t round_graph_ = nullptr;
};

// Copy a finished job into a caller result.
gst_status fill_result(Job* j, gst_result* r) {
  if (!r) return j->status;
  // a progressive answer: its derivation's edges reduced to a spanning tree
  // (once: poll and batch results call this once per job)
  if (j->status == GST_OK && j->ctl.early && j->edges.size() / 3 == j->ctl.n_edges) {
    spanning_tree(j->edges);
    int64_t sum = 0;
    for (size_t e = 0; e < j->edges.size() / 3; e++) sum += j->edges[3 * e + 2];
    j->cost = (int32_t)sum;
    j->ctl.n_edges = (uint32_t)(j->edges.size() / 3);
    j->ctl.early = 0;
    j->ctl.lb_exit = std::min<uint32_t>(j->ctl.lb_exit, (uint32_t)sum);
    j->lower_bound = j->ctl.lb_exit;
  } else if (j->status == GST_OK && !j->early_done) {
    j->lower_bound = (uint32_t)j->cost;
  }
  j->early_done = true;
  r->cost = j->status == GST_OK ? j->cost : -1;
  r->root = j->root;
  for (int i = 0; i < 12; i++) r->stats[i] = j->ctl.stat[i];
  r->stats[GST_STAT_TABLE_BYTES] = j->table_bytes;
  r->stats[GST_STAT_RETRIES] = j->retries;
  r->stats[GST_STAT_LOWER_BOUND] = j->status == GST_OK ? j->lower_bound : 0;
  r->latency_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_submit).count();
  gst_status st = j->status;
  if (st == GST_OK) {
    int32_t ne = (int32_t)(j->edges.size() / 3);
    r->n_edges = (int32_t)j->ctl.n_edges;
    if (r->edges && r->max_edges > 0) {
      int32_t m = std::min(ne, r->max_edges);
      memcpy(r->edges, j->edges.data(), (size_t)m * 12);
    }
    if ((int64_t)j->ctl.n_edges > (int64_t)r->max_edges && r->edges) st = GST_TRUNCATED;
    // internal check: the tree's weights must add up to the optimum
    int64_t sum = 0;
    for (int32_t e = 0; e < ne; e++) sum += j->edges[(size_t)e * 3 + 2];
    if ((uint32_t)ne == j->ctl.n_edges && sum != j->cost) st = GST_INTERNAL;
  } else {
    r->n_edges = 0;
  }
  return st;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* gst_last_cuda_error(void) { return cudaGetErrorString(last_cuda_error().load()); }

const char* gst_status_string(gst_status st) {
  switch (st) {
    case GST_OK: return "ok";
    case GST_NO_SOLUTION: return "no solution";
    case GST_BAD_INPUT: return "bad input";
    case GST_OOM: return "out of device memory";
    case GST_DEVICE_TIMEOUT: return "device wait timed out";
    case GST_CUDA_ERROR: return "CUDA error";
    case GST_QUEUE_OVERFLOW: return "frontier queue overflow";
    case GST_TRUNCATED: return "tree truncated";
    case GST_INTERNAL: return "internal consistency check failed";
    case GST_BUSY: return "busy";
    case GST_NOT_FOUND: return "not found";
    case GST_SCRATCH_TOO_SMALL: return "query workspace exceeds the static scratch";
    case GST_CANCELLED: return "cancelled";
  }
  return "unknown";
}

gst_status gst_graph_create(const uint32_t* beg_pos, const uint32_t* csr, const int32_t* w, uint32_t V,
                            uint64_t arcs, gst_graph** out) {
  if (!out || !beg_pos || (arcs && (!csr || !w)) || V == 0) return GST_BAD_INPUT;
  *out = nullptr;
  if (arcs >= (1ull << 32) || V >= (1u << 29)) return GST_BAD_INPUT;
  if (beg_pos[0] != 0 || beg_pos[V] != arcs) return GST_BAD_INPUT;
  for (uint32_t v = 0; v < V; v++)
    if (beg_pos[v + 1] < beg_pos[v]) return GST_BAD_INPUT;
  // validate arcs and build the weight-sorted adjacency on the host
  std::vector<uint2> adj(arcs);
  bool bad = false;
  unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  std::atomic<bool> abad{false};
  for (unsigned t = 0; t < nth; t++) {
    th.emplace_back([&, t]() {
      for (uint32_t v = t; v < V; v += nth) {
        uint32_t a0 = beg_pos[v], a1 = beg_pos[v + 1];
        for (uint32_t a = a0; a < a1; a++) {
          if (csr[a] >= V || w[a] < 1) abad = true;
          adj[a] = make_uint2(csr[a], (uint32_t)w[a]);
        }
        std::sort(adj.begin() + a0, adj.begin() + a1, [](const uint2& x, const uint2& y) {
          return x.y != y.y ? x.y < y.y : x.x < y.x;
        });
      }
    });
  }
  for (auto& x : th) x.join();
  bad = abad;
  if (bad) return GST_BAD_INPUT;
  // Integer range: every distance and tree cost is summed in 32 bits and the
  // lower bounds saturate at BIG = 2^30 (a saturated bound reads as
  // "unreachable").  A shortest path or a tree has at most V-1 edges, so the
  // V-1 heaviest arcs bound every such cost; the graph is rejected if that
  // bound can reach 2^30.
  if (arcs) {
    uint32_t wmax = 0;
    for (uint64_t a = 0; a < arcs; a++) wmax = std::max(wmax, adj[a].y);
    if ((uint64_t)(V - 1) * wmax >= (uint64_t)BIG) {
      std::vector<uint32_t> ws(arcs);
      for (uint64_t a = 0; a < arcs; a++) ws[a] = adj[a].y;
      const size_t m = std::min<size_t>(ws.size(), (size_t)V - 1);
      std::nth_element(ws.begin(), ws.begin() + m, ws.end(), std::greater<uint32_t>());
      uint64_t heavy = 0;
      for (size_t i = 0; i < m; i++) heavy += ws[i];
      if (heavy >= (uint64_t)BIG) return GST_BAD_INPUT;
    }
  }
  gst_graph* g = new gst_graph();
  g->V = V;
  g->arcs = arcs;
  g->tune.delta_sssp = std::max(1u, env_u32("GSTB_DELTA_SSSP", 16));
  g->tune.delta_dp = std::max(1u, env_u32("GSTB_DELTA_DP", 8));
  g->tune.hub_min_deg = std::max(32u, env_u32("GSTB_HUB_MIN_DEG", 256));
  g->tune.cap_pct = std::min(100u, std::max(1u, env_u32("GSTB_SSSP_CAP_PCT", 60)));
  g->tune.persistent = env_u32("GSTB_PERSIST", 0) ? 1u : 0u;
  g->tune.rounds_per_launch = std::min(64u, std::max(1u, env_u32("GSTB_ROUNDS_PER_SYNC", 4)));
  g->tune.dp_wmax = floor_pow2(std::min(32u, std::max(1u, env_u32("GSTB_DP_WMAX", 32))));
  g->tune.sssp_wmax = floor_pow2(std::min(32u, std::max(4u, env_u32("GSTB_SSSP_WMAX", 32))));
  g->tune.merge_stage = env_u32("GSTB_MERGE_STAGE", 14);
  g->tune.block_threads = env_u32("GSTB_BLOCK_THREADS", 256) == 128 ? 128u : 256u;
  cudaGetDevice(&g->device);
  cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device);
  {
    size_t fr = 0;
    if (cudaMemGetInfo(&fr, &g->total_mem) != cudaSuccess) {
      cudaGetLastError();
      g->total_mem = 0;
    }
  }
  if (cudaMalloc(&g->d_beg, (size_t)(V + 1) * 4) != cudaSuccess ||
      cudaMalloc(&g->d_adj, std::max<size_t>(arcs, 1) * 8) != cudaSuccess) {
    cudaGetLastError();
    gst_graph_destroy(g);
    return GST_OOM;
  }
  if (cudaMemcpy(g->d_beg, beg_pos, (size_t)(V + 1) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      (arcs && cudaMemcpy(g->d_adj, adj.data(), arcs * 8, cudaMemcpyHostToDevice) != cudaSuccess)) {
    gst_graph_destroy(g);
    return GST_CUDA_ERROR;
  }
  {
    // weight-bucket index: for each vertex the first arc heavier than 2^b
    std::vector<uint32_t> wc((size_t)V * 8);
    std::vector<std::thread> tw;
    for (unsigned t = 0; t < nth; t++) {
      tw.emplace_back([&, t]() {
        for (uint32_t v = t; v < V; v += nth) {
          uint32_t a = beg_pos[v], a1 = beg_pos[v + 1];
          for (int b = 0; b < 8; b++) {
            uint32_t th = 1u << b;
            while (a < a1 && adj[a].y <= th) a++;
            wc[(size_t)v * 8 + b] = a;
          }
        }
      });
    }
    for (auto& x : tw) x.join();
    if (cudaMalloc(&g->d_wcut, wc.size() * 4) != cudaSuccess) {
      cudaGetLastError();
      gst_graph_destroy(g);
      return GST_OOM;
    }
    if (cudaMemcpy(g->d_wcut, wc.data(), wc.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
      gst_graph_destroy(g);
      return GST_CUDA_ERROR;
    }
  }
  *out = g;
  return GST_OK;
}

gst_status gst_groups_set(gst_graph* g, const uint64_t* grp_ptr, const uint32_t* grp_v, uint32_t n_groups) {
  if (!g || !grp_ptr || n_groups == 0) return GST_BAD_INPUT;
  if (grp_ptr[0] != 0) return GST_BAD_INPUT;
  for (uint32_t i = 0; i < n_groups; i++)
    if (grp_ptr[i + 1] < grp_ptr[i]) return GST_BAD_INPUT;
  uint64_t n = grp_ptr[n_groups];
  if (n && !grp_v) return GST_BAD_INPUT;
  for (uint64_t t = 0; t < n; t++)
    if (grp_v[t] >= g->V) return GST_BAD_INPUT;
  std::unique_lock<std::shared_mutex> lock(g->grp_mu);
  g->grp_ptr.assign(grp_ptr, grp_ptr + n_groups + 1);
  g->grp_v.assign(grp_v, grp_v + n);
  return GST_OK;
}

void gst_graph_destroy(gst_graph* g) {
  if (!g) return;
  if (g->runner) delete static_cast<Runner*>(g->runner);
  if (g->d_beg) cudaFree(g->d_beg);
  if (g->d_adj) cudaFree(g->d_adj);
  if (g->d_wcut) cudaFree(g->d_wcut);
  delete g;
}

uint64_t gst_kernel_launches(const gst_graph* g) { return g ? g->launches.load() : 0; }

void gst_profile_enable(gst_graph* g, int on) {
  if (g) g->profile = on != 0;
}

void gst_profile_read(const gst_graph* g, double* kernel_ms, uint64_t* rounds, uint64_t* totals) {
  if (!g) return;
  if (kernel_ms) {
    kernel_ms[0] = g->prof_light_ms;
    kernel_ms[1] = g->prof_heavy_ms;
  }
  if (rounds) *rounds = g->prof_rounds;
  if (totals)
    for (int t = 0; t < GST_NSTATS; t++) totals[t] = g->prof_stats[t];
}

void gst_profile_reset(gst_graph* g) {
  if (!g) return;
  g->prof_light_ms = g->prof_heavy_ms = 0;
  g->prof_rounds = 0;
  g->prof_persistent = false;
  for (int t = 0; t < GST_NSTATS; t++) g->prof_stats[t] = 0;
}

uint32_t gst_graph_num_vertices(const gst_graph* g) { return g ? g->V : 0; }
uint64_t gst_graph_num_arcs(const gst_graph* g) { return g ? g->arcs : 0; }

gst_status gst_query_ratio(gst_graph* g, const uint32_t* groups, int k, int D, double ratio, gst_result* out) {
  int32_t ks = k, Ds = D;
  int32_t st = 0;
  if (k < 1 || k > KMAX || !groups) return GST_BAD_INPUT;
  uint32_t gg[GST_GROUPS_STRIDE] = {0};
  memcpy(gg, groups, (size_t)k * 4);
  gst_status s = gst_query_batch_ratio(g, 1, gg, &ks, &Ds, &ratio, out, &st, 1);
  if (s != GST_OK) return s;
  return (gst_status)st;
}

gst_status gst_query(gst_graph* g, const uint32_t* groups, int k, int D, gst_result* out) {
  return gst_query_ratio(g, groups, k, D, 0.0, out);
}

gst_status gst_tuning_get(gst_graph* g, gst_tuning* out) {
  if (!g || !out) return GST_BAD_INPUT;
  std::lock_guard<std::mutex> lock(g->mu);
  *out = g->tune;
  return GST_OK;
}

gst_status gst_tuning_set(gst_graph* g, const gst_tuning* t) {
  auto pow2_in = [](uint32_t x, uint32_t lo, uint32_t hi) { return x >= lo && x <= hi && (x & (x - 1)) == 0; };
  if (!g || !t || t->delta_sssp < 1 || t->delta_dp < 1 || t->hub_min_deg < 32 || t->cap_pct < 1 ||
      t->cap_pct > 100 || t->persistent > 1 || t->rounds_per_launch < 1 || t->rounds_per_launch > 64 ||
      !pow2_in(t->dp_wmax, 1, 32) || !pow2_in(t->sssp_wmax, 4, 32) ||
      (t->block_threads != 128 && t->block_threads != 256))
    return GST_BAD_INPUT;
  std::lock_guard<std::mutex> lock(g->mu);
  g->tune = *t;
  if (g->runner) return static_cast<Runner*>(g->runner)->apply_tuning();
  return GST_OK;
}

gst_status gst_query_batch(gst_graph* g, int n, const uint32_t* groups, const int32_t* ks, const int32_t* Ds,
                           gst_result* results, int32_t* statuses, int max_concurrent) {
  return gst_query_batch_ratio(g, n, groups, ks, Ds, nullptr, results, statuses, max_concurrent);
}

gst_status gst_query_batch_ratio(gst_graph* g, int n, const uint32_t* groups, const int32_t* ks, const int32_t* Ds,
                                 const double* ratios, gst_result* results, int32_t* statuses, int max_concurrent) {
  if (!g || n < 0 || (n > 0 && (!groups || !ks || !Ds || !statuses))) return GST_BAD_INPUT;
  if (!has_groups(g)) return GST_BAD_INPUT;
  std::lock_guard<std::mutex> lock(g->mu);
  if (!g->runner) {
    Runner* nr = new Runner(g);
    gst_status st = nr->init();
    if (st != GST_OK) {
      delete nr;
      return st;
    }
    g->runner = nr;
  }
  Runner& R = *static_cast<Runner*>(g->runner);
  using clk = std::chrono::steady_clock;
  const clk::time_point t0 = clk::now();
  std::vector<Job> jobs(n);
  std::deque<Job*> pending;
  for (int i = 0; i < n; i++) {
    Job& j = jobs[i];
    j.k = ks[i];
    j.D = Ds[i] < 0 ? -1 : Ds[i];
    j.tag = (uint64_t)i;
    j.ratio_num = ratios ? ratio_to_num(ratios[i]) : 0u;
    j.res = results ? &results[i] : nullptr;
    if (j.k < 1 || j.k > KMAX) {
      statuses[i] = GST_BAD_INPUT;
      j.done = true;
      j.rejected = true;
      continue;
    }
    memcpy(j.groups, groups + (size_t)i * GST_GROUPS_STRIDE, (size_t)j.k * 4);
    j.t_submit = std::chrono::steady_clock::now();
    gst_status ps = R.prepare(&j);
    if (ps != GST_OK) {
      statuses[i] = ps;
      if (j.res) {
        j.res->cost = -1;
        j.res->n_edges = 0;
      }
      j.done = true;
      j.rejected = true;
      continue;
    }
    pending.push_back(&j);
  }
  const size_t maxc = max_concurrent > 0 ? (size_t)max_concurrent : (size_t)1 << 20;
  {
    // workspace for the first wave of the batch in one arena allocation
    size_t need = 0, cnt = 0;
    for (Job* j : pending) {
      if (cnt++ >= std::min<size_t>(maxc, MAX_SLOTS - 1)) break;
      need += align_up(j->bytes, 256);
    }
    // best effort: admission still grows the arena or waits.  The device is
    // asked for its free memory only when the arena must grow (the query can
    // take milliseconds)
    if (!R.has_free(need)) {
      size_t fr = 0, tot = 0;
      if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) need = std::min(need, (size_t)(fr * 0.8));
      R.reserve(need);
    }
  }
  const clk::time_point t1 = clk::now();
  gst_status rs = R.run(
      [&]() {
        while (!pending.empty() && R.live() < maxc && R.has_free_slot()) {
          Job* j = pending.front();
          if (!R.admit(j)) {
            if (R.live() == 0) {  // cannot fit even alone
              j->status = GST_OOM;
              j->done = true;
              pending.pop_front();
              continue;
            }
            break;
          }
          pending.pop_front();
        }
      },
      [&](Job*) {});
  if (rs != GST_OK) return rs;
  // The arena keeps its chunks for the next batch (handing them back and
  // allocating them again cost a cudaFree / cudaMalloc pair per batch).
  // GSTB_ARENA_KEEP_MB caps what it keeps; a serving loop opened on this
  // graph takes back the wholly free chunks first (gst_serve_open).
  {
    const uint32_t keep_mb = env_u32("GSTB_ARENA_KEEP_MB", 0);
    if (keep_mb) R.release_arena_above((size_t)keep_mb << 20);
  }

  const clk::time_point t2 = clk::now();
  for (int i = 0; i < n; i++) {
    Job& j = jobs[i];
    if (j.rejected) continue;
    statuses[i] = fill_result(&j, j.res);
    if (j.res) j.res->device_ms = R.last_call_ms();
    if (g->profile)
      for (int t = 0; t < 12; t++) g->prof_stats[t] += j.ctl.stat[t];
  }
  const double tr = R.trace_ms();
  if (tr > 0) {
    auto ms = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    const double all = ms(t0, clk::now());
    if (all >= tr)
      fprintf(stderr, "gstb: batch of %d: %.2f ms (prepare %.2f, run %.2f with %.2f on the device, results %.2f)\n", n,
              all, ms(t0, t1), ms(t1, t2), R.last_call_ms(), ms(t2, clk::now()));
  }
  return GST_OK;
}

gst_status gst_autotune(gst_graph* g, int n, const uint32_t* groups, const int32_t* ks, const int32_t* Ds,
                        int objective, gst_tuning* out) {
  if (!g || n < 1 || !groups || !ks || !Ds || (objective != 0 && objective != 1)) return GST_BAD_INPUT;
  std::vector<int32_t> statuses(n);
  std::vector<uint32_t> edges;  // trees are not needed: results without edge buffers
  std::vector<gst_result> res(n);
  // time of the sample under the current tuning: the batch once (throughput)
  // or every query alone (latency), best of two runs after a warm-up
  auto measure = [&](double& ms) -> gst_status {
    double bestv = 1e300;
    for (int rep = 0; rep < 3; rep++) {
      auto t0 = std::chrono::steady_clock::now();
      if (objective == 0) {
        for (auto& r : res) r = gst_result{};
        gst_status st = gst_query_batch(g, n, groups, ks, Ds, res.data(), statuses.data(), 0);
        if (st != GST_OK) return st;
      } else {
        for (int i = 0; i < n; i++) {
          gst_result r{};
          gst_status st = gst_query(g, groups + (size_t)i * GST_GROUPS_STRIDE, ks[i], Ds[i], &r);
          if (st == GST_CUDA_ERROR || st == GST_INTERNAL) return st;
        }
      }
      double t = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (rep > 0) bestv = std::min(bestv, t);
    }
    ms = bestv;
    return GST_OK;
  };
  gst_tuning cur;
  gst_status st = gst_tuning_get(g, &cur);
  if (st != GST_OK) return st;
  double best_ms = 0;
  st = measure(best_ms);
  if (st != GST_OK) return st;
  // one parameter at a time over a few candidates each
  struct Cand {
    uint32_t gst_tuning::*field;
    std::vector<uint32_t> vals;
  };
  const Cand cands[] = {
      {&gst_tuning::cap_pct, {50, 60, 67, 75}},
      {&gst_tuning::delta_sssp, {8, 16, 32, 64}},
      {&gst_tuning::delta_dp, {2, 4, 8, 16}},
      {&gst_tuning::hub_min_deg, {128, 256, 512, 1024}},
      {&gst_tuning::persistent, {0, 1}},
      {&gst_tuning::rounds_per_launch, {2, 4, 8, 16}},
      {&gst_tuning::dp_wmax, {4, 8, 16, 32}},
      {&gst_tuning::sssp_wmax, {8, 16, 32}},
      {&gst_tuning::merge_stage, {0, 6, 14, 30}},
      {&gst_tuning::block_threads, {128, 256}},
  };
  for (const Cand& cd : cands) {
    for (uint32_t v : cd.vals) {
      if (v == cur.*cd.field) continue;
      gst_tuning t = cur;
      t.*cd.field = v;
      if ((st = gst_tuning_set(g, &t)) != GST_OK) return st;
      double ms = 0;
      if ((st = measure(ms)) != GST_OK) return st;
      if (ms < best_ms * 0.98) {  // keep a change only if it is clearly faster
        best_ms = ms;
        cur = t;
      }
    }
    if ((st = gst_tuning_set(g, &cur)) != GST_OK) return st;
  }
  if (out) *out = cur;
  return GST_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving loop (continuous batching).  A host thread owns a Runner; requests
// submitted while others run are admitted as soon as a slot and HBM budget
// free up, and share every device round with the requests already running.
// ---------------------------------------------------------------------------
struct gst_server {
  gst_graph* g = nullptr;
  Runner* runner = nullptr;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Job*> pending;
  std::deque<Job*> finished;
  bool stop = false;
  uint64_t budget = 0, in_use = 0;
  size_t max_inflight = 0, inflight = 0;
  size_t max_pending = 1u << 20;
  std::vector<uint64_t> cancels;  // admitted requests to withdraw (the loop applies them)
  std::unordered_multiset<uint64_t> running;  // ids of the admitted requests
  uint64_t n_submitted = 0, n_completed = 0, n_busy = 0, n_cancelled = 0, n_oom = 0;
  gst_status fatal = GST_OK;
};

static void serve_loop(gst_server* S) {
  cudaSetDevice(S->g->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv.wait(lk, [&] { return S->stop || !S->pending.empty(); });
      if (S->stop && S->pending.empty()) return;
    }
    gst_status st = S->runner->run(
        [&]() {
          std::lock_guard<std::mutex> lk(S->mu);
          for (uint64_t id : S->cancels) S->runner->cancel_tag(id);
          S->cancels.clear();
          while (!S->pending.empty() && S->inflight < S->max_inflight && S->runner->has_free_slot()) {
            Job* j = S->pending.front();
            if (S->in_use + j->bytes > S->budget && S->inflight > 0) break;  // wait for memory
            if (!S->runner->admit(j)) {
              if (S->inflight == 0) {  // does not fit even alone
                j->status = GST_OOM;
                j->done = true;
                j->t_done = std::chrono::steady_clock::now();
                S->pending.pop_front();
                S->finished.push_back(j);
                S->n_completed++;
                S->n_oom++;
                continue;
              }
              break;
            }
            S->pending.pop_front();
            S->inflight++;
            S->in_use += j->bytes;
            S->running.insert(j->tag);
          }
        },
        [&](Job* j) {
          std::lock_guard<std::mutex> lk(S->mu);
          S->inflight--;
          S->in_use -= j->bytes;
          {
            auto it = S->running.find(j->tag);
            if (it != S->running.end()) S->running.erase(it);
          }
          S->finished.push_back(j);
          S->n_completed++;
          if (j->status == GST_CANCELLED) S->n_cancelled++;
          if (j->status == GST_OOM) S->n_oom++;
        });
    if (st != GST_OK) {
      std::lock_guard<std::mutex> lk(S->mu);
      S->fatal = st;
      return;
    }
  }
}

extern "C" {

gst_status gst_serve_open(gst_graph* g, uint64_t hbm_budget_bytes, int max_inflight, gst_server** out) {
  if (!g || !out || !has_groups(g)) return GST_BAD_INPUT;
  *out = nullptr;
  {
    // the batch engine of this graph gives back its wholly free workspace
    // chunks, which the serving loop's own arena may need
    std::lock_guard<std::mutex> lock(g->mu);
    if (g->runner) static_cast<Runner*>(g->runner)->release_arena_above(0);
  }
  gst_server* S = new gst_server();
  S->g = g;
  S->runner = new Runner(g);
  gst_status st = S->runner->init();
  if (st != GST_OK) {
    delete S->runner;
    delete S;
    return st;
  }
  if (hbm_budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    hbm_budget_bytes = (uint64_t)(fr * 0.8);
  }
  S->budget = hbm_budget_bytes;
  // reserve the whole budget now, in one allocation, rather than growing
  // while requests wait: a growth is a cudaMalloc on the loop's thread, and
  // on the 3M-vertex mix growing request by request held the closed-loop
  // rate at 64 in flight to 136 q/s against 181 q/s for batches.
  // GSTB_SERVE_RESERVE_MB caps the reservation; if it cannot be had at once,
  // the arena grows per request as before
  {
    const uint32_t cap_mb = env_u32("GSTB_SERVE_RESERVE_MB", 0);
    const uint64_t want = cap_mb ? std::min<uint64_t>(hbm_budget_bytes, (uint64_t)cap_mb << 20) : hbm_budget_bytes;
    S->runner->reserve(want);
  }
  S->max_inflight = max_inflight > 0 ? (size_t)max_inflight : (size_t)(MAX_SLOTS - 1);
  S->th = std::thread(serve_loop, S);
  *out = S;
  return GST_OK;
}

gst_status gst_serve_submit(gst_server* S, uint64_t req_id, const uint32_t* groups, int k, int D) {
  return gst_serve_submit_ratio(S, req_id, groups, k, D, 0.0);
}

gst_status gst_serve_submit_ratio(gst_server* S, uint64_t req_id, const uint32_t* groups, int k, int D,
                                  double ratio) {
  if (!S || !groups) return GST_BAD_INPUT;
  Job* j = new Job();
  j->tag = req_id;
  j->ratio_num = ratio_to_num(ratio);
  j->k = k;
  j->D = D < 0 ? -1 : D;
  j->t_submit = std::chrono::steady_clock::now();
  gst_status ps = (k >= 1 && k <= KMAX) ? GST_OK : GST_BAD_INPUT;
  if (ps == GST_OK) {
    memcpy(j->groups, groups, (size_t)k * 4);
    ps = S->runner->prepare(j);  // host-only validation, no device work
  }
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal != GST_OK) {
    delete j;
    return S->fatal;
  }
  if (ps != GST_OK) {  // rejected: reported through poll like any result
    j->status = ps;
    j->rejected = true;
    j->done = true;
    j->t_done = j->t_submit;
    S->finished.push_back(j);
    S->n_submitted++;
    S->n_completed++;
    return GST_OK;
  }
  if (S->pending.size() >= S->max_pending) {
    delete j;
    S->n_busy++;
    return GST_BUSY;
  }
  S->n_submitted++;
  S->pending.push_back(j);
  S->cv.notify_one();
  return GST_OK;
}

gst_status gst_serve_poll(gst_server* S, uint64_t* ids, int32_t* statuses, gst_result* results, int max_results,
                          int* n_out) {
  if (!S || !n_out || max_results < 0 || (max_results > 0 && (!ids || !statuses))) return GST_BAD_INPUT;
  std::vector<Job*> got;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    while (!S->finished.empty() && (int)got.size() < max_results) {
      got.push_back(S->finished.front());
      S->finished.pop_front();
    }
    if (got.empty() && S->fatal != GST_OK) {
      *n_out = 0;
      return S->fatal;
    }
  }
  for (size_t i = 0; i < got.size(); i++) {
    Job* j = got[i];
    ids[i] = j->tag;
    if (j->rejected) {
      statuses[i] = j->status;
      if (results) {
        results[i].cost = -1;
        results[i].n_edges = 0;
        results[i].latency_ms = 0;
      }
    } else {
      statuses[i] = fill_result(j, results ? &results[i] : nullptr);
    }
    delete j;
  }
  *n_out = (int)got.size();
  return GST_OK;
}

gst_status gst_serve_cancel(gst_server* S, uint64_t req_id) {
  if (!S) return GST_BAD_INPUT;
  std::lock_guard<std::mutex> lk(S->mu);
  for (auto it = S->pending.begin(); it != S->pending.end(); ++it) {
    Job* j = *it;
    if (j->tag != req_id) continue;
    S->pending.erase(it);  // never admitted: finished at once
    j->status = GST_CANCELLED;
    j->rejected = true;
    j->done = true;
    j->t_done = std::chrono::steady_clock::now();
    S->finished.push_back(j);
    S->n_completed++;
    S->n_cancelled++;
    return GST_OK;
  }
  if (S->running.find(req_id) == S->running.end()) return GST_NOT_FOUND;
  // admitted: the serving loop withdraws it at its next iteration (a request
  // that finishes meanwhile keeps its own result)
  S->cancels.push_back(req_id);
  return GST_OK;
}

gst_status gst_serve_set_max_pending(gst_server* S, uint64_t max_pending) {
  if (!S || max_pending == 0) return GST_BAD_INPUT;
  std::lock_guard<std::mutex> lk(S->mu);
  S->max_pending = (size_t)max_pending;
  return GST_OK;
}

gst_status gst_serve_stats(gst_server* S, gst_serve_info* out) {
  if (!S || !out) return GST_BAD_INPUT;
  std::lock_guard<std::mutex> lk(S->mu);
  out->pending = S->pending.size();
  out->inflight = S->inflight;
  out->finished_unpolled = S->finished.size();
  out->budget_bytes = S->budget;
  out->in_use_bytes = S->in_use;
  out->submitted = S->n_submitted;
  out->completed = S->n_completed;
  out->rejected_busy = S->n_busy;
  out->cancelled = S->n_cancelled;
  out->oom = S->n_oom;
  return GST_OK;
}

gst_status gst_debug_fail_allocs(gst_graph* g, int n) {
  if (!g || n < 0) return GST_BAD_INPUT;
  g->fail_allocs.store(n);
  return GST_OK;
}

gst_status gst_debug_hold_rounds(gst_graph* g, int hold, uint32_t timeout_ms) {
  if (!g || hold < 0 || hold > 1) return GST_BAD_INPUT;
  g->wait_ms.store(timeout_ms);
  g->hold_rounds.store((uint32_t)hold);
  return GST_OK;
}

gst_status gst_serve_close(gst_server* S) {
  if (!S) return GST_BAD_INPUT;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  if (S->th.joinable()) S->th.join();
  for (Job* j : S->pending) delete j;
  for (Job* j : S->finished) delete j;
  delete S->runner;
  delete S;
  return GST_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free query (gst_query_noalloc).  One static device array holds
// every buffer of a single query; its device address is looked up once per
// device.  Uses the kernels of the regular path with a single slot.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[GST_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_noalloc_mu;
constexpr int NOALLOC_MAX_DEVICES = 64;
void* g_noalloc_base[NOALLOC_MAX_DEVICES] = {nullptr};

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
}  // namespace

extern "C" gst_status gst_query_noalloc(gst_graph* g, const uint32_t* groups, int k, int D, gst_result* out) {
  if (!g || !groups || k < 1 || k > KMAX || D > DMAX) return GST_BAD_INPUT;
  if (D < 0) D = -1;
  for (int a = 0; a < k; a++)
    for (int b = a + 1; b < k; b++)
      if (groups[a] == groups[b]) return GST_BAD_INPUT;
  const int nd = D < 0 ? 1 : D + 1;
  const uint32_t WT = (1u << k) * (uint32_t)nd;
  // the same size limits as the other entry points (member items are v*8+j in 32 bits)
  if ((uint64_t)g->V * WT >= (1ull << 32) || g->V >= (1u << 29)) return GST_BAD_INPUT;
  if (g->device < 0 || g->device >= NOALLOC_MAX_DEVICES) return GST_BAD_INPUT;
  // the graph's lock first (the group index and the tuning are read below and
  // gst_groups_set / gst_tuning_set change them under it), then the scratch's
  std::lock_guard<std::mutex> glock(g->mu);
  std::shared_lock<std::shared_mutex> grlock(g->grp_mu);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g->grp_ptr.empty()) return GST_BAD_INPUT;
  const uint32_t ng = (uint32_t)(g->grp_ptr.size() - 1);
  for (int i = 0; i < k; i++)
    if (groups[i] >= ng) return GST_BAD_INPUT;
  uint64_t n_members = 0;
  for (int i = 0; i < k; i++) {
    uint64_t n = g->grp_ptr[groups[i] + 1] - g->grp_ptr[groups[i]];
    if (n == 0) return GST_NO_SOLUTION;
    n_members += n;
  }
  DeviceGuard guard;
  CK(cudaGetDevice(&guard.prev));
  CK(cudaSetDevice(g->device));
  if (!g_noalloc_base[g->device]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_base[g->device] = p;
  }
  char* base = static_cast<char*>(g_noalloc_base[g->device]);

  // scratch = [QDev][QCtl][RoundDesc][pre: NT x (MAX_SLOTS+1)][workspace]
  const uint32_t max_edges = 4096;
  size_t o = 0;
  const size_t o_qd = o;
  o = align_up(o + sizeof(QDev), 256);
  const size_t o_ctl = o;
  o = align_up(o + sizeof(QCtl), 256);
  const size_t o_rd = o;
  o = align_up(o + sizeof(RoundDesc), 256);
  const size_t o_pre = o;
  o = align_up(o + (size_t)NT * (MAX_SLOTS + 1) * 4, 256);
  const size_t o_ws = o;
  Layout L = layout_for(g, k, D, (size_t)n_members, max_edges);
  if (o_ws + L.total > GST_NOALLOC_SCRATCH_BYTES) return GST_SCRATCH_TOO_SMALL;

  QDev* d_qd = reinterpret_cast<QDev*>(base + o_qd);
  QCtl* d_ctl = reinterpret_cast<QCtl*>(base + o_ctl);
  RoundDesc* d_rd = reinterpret_cast<RoundDesc*>(base + o_rd);
  uint32_t* d_pre = reinterpret_cast<uint32_t*>(base + o_pre);
  char* ws = base + o_ws;

  QDev q;
  memset(&q, 0, sizeof(q));
  q.table = (unsigned long long*)(ws + L.table);
  q.dist = (uint32_t*)(ws + L.dist);
  q.dist_nx = D >= 0 ? (uint32_t*)(ws + L.dist2) : q.dist;
  q.dflag = (uint32_t*)(ws + L.dflag);
  for (int b = 0; b < 4; b++) q.qbuf[b] = (uint32_t*)(ws + L.qbuf) + (size_t)b * L.cap;
  q.tour = (uint32_t*)(ws + L.tour);
  q.lbt = (unsigned short*)(ws + L.lbt);
  q.snap = (uint32_t*)(ws + L.snap);
  q.members = (const uint32_t*)(ws + L.members);
  q.out_edges = (uint32_t*)(ws + L.edges);
  q.ctl = d_ctl;
  q.cap = L.cap;
  q.nv = g->V;
  q.n_members = (uint32_t)n_members;
  q.max_edges = max_edges;
  q.k = k;
  q.D = D;
  q.nd = nd;
  q.full = (int)((1u << k) - 1u);
  q.WT = WT;
  q.phase = PH_SSSP;
  q.cap_num = D >= 0 ? 1u : g->tune.cap_pct;
  q.cap_den = D >= 0 ? 1u : 100u;
  q.star_h = D >= 2 ? (uint32_t)D / 2u : 0u;
  q.center_h = D >= 2 ? ((uint32_t)D + 1u) / 2u : 0u;
  q.in_idx = 0;
  q.out_idx = 1;
  q.far_idx = 2;
  q.far2_idx = 3;
  q.st = J_INIT;
  q.act = A_NONE;
  q.delta_sssp = g->tune.delta_sssp;
  q.delta_dp = g->tune.delta_dp;
  QCtl c;
  memset(&c, 0, sizeof(c));
  c.best = INF32;
  c.best_full = INF64;

  auto t0 = std::chrono::steady_clock::now();
  // the array keeps the previous call's contents: reset what must start empty
  CK(cudaMemsetAsync(q.table, 0xFF, (size_t)g->V * WT * 8, 0));
  CK(cudaMemsetAsync(q.dist, 0xFF, (size_t)g->V * ROW * 4, 0));
  CK(cudaMemset2DAsync(q.dist + FLAGW, ROW * 4, 0, 4, g->V, 0));
  if (q.dist_nx != q.dist) {
    CK(cudaMemsetAsync(q.dist_nx, 0xFF, (size_t)g->V * ROW * 4, 0));
    CK(cudaMemset2DAsync(q.dist_nx + FLAGW, ROW * 4, 0, 4, g->V, 0));
  }
  CK(cudaMemsetAsync(q.dflag, 0, L.qbuf - L.dflag, 0));
  // grids: every SM filled to the occupancy limit of each kernel
  int bl = 0, bh = 0;
  const void* kl = light_kernel(256);
  const void* kh = heavy_kernel(256);
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bl, kl, 256, 0));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bh, kh, 256, 0));
  const unsigned light_grid = (unsigned)g->num_sms * (unsigned)std::max(1, bl);
  const unsigned heavy_grid = (unsigned)g->num_sms * (unsigned)std::max(1, bh);
  {
    RoundDesc rd0;  // no arc chunk list: chunking stays off
    memset(&rd0, 0, sizeof(rd0));
    rd0.light_warps = light_grid * (256 / 32);
    rd0.sssp_w = 4;
    rd0.dp_wmax = g->tune.dp_wmax;
    rd0.sssp_wmax = g->tune.sssp_wmax;
    rd0.merge_stage = g->tune.merge_stage;
    CK(cudaMemcpy(d_rd, &rd0, sizeof(RoundDesc), cudaMemcpyHostToDevice));
  }
  // member items v*8 + j, staged through a fixed host array (calls are
  // serialised, so one array serves them all): one copy per 64K members
  {
    static uint32_t stage[1u << 16];
    size_t n = 0, off = 0;
    for (int i = 0; i < k; i++) {
      for (uint64_t t = g->grp_ptr[groups[i]]; t < g->grp_ptr[groups[i] + 1]; t++) {
        stage[n++] = g->grp_v[t] * 8u + (uint32_t)i;
        if (n == (1u << 16)) {
          CK(cudaMemcpy((uint32_t*)q.members + off, stage, n * 4, cudaMemcpyHostToDevice));
          off += n;
          n = 0;
        }
      }
    }
    if (n) CK(cudaMemcpy((uint32_t*)q.members + off, stage, n * 4, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(d_qd, &q, sizeof(QDev), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_ctl, &c, sizeof(QCtl), cudaMemcpyHostToDevice));

  GraphDev gd{g->d_beg, g->d_adj, g->V, g->d_wcut};
  const uint32_t R = 6;
  const uint64_t max_rounds = 1ull << 22;
  uint64_t rounds = 0;
  for (;;) {
    for (uint32_t r = 0; r < R; r++) {
      k_control<<<1, 1024, 0, 0>>>(d_qd, d_ctl, 1, d_rd, d_pre);
      {
        int one = 1;
        void* args[] = {&d_qd, &d_rd, &d_pre, &one, &gd};
        CK(cudaLaunchKernel(kl, dim3(light_grid), dim3(256), args, 0, 0));
        CK(cudaLaunchKernel(kh, dim3(heavy_grid), dim3(256), args, 0, 0));
      }
    }
    CK(cudaGetLastError());
    g->launches += 3ull * R;
    rounds += R;
    CK(cudaMemcpy(&c, d_ctl, sizeof(QCtl), cudaMemcpyDeviceToHost));
    if (c.done) break;
    if (rounds > max_rounds) return GST_INTERNAL;
  }
  auto t1 = std::chrono::steady_clock::now();
  gst_status st = (gst_status)c.final_status;
  if (out) {
    out->cost = st == GST_OK ? (int32_t)(c.best_full >> 32) : -1;
    out->root = c.root;
    out->n_edges = st == GST_OK ? (int32_t)c.n_edges : 0;
    for (int i = 0; i < 12; i++) out->stats[i] = c.stat[i];
    out->stats[GST_STAT_TABLE_BYTES] = (uint64_t)g->V * WT * 8;
    out->stats[GST_STAT_RETRIES] = 0;
    out->stats[GST_STAT_LOWER_BOUND] = st == GST_OK ? (uint64_t)(c.best_full >> 32) : 0;
    out->device_ms = out->latency_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (st == GST_OK) {
      uint32_t ne = std::min<uint32_t>(c.n_edges, max_edges);
      int32_t m = out->edges ? std::min<int32_t>((int32_t)ne, out->max_edges) : 0;
      if (m > 0) CK(cudaMemcpy(out->edges, q.out_edges, (size_t)m * 12, cudaMemcpyDeviceToHost));
      if ((int64_t)c.n_edges > (int64_t)std::max(out->max_edges, 0) && out->edges) st = GST_TRUNCATED;
      if (c.n_edges > max_edges) st = GST_TRUNCATED;
      if (st == GST_OK && m == (int32_t)c.n_edges) {
        int64_t sum = 0;
        for (int32_t e = 0; e < m; e++) sum += out->edges[(size_t)e * 3 + 2];
        if (sum != out->cost) st = GST_INTERNAL;
      }
    }
  }
  return st;
}
