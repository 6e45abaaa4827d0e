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
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gstb.h"
#include "gst_device.cuh"

namespace gstb {
__global__ void k_work(const QDev*, const uint32_t*, const uint32_t*, int, uint32_t, GraphDev);
__global__ void k_split(const QDev*, const uint32_t*, const uint32_t*, int, uint32_t);
__global__ void k_sssp_seed(const QDev*, const uint32_t*, const uint32_t*, int, uint32_t);
__global__ void k_dp_seed(const QDev*, const uint32_t*, const uint32_t*, int, uint32_t);
__global__ void k_tour(const QDev*, const uint32_t*);
__global__ void k_extract(const QDev*, const uint32_t*, int, GraphDev);
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

static cudaError_t& last_cuda_error() {
  static thread_local cudaError_t e = cudaSuccess;
  return e;
}

struct gst_graph {
  uint32_t V = 0;
  uint64_t arcs = 0;
  uint32_t* d_beg = nullptr;
  uint2* d_adj = nullptr;
  // group index (host copy; member lists of a query are built on the host)
  std::vector<uint64_t> grp_ptr;
  std::vector<uint32_t> grp_v;
  int device = 0;
  int num_sms = 148;
};

namespace {

uint32_t env_u32(const char* name, uint32_t def) {
  const char* s = getenv(name);
  if (!s || !*s) return def;
  return (uint32_t)strtoul(s, nullptr, 10);
}

enum JobState { J_INIT, J_SSSP, J_TOUR, J_DPSEED, J_DP, J_EXTRACT, J_DONE };
enum Action { A_NONE, A_SSEED, A_WORK, A_SPLIT, A_TOUR, A_DSEED, A_EXTRACT };

struct Job {
  // request
  uint32_t groups[KMAX];
  int k = 0, D = -1;
  uint64_t tag = 0;
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
  JobState st = J_INIT;
  Action act = A_NONE;
  uint32_t delta = 1;
  gst_status status = GST_OK;
  bool rejected = false;      // failed validation before admission
  uint64_t rounds = 0;
  // results
  int32_t cost = -1;
  uint32_t root = 0;
  std::vector<uint32_t> edges;
  std::chrono::steady_clock::time_point t_submit, t_admit, t_done;
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Workspace layout of one query (see gst_device.cuh).
struct Layout {
  size_t table, dist, dflag, sflag, qbuf, tour, members, edges, total;
  uint32_t cap;
};

Layout layout_for(const gst_graph* g, int k, int nd, size_t n_members, uint32_t max_edges) {
  Layout L{};
  uint64_t WT = (uint64_t)(1u << k) * nd;
  uint64_t states = (uint64_t)g->V * WT;
  uint64_t caplim = env_u32("GSTB_QUEUE_CAP", 1u << 25);
  uint64_t cap = std::max<uint64_t>(std::min<uint64_t>(states, caplim), std::min<uint64_t>((uint64_t)g->V * k, caplim));
  cap = std::max<uint64_t>(cap, 1024);
  L.cap = (uint32_t)cap;
  size_t o = 0;
  L.table = o; o = align_up(o + states * 8, 256);
  L.dist = o; o = align_up(o + (size_t)g->V * 8 * 4, 256);
  L.dflag = o; o = align_up(o + ((states + 15) / 16) * 4, 256);
  L.sflag = o; o = align_up(o + (((size_t)g->V * 8 + 15) / 16) * 4, 256);
  L.qbuf = o; o = align_up(o + 4 * cap * 4, 256);
  L.tour = o; o = align_up(o + ((size_t)k * (1u << k) * k + (size_t)k * (1u << k)) * 4, 256);
  L.members = o; o = align_up(o + std::max<size_t>(n_members, 1) * 4, 256);
  L.edges = o; o = align_up(o + (size_t)std::max<uint32_t>(max_edges, 1) * 12, 256);
  L.total = o;
  return L;
}

// ---------------------------------------------------------------------------
// Round driver
// ---------------------------------------------------------------------------
class Runner {
 public:
  explicit Runner(gst_graph* g) : g_(g) {}
  ~Runner() { release(); }

  gst_status init() {
    CK(cudaSetDevice(g_->device));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, g_->device));
    uint64_t thr = ~0ull;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    delta_sssp_ = env_u32("GSTB_DELTA_SSSP", 4);
    delta_dp_ = env_u32("GSTB_DELTA_DP", 2);
    max_edges_dev_ = env_u32("GSTB_MAX_TREE_EDGES", 1u << 16);
    return GST_OK;
  }

  void release() {
    for (auto* j : active_) free_job(j);
    active_.clear();
    if (d_qd_) cudaFree(d_qd_);
    if (d_ctl_) cudaFree(d_ctl_);
    if (d_lists_) cudaFree(d_lists_);
    if (h_ctl_) cudaFreeHost(h_ctl_);
    if (h_qd_) cudaFreeHost(h_qd_);
    if (h_lists_) cudaFreeHost(h_lists_);
    if (stream_) cudaStreamDestroy(stream_);
    d_qd_ = nullptr;
    d_ctl_ = nullptr;
    d_lists_ = nullptr;
    h_ctl_ = nullptr;
    h_qd_ = nullptr;
    h_lists_ = nullptr;
    stream_ = nullptr;
  }

  // Prepare a job (validation, member list, sizes).  Does not allocate.
  gst_status prepare(Job* j) {
    if (j->k < 1 || j->k > KMAX) return GST_BAD_INPUT;
    if (j->D > DMAX) return GST_BAD_INPUT;
    const uint32_t ng = (uint32_t)(g_->grp_ptr.empty() ? 0 : g_->grp_ptr.size() - 1);
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
    Layout L = layout_for(g_, j->k, j->nd, j->members.size(), max_edges_dev_);
    j->table_bytes = (size_t)g_->V * j->WT * 8;
    j->bytes = L.total;
    return GST_OK;
  }

  // Allocate the workspace and queue the initial memsets; false if no memory.
  bool admit(Job* j) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, j->bytes, stream_) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    j->mem = (char*)p;
    Layout L = layout_for(g_, j->k, j->nd, j->members.size(), max_edges_dev_);
    QDev& q = j->qd;
    memset(&q, 0, sizeof(q));
    q.table = (unsigned long long*)(j->mem + L.table);
    q.dist = (uint32_t*)(j->mem + L.dist);
    q.dflag = (uint32_t*)(j->mem + L.dflag);
    q.sflag = (uint32_t*)(j->mem + L.sflag);
    for (int b = 0; b < 4; b++) q.qbuf[b] = (uint32_t*)(j->mem + L.qbuf) + (size_t)b * L.cap;
    q.tour = (uint32_t*)(j->mem + L.tour);
    q.members = (const uint32_t*)(j->mem + L.members);
    q.out_edges = (uint32_t*)(j->mem + L.edges);
    q.cap = L.cap;
    q.n_members = (uint32_t)j->members.size();
    q.max_edges = max_edges_dev_;
    q.k = j->k;
    q.D = j->D;
    q.nd = j->nd;
    q.full = (int)j->full;
    q.WT = j->WT;
    q.phase = PH_SSSP;
    q.in_idx = 0;
    q.out_idx = 1;
    q.far_idx = 2;
    q.far2_idx = 3;
    memset(&j->ctl, 0, sizeof(j->ctl));
    j->ctl.best = INF32;
    j->ctl.best_full = INF64;
    cudaMemsetAsync(q.table, 0xFF, (size_t)g_->V * j->WT * 8, stream_);
    cudaMemsetAsync(q.dist, 0xFF, (size_t)g_->V * 8 * 4, stream_);
    cudaMemsetAsync(q.dflag, 0, L.sflag - L.dflag, stream_);
    cudaMemsetAsync(q.sflag, 0, L.qbuf - L.sflag, stream_);
    cudaMemcpyAsync((void*)q.members, j->members.data(), j->members.size() * 4, cudaMemcpyHostToDevice,
                    stream_);
    j->st = J_INIT;
    j->t_admit = std::chrono::steady_clock::now();
    return true;
  }

  void free_job(Job* j) {
    if (j->mem) cudaFreeAsync(j->mem, stream_);
    j->mem = nullptr;
  }

  // Run rounds until every job in `jobs` is done.  `more` (optional) is
  // polled between rounds to admit new jobs (serving / batch admission).
  template <class AdmitFn>
  gst_status run(AdmitFn&& admit_more) {
    for (;;) {
      admit_more(active_);
      if (active_.empty()) return GST_OK;
      gst_status st = round();
      if (st != GST_OK) return st;
      // retire finished jobs
      std::vector<Job*> keep;
      for (Job* j : active_) {
        if (j->st == J_DONE) {
          free_job(j);
          finished_.push_back(j);
        } else {
          keep.push_back(j);
        }
      }
      active_.swap(keep);
    }
  }

  std::vector<Job*>& active() { return active_; }
  std::vector<Job*>& finished() { return finished_; }
  cudaStream_t stream() const { return stream_; }

 private:
  gst_status ensure_buffers(size_t nj, size_t list_words) {
    if (nj > cap_jobs_) {
      size_t n = std::max(nj, cap_jobs_ * 2 + 16);
      if (d_qd_) cudaFree(d_qd_);
      if (d_ctl_) cudaFree(d_ctl_);
      if (h_ctl_) cudaFreeHost(h_ctl_);
      if (h_qd_) cudaFreeHost(h_qd_);
      CK(cudaMalloc(&d_qd_, n * sizeof(QDev)));
      CK(cudaMalloc(&d_ctl_, n * sizeof(QCtl)));
      CK(cudaMallocHost(&h_ctl_, n * sizeof(QCtl)));
      CK(cudaMallocHost(&h_qd_, n * sizeof(QDev)));
      cap_jobs_ = n;
    }
    if (list_words > cap_lists_) {
      size_t n = std::max(list_words, cap_lists_ * 2 + 256);
      if (d_lists_) cudaFree(d_lists_);
      if (h_lists_) cudaFreeHost(h_lists_);
      CK(cudaMalloc(&d_lists_, n * 4));
      CK(cudaMallocHost(&h_lists_, n * 4));
      cap_lists_ = n;
    }
    return GST_OK;
  }

  // Decide this round's action for a job (host state machine).
  void decide(Job* j) {
    QDev& q = j->qd;
    QCtl& c = j->ctl;
    j->act = A_NONE;
    for (;;) {
      switch (j->st) {
        case J_INIT:
          q.phase = PH_SSSP;
          q.theta_lo = 0;
          q.theta_hi = delta_sssp_;
          j->delta = delta_sssp_;
          c.n_near = 0;
          j->act = A_SSEED;
          return;
        case J_SSSP:
        case J_DP: {
          if (q.n_in > 0) {
            c.n_near = 0;
            c.n_far = q.n_far;
            j->act = A_WORK;
            return;
          }
          uint32_t next_lo = q.theta_hi;
          bool exhausted = q.n_far == 0 || next_lo > c.best;
          if (!exhausted) {
            q.theta_lo = next_lo;
            q.theta_hi = next_lo + j->delta;
            c.n_near = 0;
            c.n_far2 = 0;
            j->act = A_SPLIT;
            return;
          }
          if (j->st == J_SSSP) {
            // every distance below theta_hi is exact, every distance <= best
            // was discovered; unknown ones are at least min(theta_hi, best+1)
            uint64_t b1 = c.best == INF32 ? (uint64_t)INF32 : (uint64_t)c.best + 1;
            uint64_t cap1 = std::min<uint64_t>(q.theta_hi, b1);
            if (q.n_far == 0) cap1 = b1;  // nothing pending: all reachable distances are final
            q.cap1 = (uint32_t)std::min<uint64_t>(cap1, BIG);
            j->st = J_TOUR;
            continue;
          }
          j->st = J_EXTRACT;
          continue;
        }
        case J_TOUR:
          j->act = A_TOUR;
          return;
        case J_DPSEED:
          q.phase = j->D < 0 ? PH_DP : PH_HOP;
          q.theta_lo = 0;
          q.theta_hi = delta_dp_;
          j->delta = delta_dp_;
          q.n_in = 0;
          q.n_far = 0;
          c.n_near = 0;
          c.n_far = 0;
          j->act = A_DSEED;
          return;
        case J_EXTRACT:
          j->act = A_EXTRACT;
          return;
        case J_DONE:
          return;
      }
    }
  }

  // Apply the effects of this round's action after the control blocks are back.
  void absorb(Job* j) {
    QDev& q = j->qd;
    QCtl& c = j->ctl;
    if (c.overflow) {
      j->status = GST_QUEUE_OVERFLOW;
      j->st = J_DONE;
      finish_timestamps(j);
      return;
    }
    switch (j->act) {
      case A_SSEED:
        std::swap(q.in_idx, q.out_idx);
        q.n_in = c.n_near;
        q.n_far = 0;
        j->st = J_SSSP;
        break;
      case A_WORK:
        std::swap(q.in_idx, q.out_idx);
        q.n_in = c.n_near;
        q.n_far = c.n_far;
        break;
      case A_SPLIT:
        std::swap(q.in_idx, q.out_idx);
        std::swap(q.far_idx, q.far2_idx);
        q.n_in = c.n_near;
        q.n_far = c.n_far2;
        break;
      case A_TOUR:
        j->st = J_DPSEED;
        break;
      case A_DSEED:
        std::swap(q.in_idx, q.out_idx);
        q.n_in = c.n_near;
        q.n_far = 0;
        j->st = J_DP;
        break;
      case A_EXTRACT:
        j->st = J_DONE;
        if (c.status == 1) {
          j->status = GST_NO_SOLUTION;
        } else if (c.status != 0) {
          j->status = GST_INTERNAL;
        } else {
          j->status = GST_OK;
          j->cost = (int32_t)(c.best_full >> 32);
          j->root = c.root;
        }
        break;
      default:
        break;
    }
    if (j->act != A_NONE) j->rounds++;
  }

  void finish_timestamps(Job* j) { j->t_done = std::chrono::steady_clock::now(); }

  gst_status round() {
    const size_t nj = active_.size();
    for (Job* j : active_) decide(j);
    // launch lists: for each action type, job slots + exclusive prefix of items
    std::vector<uint32_t> lists;
    struct L {
      size_t jobs_off = 0, pre_off = 0;
      int n = 0;
      uint32_t total = 0;
    };
    auto build = [&](Action a, auto items_of) {
      L l;
      std::vector<uint32_t> js, pre;
      uint32_t tot = 0;
      for (size_t i = 0; i < nj; i++) {
        Job* j = active_[i];
        if (j->act != a) continue;
        uint32_t n = items_of(j);
        js.push_back((uint32_t)i);
        pre.push_back(tot);
        tot += n;
      }
      pre.push_back(tot);
      l.n = (int)js.size();
      l.total = tot;
      l.jobs_off = lists.size();
      lists.insert(lists.end(), js.begin(), js.end());
      l.pre_off = lists.size();
      lists.insert(lists.end(), pre.begin(), pre.end());
      return l;
    };
    L lw = build(A_WORK, [](Job* j) { return j->qd.n_in; });
    L ls = build(A_SPLIT, [](Job* j) { return j->qd.n_far; });
    L lss = build(A_SSEED, [](Job* j) { return (uint32_t)j->members.size(); });
    L lds = build(A_DSEED, [](Job* j) { return (uint32_t)j->members.size(); });
    L lt = build(A_TOUR, [](Job*) { return 1u; });
    L le = build(A_EXTRACT, [](Job*) { return 1u; });
    gst_status st = ensure_buffers(nj, lists.size());
    if (st != GST_OK) return st;
    for (size_t i = 0; i < nj; i++) {
      active_[i]->qd.ctl = d_ctl_ + i;
      h_qd_[i] = active_[i]->qd;
      h_ctl_[i] = active_[i]->ctl;
    }
    memcpy(h_lists_, lists.data(), lists.size() * 4);
    CK(cudaMemcpyAsync(d_qd_, h_qd_, nj * sizeof(QDev), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(d_ctl_, h_ctl_, nj * sizeof(QCtl), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(d_lists_, h_lists_, lists.size() * 4, cudaMemcpyHostToDevice, stream_));
    GraphDev gd{g_->d_beg, g_->d_adj, g_->V};
    const uint32_t* D = d_lists_;
    auto grid_for = [&](uint64_t threads) {
      uint64_t b = (threads + 255) / 256;
      uint64_t maxb = (uint64_t)g_->num_sms * 8;
      return (unsigned)std::max<uint64_t>(1, std::min(b, maxb));
    };
    if (lss.n)
      k_sssp_seed<<<grid_for(lss.total), 256, 0, stream_>>>(d_qd_, D + lss.jobs_off, D + lss.pre_off, lss.n,
                                                           lss.total);
    if (lds.n)
      k_dp_seed<<<grid_for(lds.total), 256, 0, stream_>>>(d_qd_, D + lds.jobs_off, D + lds.pre_off, lds.n,
                                                         lds.total);
    if (ls.n && ls.total)
      k_split<<<grid_for(ls.total), 256, 0, stream_>>>(d_qd_, D + ls.jobs_off, D + ls.pre_off, ls.n, ls.total);
    if (lw.n && lw.total)
      k_work<<<grid_for((uint64_t)lw.total * 32), 256, 0, stream_>>>(d_qd_, D + lw.jobs_off, D + lw.pre_off,
                                                                     lw.n, lw.total, gd);
    if (lt.n) k_tour<<<lt.n, 256, 0, stream_>>>(d_qd_, D + lt.jobs_off);
    if (le.n) k_extract<<<(le.n + 63) / 64, 64, 0, stream_>>>(d_qd_, D + le.jobs_off, le.n, gd);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_ctl_, d_ctl_, nj * sizeof(QCtl), cudaMemcpyDeviceToHost, stream_));
    // tree edges of extracted jobs
    CK(cudaStreamSynchronize(stream_));
    for (size_t i = 0; i < nj; i++) active_[i]->ctl = h_ctl_[i];
    for (size_t i = 0; i < nj; i++) {
      Job* j = active_[i];
      if (j->act == A_EXTRACT && j->ctl.status == 0 && j->ctl.best_full != INF64) {
        uint32_t ne = std::min(j->ctl.n_edges, j->qd.max_edges);
        j->edges.resize((size_t)ne * 3);
        if (ne) CK(cudaMemcpyAsync(j->edges.data(), j->qd.out_edges, (size_t)ne * 12, cudaMemcpyDeviceToHost, stream_));
      }
    }
    CK(cudaStreamSynchronize(stream_));
    for (Job* j : active_) {
      absorb(j);
      if (j->st == J_DONE && j->t_done.time_since_epoch().count() == 0) finish_timestamps(j);
    }
    return GST_OK;
  }

  gst_graph* g_;
  cudaStream_t stream_ = nullptr;
  std::vector<Job*> active_, finished_;
  QDev* d_qd_ = nullptr;
  QCtl* d_ctl_ = nullptr;
  uint32_t* d_lists_ = nullptr;
  QDev* h_qd_ = nullptr;
  QCtl* h_ctl_ = nullptr;
  uint32_t* h_lists_ = nullptr;
  size_t cap_jobs_ = 0, cap_lists_ = 0;
  uint32_t delta_sssp_ = 4, delta_dp_ = 2, max_edges_dev_ = 1u << 16;
};

// Copy a finished job into a caller result.
gst_status fill_result(Job* j, gst_result* r) {
  if (!r) return j->status;
  r->cost = j->status == GST_OK ? j->cost : -1;
  r->root = j->root;
  for (int i = 0; i < GST_NSTATS; i++) r->stats[i] = j->ctl.stat[i];
  r->stats[GST_STAT_ROUNDS] = j->rounds;
  r->stats[GST_STAT_TABLE_BYTES] = j->table_bytes;
  r->device_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_admit).count();
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
  gst_graph* g = new gst_graph();
  g->V = V;
  g->arcs = arcs;
  cudaGetDevice(&g->device);
  cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device);
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
  g->grp_ptr.assign(grp_ptr, grp_ptr + n_groups + 1);
  g->grp_v.assign(grp_v, grp_v + n);
  return GST_OK;
}

void gst_graph_destroy(gst_graph* g) {
  if (!g) return;
  if (g->d_beg) cudaFree(g->d_beg);
  if (g->d_adj) cudaFree(g->d_adj);
  delete g;
}

uint32_t gst_graph_num_vertices(const gst_graph* g) { return g ? g->V : 0; }
uint64_t gst_graph_num_arcs(const gst_graph* g) { return g ? g->arcs : 0; }

gst_status gst_query(gst_graph* g, const uint32_t* groups, int k, int D, gst_result* out) {
  int32_t ks = k, Ds = D;
  int32_t st = 0;
  if (k < 1 || k > KMAX || !groups) return GST_BAD_INPUT;
  uint32_t gg[KMAX] = {0};
  memcpy(gg, groups, (size_t)k * 4);
  gst_status s = gst_query_batch(g, 1, gg, &ks, &Ds, out, &st, 1);
  if (s != GST_OK) return s;
  return (gst_status)st;
}

gst_status gst_query_batch(gst_graph* g, int n, const uint32_t* groups, const int32_t* ks, const int32_t* Ds,
                           gst_result* results, int32_t* statuses, int max_concurrent) {
  if (!g || n < 0 || (n > 0 && (!groups || !ks || !Ds || !statuses))) return GST_BAD_INPUT;
  if (g->grp_ptr.empty()) return GST_BAD_INPUT;
  Runner R(g);
  gst_status st = R.init();
  if (st != GST_OK) return st;
  std::vector<Job> jobs(n);
  std::deque<Job*> pending;
  for (int i = 0; i < n; i++) {
    Job& j = jobs[i];
    j.k = ks[i];
    j.D = Ds[i] < 0 ? -1 : Ds[i];
    j.tag = (uint64_t)i;
    j.res = results ? &results[i] : nullptr;
    if (j.k < 1 || j.k > KMAX) {
      statuses[i] = GST_BAD_INPUT;
      j.st = J_DONE;
      j.rejected = true;
      continue;
    }
    memcpy(j.groups, groups + (size_t)i * KMAX, (size_t)j.k * 4);
    j.t_submit = std::chrono::steady_clock::now();
    gst_status ps = R.prepare(&j);
    if (ps != GST_OK) {
      statuses[i] = ps;
      if (j.res) {
        j.res->cost = -1;
        j.res->n_edges = 0;
      }
      j.st = J_DONE;
      j.rejected = true;
      continue;
    }
    pending.push_back(&j);
  }
  const size_t maxc = max_concurrent > 0 ? (size_t)max_concurrent : (size_t)1 << 20;
  gst_status rs = R.run([&](std::vector<Job*>& act) {
    while (!pending.empty() && act.size() < maxc) {
      Job* j = pending.front();
      if (!R.admit(j)) {
        if (act.empty()) {  // cannot fit even alone
          j->status = GST_OOM;
          j->st = J_DONE;
          pending.pop_front();
          continue;
        }
        break;
      }
      pending.pop_front();
      act.push_back(j);
    }
  });
  if (rs != GST_OK) return rs;
  for (int i = 0; i < n; i++) {
    Job& j = jobs[i];
    if (j.rejected) continue;
    statuses[i] = fill_result(&j, j.res);
  }
  return GST_OK;
}

}  // extern "C"
