// ORACLE -- test infrastructure only.  Nothing in the product links this file;
// only tests/, the smoke check and bench.py's CPU-baseline leg load it, as the
// checker.  It is a CPU restatement of the reference's exact group Steiner tree
// algorithms, written from the reference's source:
//
//   prunedpp()  PrunedDP++ (Li et al. SIGMOD'16) as in
//               code/PrunedDP++/include/CPUNONHOP.h:499-992 (main loop),
//               :21-80 (SPs to groups), :175-210 (virtual distances),
//               :269-386 (AllPaths W), :567-587 (W2), :436-496 (LB),
//               :390-432 (build_tree), with the one-label feasible solution
//               post-processed by an MST (graph_hash_of_mixed_weighted_MST_
//               postprocessing.h:10-35).  `ratio` is the reference's
//               maximum_return_app_ratio; ratio = 0 disables the progressive
//               exit (integer division at CPUNONHOP.h:733-735), leaving only the
//               exact exits.
//   hop()       HOP_cpu, code/D-PrunedDP++/include/CPUHOP.h:107-288 (Dijkstra
//               over (v,p,d); grow d->d+1 while d<D; merge complements with
//               d2 <= D-d1 into max(d1,d2); stop at the first popped full set).
//   dpbf()      plain DPBF (Dijkstra over (v,p), no pruning): an independent
//               exact cross-check for prunedpp().
//   brute()     minimum over all edge subsets that form a tree (tiny graphs).
//   validate()  tree checks: edges exist with their weights, connected, acyclic,
//               covers every query group, weights sum to the cost, hop diameter
//               <= D (feasibility check of exp_CPU_nonHop.h:17-48 plus the
//               weight-sum and diameter checks the reference lacks).
//
// Parity is pinned by cross-agreement: prunedpp(ratio 0) == dpbf() == brute()
// on small cases, and the reference's own PrunedDP++ / HOP_cpu sources compiled
// in oracle/_ref (see oracle/Makefile) agree with prunedpp()/hop().

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <functional>
#include <numeric>
#include <queue>
#include <unordered_map>
#include <vector>

namespace {

const int INF = 100000;  // the reference's sentinel (CPUNONHOP.h:14, DPQ.cuh:50)

struct Csr {
  uint32_t V;
  const uint32_t* beg;
  const uint32_t* adj;
  const int32_t* w;
};

struct Query {
  int k;
  std::vector<std::vector<uint32_t>> groups;  // member lists
  std::vector<uint32_t> mask;                  // per-vertex membership mask
};

Query make_query(const Csr& g, int k, const uint64_t* qptr, const uint32_t* qv) {
  Query q;
  q.k = k;
  q.groups.resize(k);
  q.mask.assign(g.V, 0);
  for (int j = 0; j < k; j++) {
    for (uint64_t t = qptr[j]; t < qptr[j + 1]; t++) {
      q.groups[j].push_back(qv[t]);
      q.mask[qv[t]] |= 1u << j;
    }
  }
  return q;
}

int edge_weight(const Csr& g, uint32_t a, uint32_t b) {
  const uint32_t* lo = g.adj + g.beg[a];
  const uint32_t* hi = g.adj + g.beg[a + 1];
  const uint32_t* it = std::lower_bound(lo, hi, b);
  if (it == hi || *it != b) return -1;
  return g.w[it - g.adj];
}

// Multi-source Dijkstra from all members of one group (the dummy-vertex
// construction of CPUNONHOP.h:21-67); predecessor of a member is itself.
void group_sssp(const Csr& g, const std::vector<uint32_t>& src, std::vector<int>& dist,
                std::vector<uint32_t>& pred) {
  dist.assign(g.V, INF);
  pred.resize(g.V);
  std::iota(pred.begin(), pred.end(), 0u);
  typedef std::pair<int, uint32_t> E;
  std::priority_queue<E, std::vector<E>, std::greater<E>> pq;
  for (uint32_t s : src) {
    if (dist[s] != 0) {
      dist[s] = 0;
      pq.push({0, s});
    }
  }
  std::vector<char> done(g.V, 0);
  while (!pq.empty()) {
    E e = pq.top();
    pq.pop();
    uint32_t v = e.second;
    if (done[v] || e.first != dist[v]) continue;
    done[v] = 1;
    for (uint32_t a = g.beg[v]; a < g.beg[v + 1]; a++) {
      uint32_t u = g.adj[a];
      int nd = e.first + g.w[a];
      if (nd < dist[u]) {
        dist[u] = nd;
        pred[u] = v;
        pq.push({nd, u});
      }
    }
  }
}

// Kruskal MST weight of an edge multiset (duplicates collapse).
struct Edge3 {
  uint32_t a, b;
  int w;
};

int mst_weight(std::vector<Edge3> es) {
  for (auto& e : es)
    if (e.a > e.b) std::swap(e.a, e.b);
  std::sort(es.begin(), es.end(), [](const Edge3& x, const Edge3& y) {
    if (x.a != y.a) return x.a < y.a;
    if (x.b != y.b) return x.b < y.b;
    return x.w < y.w;
  });
  es.erase(std::unique(es.begin(), es.end(),
                       [](const Edge3& x, const Edge3& y) { return x.a == y.a && x.b == y.b; }),
           es.end());
  std::vector<uint32_t> vs;
  for (auto& e : es) {
    vs.push_back(e.a);
    vs.push_back(e.b);
  }
  std::sort(vs.begin(), vs.end());
  vs.erase(std::unique(vs.begin(), vs.end()), vs.end());
  std::vector<int> par(vs.size());
  std::iota(par.begin(), par.end(), 0);
  std::function<int(int)> find = [&](int x) { return par[x] == x ? x : par[x] = find(par[x]); };
  std::stable_sort(es.begin(), es.end(), [](const Edge3& x, const Edge3& y) { return x.w < y.w; });
  int tot = 0;
  for (auto& e : es) {
    int a = std::lower_bound(vs.begin(), vs.end(), e.a) - vs.begin();
    int b = std::lower_bound(vs.begin(), vs.end(), e.b) - vs.begin();
    a = find(a);
    b = find(b);
    if (a != b) {
      par[a] = b;
      tot += e.w;
    }
  }
  return tot;
}

// DP table entry shared by the restatements.
struct TNode {
  int cost;
  int8_t type;  // 0 seed, 1 grow, 2 merge
  uint32_t u;   // grow predecessor vertex
  int p1, p2;   // merge parts
  int d1, d2;   // merge depths (hop variant)
};

void emit_edges(const std::vector<Edge3>& es, int32_t* n_edges, uint32_t* edges, int max_edges) {
  // dedupe, then write (u, v, w) triples
  std::vector<Edge3> t = es;
  for (auto& e : t)
    if (e.a > e.b) std::swap(e.a, e.b);
  std::sort(t.begin(), t.end(), [](const Edge3& x, const Edge3& y) {
    return x.a != y.a ? x.a < y.a : x.b < y.b;
  });
  t.erase(std::unique(t.begin(), t.end(),
                      [](const Edge3& x, const Edge3& y) { return x.a == y.a && x.b == y.b; }),
          t.end());
  *n_edges = (int32_t)t.size();
  for (size_t i = 0; i < t.size() && (int)i < max_edges; i++) {
    edges[3 * i] = t[i].a;
    edges[3 * i + 1] = t[i].b;
    edges[3 * i + 2] = (uint32_t)t[i].w;
  }
}

// ---------------------------------------------------------------------------
// PrunedDP++ restatement (CPUNONHOP.h:499-992)
// ---------------------------------------------------------------------------
struct PrunedDP {
  const Csr& g;
  const Query& q;
  int k, full, W_;  // W_ = 2^k
  std::vector<std::vector<int>> sp_dist;
  std::vector<std::vector<uint32_t>> sp_pred;
  std::vector<int> Wt;   // W[i][j][X] flattened (i*k + j)*W_ + X
  std::vector<int> W2;   // W2[i][X]
  std::vector<TNode> tree;
  std::vector<char> has, popped;
  std::vector<int> inq;  // priority in queue, INT_MAX if absent
  std::vector<std::vector<int>> nonover;  // CPUNONHOP.h:115-141
  std::vector<std::vector<int>> uncovered;
  int64_t process = 0;

  PrunedDP(const Csr& g_, const Query& q_) : g(g_), q(q_) {
    k = q.k;
    W_ = 1 << k;
    full = W_ - 1;
  }

  TNode& T(uint32_t v, int p) { return tree[(size_t)v * W_ + p]; }

  // AllPaths (CPUNONHOP.h:269-386): Dijkstra over (vi, vj, X) from (i, i, 0);
  // a pop lowers W of every subset of X (the "subset" rule at :320-338).
  void all_paths(const std::vector<std::vector<int>>& vd) {
    Wt.assign((size_t)k * k * W_, INT32_MAX);
    std::vector<int> best((size_t)k * k * W_, INT32_MAX);
    std::vector<char> done((size_t)k * k * W_, 0);
    typedef std::pair<int, int> E;  // (cost, key)
    std::priority_queue<E, std::vector<E>, std::greater<E>> pq;
    auto key = [&](int i, int j, int X) { return (i * k + j) * W_ + X; };
    for (int i = 0; i < k; i++) {
      best[key(i, i, 0)] = 0;
      pq.push({0, key(i, i, 0)});
    }
    while (!pq.empty()) {
      E e = pq.top();
      pq.pop();
      int kk = e.second;
      if (done[kk] || e.first != best[kk]) continue;
      done[kk] = 1;
      int X = kk % W_, ij = kk / W_, i = ij / k, j = ij % k;
      int cost = e.first;
      Wt[kk] = std::min(Wt[kk], cost);
      for (int s = 0; s < X; s++)
        if ((s | X) == X) Wt[key(i, j, s)] = std::min(Wt[key(i, j, s)], cost);
      for (int p = 0; p < k; p++) {
        int pb = 1 << p;
        if ((pb | X) == X) continue;
        int nk = key(i, p, X + pb);
        if (done[nk]) continue;
        int c = cost + vd[j][p];
        if (c < best[nk]) {
          best[nk] = c;
          pq.push({c, nk});
        }
      }
    }
    // the reference reads absent keys through operator[] (value 0)
    for (auto& x : Wt)
      if (x == INT32_MAX) x = 0;
    W2.assign((size_t)k * W_, INF);
    for (int i = 0; i < k; i++)
      for (int X = 1; X <= full; X++) {
        int dis = INF;
        for (int j = 0; j < k; j++) dis = std::min(dis, Wt[key(i, j, X)]);
        W2[i * W_ + X] = dis;
      }
  }

  // LB_procedure (CPUNONHOP.h:436-496)
  int lb(uint32_t v, int X, int cost) {
    int lbv = 0;
    if (X != full) {
      int Xs = full - X;
      int lb1 = INF, lb2 = -1, lb_one = -1;
      for (int i : uncovered[X]) {
        int dvi = sp_dist[i][v];
        int xxx = INF;
        for (int j : uncovered[X]) {
          int dvj = sp_dist[j][v];
          if (xxx > dvj) xxx = dvj;
          int l1 = (dvi + Wt[(i * k + j) * W_ + Xs] + dvj) / 2;
          if (lb1 > l1) lb1 = l1;
        }
        int l2 = (dvi + W2[i * W_ + Xs] + xxx) / 2;
        if (lb2 < l2) lb2 = l2;
        if (lb_one < dvi) lb_one = dvi;
      }
      lbv = lb1 < lb2 ? lb2 : lb1;
      if (lbv < lb_one) lbv = lb_one;
    }
    return cost + lbv;
  }

  // build_tree (CPUNONHOP.h:390-432)
  void build_tree(uint32_t root, int rp, std::vector<Edge3>& out, std::vector<uint32_t>* verts) {
    std::queue<std::pair<uint32_t, int>> wq;
    wq.push({root, rp});
    while (!wq.empty()) {
      auto pr = wq.front();
      wq.pop();
      if (verts) verts->push_back(pr.first);
      TNode& n = T(pr.first, pr.second);
      if (n.type == 1) {
        wq.push({n.u, pr.second});
        out.push_back({n.u, pr.first, edge_weight(g, n.u, pr.first)});
      } else if (n.type == 2) {
        wq.push({pr.first, n.p1});
        wq.push({pr.first, n.p2});
      }
    }
  }

  int run(int ratio, int32_t* cost_out, uint32_t* root_out, int32_t* n_edges, uint32_t* edges,
          int max_edges, int64_t* stats) {
    sp_dist.resize(k);
    sp_pred.resize(k);
    for (int j = 0; j < k; j++) group_sssp(g, q.groups[j], sp_dist[j], sp_pred[j]);
    nonover.assign(W_, {});
    for (int i = 1; i <= full; i++)
      for (int j = 1; j < full; j++)
        if ((i & j) == 0) nonover[i].push_back(j);
    uncovered.assign(W_, {});
    for (int p = 1; p <= full; p++)
      for (int j = 0; j < k; j++)
        if (!(p >> j & 1)) uncovered[p].push_back(j);
    std::vector<std::vector<int>> vd(k, std::vector<int>(k, INF));  // :175-210
    for (int a = 0; a < k; a++)
      for (int b = 0; b < k; b++)
        for (uint32_t v : q.groups[b]) vd[a][b] = std::min(vd[a][b], sp_dist[a][v]);
    all_paths(vd);

    size_t NS = (size_t)g.V * W_;
    tree.assign(NS, TNode{INF, 0, 0, 0, 0, 0, 0});
    has.assign(NS, 0);
    popped.assign(NS, 0);
    inq.assign(NS, INT32_MAX);
    typedef std::pair<int, uint32_t> QE;  // (priority, state)
    std::priority_queue<QE, std::vector<QE>, std::greater<QE>> Q;
    auto push = [&](uint32_t v, int p, int pri) {
      size_t s = (size_t)v * W_ + p;
      if (inq[s] == INT32_MAX || pri < inq[s]) {
        inq[s] = pri;
        Q.push({pri, (uint32_t)s});
      }
    };
    for (uint32_t v = 0; v < g.V; v++) {  // :596-624
      uint32_t m = q.mask[v];
      for (uint32_t p = 1; p <= m; p++)
        if ((p | m) == m) {
          T(v, p) = TNode{0, 0, 0, 0, 0, 0, 0};
          has[(size_t)v * W_ + p] = 1;
          push(v, p, 0);
        }
    }
    const int safeguard = 2;
    int best_cost = INF;
    std::vector<Edge3> best_solu;
    uint32_t best_root = 0;
    bool best_is_dp = false;

    auto finish_tree = [&](uint32_t v, int p, int cost_value) {
      std::vector<Edge3> es;
      build_tree(v, p, es, nullptr);
      *cost_out = cost_value;
      *root_out = v;
      emit_edges(es, n_edges, edges, max_edges);
    };

    while (!Q.empty()) {  // :635
      QE top = Q.top();
      Q.pop();
      size_t s = top.second;
      if (popped[s] || inq[s] != top.first) continue;  // stale duplicate
      inq[s] = INT32_MAX;
      process++;
      uint32_t v = (uint32_t)(s / W_);
      int X = (int)(s % W_);
      int cost = T(v, X).cost;
      if (X == full) {  // :658-678 exact exit
        stats[0] = process;
        finish_tree(v, X, cost);
        return 0;
      }
      popped[s] = 1;
      // one-label feasible solution (:684-726)
      int feas = cost;
      for (int j : uncovered[X]) {
        if (sp_dist[j][v] == INF) {
          feas = INF;
          break;
        }
        feas += sp_dist[j][v];
      }
      if (feas < best_cost) {
        std::vector<Edge3> sol;
        build_tree(v, X, sol, nullptr);
        for (int j : uncovered[X]) {
          uint32_t a = v, pre = sp_pred[j][a];
          while (a != pre) {
            sol.push_back({a, pre, edge_weight(g, a, pre)});
            a = pre;
            pre = sp_pred[j][a];
          }
        }
        best_cost = mst_weight(sol);
        best_solu = sol;
        best_root = v;
        best_is_dp = false;
      }
      // progressive exit (:730-755)
      if (cost > 0) {
        int r = best_cost / cost;
        if (r <= ratio + 1e-5) {
          stats[0] = process;
          *cost_out = best_cost;
          *root_out = best_root;
          if (best_is_dp) {
            emit_edges(best_solu, n_edges, edges, max_edges);
          } else {
            // MST of the feasible union, as the reference post-processes it
            std::vector<Edge3> t = best_solu;
            for (auto& e : t)
              if (e.a > e.b) std::swap(e.a, e.b);
            std::stable_sort(t.begin(), t.end(),
                             [](const Edge3& x, const Edge3& y) { return x.w < y.w; });
            std::vector<uint32_t> vs;
            for (auto& e : t) {
              vs.push_back(e.a);
              vs.push_back(e.b);
            }
            std::sort(vs.begin(), vs.end());
            vs.erase(std::unique(vs.begin(), vs.end()), vs.end());
            std::vector<int> par(vs.size());
            std::iota(par.begin(), par.end(), 0);
            std::function<int(int)> find = [&](int x) {
              return par[x] == x ? x : par[x] = find(par[x]);
            };
            std::vector<Edge3> mst;
            for (auto& e : t) {
              int a = find(std::lower_bound(vs.begin(), vs.end(), e.a) - vs.begin());
              int b = find(std::lower_bound(vs.begin(), vs.end(), e.b) - vs.begin());
              if (a != b) {
                par[a] = b;
                mst.push_back(e);
              }
            }
            emit_edges(mst, n_edges, edges, max_edges);
          }
          return 0;
        }
      }
      // complement merge (:758-817)
      int Xs = full - X;
      if (popped[(size_t)v * W_ + Xs]) {
        int merged = cost + T(v, Xs).cost;
        int cur = has[(size_t)v * W_ + full] ? T(v, full).cost : INF;
        if (merged < cur) {
          T(v, full) = TNode{merged, 2, 0, X, Xs, 0, 0};
          has[(size_t)v * W_ + full] = 1;
          if (!(merged > best_cost + safeguard)) {
            if (merged < best_cost) {
              best_cost = merged;
              best_solu.clear();
              build_tree(v, full, best_solu, nullptr);
              best_root = v;
              best_is_dp = true;
            }
            push(v, full, merged);
          }
        }
        continue;
      }
      if (cost < best_cost / 2 + safeguard) {  // :820
        for (uint32_t a = g.beg[v]; a < g.beg[v + 1]; a++) {  // grow :826-894
          uint32_t u = g.adj[a];
          int gc = cost + g.w[a];
          size_t su = (size_t)u * W_ + X;
          if (popped[su]) continue;
          int tup = has[su] ? tree[su].cost : INF;
          if (gc < tup) {
            tree[su] = TNode{gc, 1, v, 0, 0, 0, 0};
            has[su] = 1;
            int l = lb(u, X, gc);
            if (l > best_cost + safeguard) continue;
            push(u, X, gc);
          }
        }
        for (int p2 : nonover[X]) {  // merge :899-983
          if (!popped[(size_t)v * W_ + p2]) continue;
          int pu = X + p2;
          size_t sm = (size_t)v * W_ + pu;
          if (popped[sm]) continue;
          int merged = cost + T(v, p2).cost;
          int cur = has[sm] ? tree[sm].cost : INF;
          if (merged < cur) {
            tree[sm] = TNode{merged, 2, 0, X, p2, 0, 0};
            has[sm] = 1;
            if (merged <= best_cost * 0.667 + safeguard) {
              int l = lb(v, pu, merged);
              if (l > best_cost + safeguard) continue;
              if (pu == full && merged < best_cost) {
                best_cost = merged;
                best_solu.clear();
                build_tree(v, full, best_solu, nullptr);
                best_root = v;
                best_is_dp = true;
              }
              push(v, pu, merged);
            }
          }
        }
      }
    }
    stats[0] = process;
    *cost_out = -1;
    *n_edges = 0;
    return 1;  // no feasible solution (:987)
  }
};

// Cheapest path from group j to v with at most b hops, b = 0..D (synchronous
// Bellman-Ford rounds), as hd[(b * k + j) * V + v]; HD_INF if none.
const int32_t HD_INF = 0x3FFFFFFF;
std::vector<int32_t> hop_limited_distances(const Csr& g, const Query& q, int D) {
  const size_t V = g.V;
  std::vector<int32_t> hd((size_t)(D + 1) * q.k * V, HD_INF);
  for (int j = 0; j < q.k; j++)
    for (uint32_t m : q.groups[j]) hd[(size_t)j * V + m] = 0;
  for (int b = 1; b <= D; b++)
    for (int j = 0; j < q.k; j++) {
      const int32_t* prev = &hd[((size_t)(b - 1) * q.k + j) * V];
      int32_t* cur = &hd[((size_t)b * q.k + j) * V];
      std::copy(prev, prev + V, cur);
      for (uint32_t u = 0; u < g.V; u++) {
        if (prev[u] >= HD_INF) continue;
        for (uint32_t a = g.beg[u]; a < g.beg[u + 1]; a++)
          cur[g.adj[a]] = std::min(cur[g.adj[a]], prev[u] + g.w[a]);
      }
    }
  return hd;
}

// ---------------------------------------------------------------------------
// HOP_cpu restatement (CPUHOP.h:107-288).  With `hd` (the hop-limited
// distances) it also applies the GPU engine's hop-budget bound at pop time,
// against the upper bound `ub`: a state (v, p, d) is dropped when a group
// missing from p has no member within D - d hops of v, or when its cost plus
// the largest such distance exceeds ub.  This variant is test infrastructure
// for that bound's exactness.
// ---------------------------------------------------------------------------
int run_hop(const Csr& g, const Query& q, int D, int32_t* cost_out, uint32_t* root_out,
            int32_t* n_edges, uint32_t* edges, int max_edges, int64_t* stats,
            const std::vector<int32_t>* hd = nullptr, int64_t ub = INT64_MAX) {
  int k = q.k, W_ = 1 << k, full = W_ - 1, DD = D + 1;
  size_t NS = (size_t)g.V * W_ * DD;
  std::vector<TNode> t(NS, TNode{INF, 0, 0, 0, 0, 0, 0});
  auto at = [&](uint32_t v, int p, int d) -> TNode& { return t[((size_t)v * W_ + p) * DD + d]; };
  std::vector<std::vector<int>> nonover(W_ + 1);  // :84-105
  for (int i = 1; i <= full; i++)
    for (int j = 1; j <= full; j++)
      if ((i & j) == 0) nonover[i].push_back(j);
  struct QE {
    int v, p, d, cost;
    bool operator>(const QE& o) const { return cost > o.cost; }
  };
  std::priority_queue<QE, std::vector<QE>, std::greater<QE>> pq;
  for (uint32_t v = 0; v < g.V; v++)  // :158-170 singletons only
    for (int i = 1; i <= (int)q.mask[v]; i <<= 1)
      if (i & q.mask[v]) {
        at(v, i, 0).cost = 0;
        at(v, i, 0).type = 0;
        pq.push(QE{(int)v, i, 0, 0});
      }
  int64_t process = 0;
  bool found = false;
  QE fin{0, 0, 0, 0};
  while (!pq.empty()) {  // :174-228
    process++;
    QE e = pq.top();
    pq.pop();
    if (e.cost != at(e.v, e.p, e.d).cost) continue;
    if (e.p == full) {
      fin = e;
      found = true;
      break;
    }
    if (hd) {
      int64_t lb = 0;
      bool reach = true;
      const int b = D - e.d;
      for (int j = 0; j < k; j++)
        if (!((e.p >> j) & 1)) {
          const int32_t x = (*hd)[((size_t)b * k + j) * g.V + e.v];
          if (x >= HD_INF) reach = false;
          lb = std::max<int64_t>(lb, x);
        }
      if (!reach || e.cost + lb > ub) continue;
    }
    if (e.d < D) {
      for (uint32_t a = g.beg[e.v]; a < g.beg[e.v + 1]; a++) {
        uint32_t u = g.adj[a];
        int c = e.cost + g.w[a];
        TNode& n = at(u, e.p, e.d + 1);
        if (n.cost > c) {
          n.cost = c;
          n.type = 1;
          n.u = e.v;
          pq.push(QE{(int)u, e.p, e.d + 1, c});
        }
      }
    }
    for (int p2 : nonover[e.p])
      for (int d2 = 0; d2 <= D - e.d; d2++) {
        int pu = e.p | p2, nd = std::max(e.d, d2);
        int mc = e.cost + at(e.v, p2, d2).cost;
        TNode& n = at(e.v, pu, nd);
        if (n.cost > mc) {
          n = TNode{mc, 2, 0, e.p, p2, e.d, d2};
          pq.push(QE{e.v, pu, nd, mc});
        }
      }
  }
  stats[0] = process;
  if (!found) {
    *cost_out = -1;
    *n_edges = 0;
    return 1;
  }
  std::vector<Edge3> es;  // extraction :234-259
  std::queue<QE> wq;
  wq.push(fin);
  while (!wq.empty()) {
    QE e = wq.front();
    wq.pop();
    TNode& n = at(e.v, e.p, e.d);
    if (n.type == 1) {
      es.push_back({n.u, (uint32_t)e.v, edge_weight(g, n.u, e.v)});
      wq.push(QE{(int)n.u, e.p, e.d - 1, 0});
    } else if (n.type == 2) {
      wq.push(QE{e.v, n.p1, n.d1, 0});
      wq.push(QE{e.v, n.p2, n.d2, 0});
    }
  }
  *cost_out = fin.cost;
  *root_out = fin.v;
  emit_edges(es, n_edges, edges, max_edges);
  return 0;
}

// ---------------------------------------------------------------------------
// Plain DPBF: Dijkstra over (v,p), grow + merge with settled partners, no
// pruning.  Independent of PrunedDP++'s gates.
// ---------------------------------------------------------------------------
int run_dpbf(const Csr& g, const Query& q, int32_t* cost_out, uint32_t* root_out, int32_t* n_edges,
             uint32_t* edges, int max_edges, int64_t* stats) {
  int k = q.k, W_ = 1 << k, full = W_ - 1;
  size_t NS = (size_t)g.V * W_;
  std::vector<TNode> t(NS, TNode{INF, 0, 0, 0, 0, 0, 0});
  std::vector<char> done(NS, 0);
  typedef std::pair<int, uint32_t> QE;
  std::priority_queue<QE, std::vector<QE>, std::greater<QE>> pq;
  for (uint32_t v = 0; v < g.V; v++) {
    uint32_t m = q.mask[v];
    for (uint32_t p = 1; p <= m; p++)
      if ((p | m) == m) {
        t[(size_t)v * W_ + p].cost = 0;
        pq.push({0, (uint32_t)((size_t)v * W_ + p)});
      }
  }
  int64_t process = 0;
  while (!pq.empty()) {
    QE e = pq.top();
    pq.pop();
    size_t s = e.second;
    if (done[s] || e.first != t[s].cost) continue;
    done[s] = 1;
    process++;
    uint32_t v = (uint32_t)(s / W_);
    int p = (int)(s % W_);
    int c = e.first;
    if (p == full) {
      stats[0] = process;
      std::vector<Edge3> es;
      std::vector<std::pair<uint32_t, int>> st{{v, p}};
      while (!st.empty()) {
        auto pr = st.back();
        st.pop_back();
        TNode& n = t[(size_t)pr.first * W_ + pr.second];
        if (n.type == 1) {
          es.push_back({n.u, pr.first, edge_weight(g, n.u, pr.first)});
          st.push_back({n.u, pr.second});
        } else if (n.type == 2) {
          st.push_back({pr.first, n.p1});
          st.push_back({pr.first, n.p2});
        }
      }
      *cost_out = c;
      *root_out = v;
      emit_edges(es, n_edges, edges, max_edges);
      return 0;
    }
    for (uint32_t a = g.beg[v]; a < g.beg[v + 1]; a++) {
      size_t su = (size_t)g.adj[a] * W_ + p;
      int nc = c + g.w[a];
      if (!done[su] && nc < t[su].cost) {
        t[su] = TNode{nc, 1, v, 0, 0, 0, 0};
        pq.push({nc, (uint32_t)su});
      }
    }
    int comp = full ^ p;
    for (int p2 = comp; p2 > 0; p2 = (p2 - 1) & comp) {
      size_t s2 = (size_t)v * W_ + p2;
      if (!done[s2]) continue;
      size_t sm = (size_t)v * W_ + (p | p2);
      int mc = c + t[s2].cost;
      if (!done[sm] && mc < t[sm].cost) {
        t[sm] = TNode{mc, 2, 0, p, p2, 0, 0};
        pq.push({mc, (uint32_t)sm});
      }
    }
  }
  stats[0] = process;
  *cost_out = -1;
  *n_edges = 0;
  return 1;
}

// hop diameter of a tree given as an edge list (BFS twice); -1 if not a tree
int tree_diameter(const std::vector<Edge3>& es, uint32_t root) {
  std::vector<uint32_t> vs{root};
  for (auto& e : es) {
    vs.push_back(e.a);
    vs.push_back(e.b);
  }
  std::sort(vs.begin(), vs.end());
  vs.erase(std::unique(vs.begin(), vs.end()), vs.end());
  int n = (int)vs.size();
  std::vector<std::vector<int>> adj(n);
  for (auto& e : es) {
    int a = std::lower_bound(vs.begin(), vs.end(), e.a) - vs.begin();
    int b = std::lower_bound(vs.begin(), vs.end(), e.b) - vs.begin();
    adj[a].push_back(b);
    adj[b].push_back(a);
  }
  auto bfs = [&](int s, int& far) {
    std::vector<int> d(n, -1);
    std::queue<int> qq;
    d[s] = 0;
    qq.push(s);
    far = s;
    while (!qq.empty()) {
      int x = qq.front();
      qq.pop();
      if (d[x] > d[far]) far = x;
      for (int y : adj[x])
        if (d[y] < 0) {
          d[y] = d[x] + 1;
          qq.push(y);
        }
    }
    for (int i = 0; i < n; i++)
      if (d[i] < 0) return -1;
    return d[far];
  };
  int far;
  if (bfs(0, far) < 0) return -1;
  int far2;
  return bfs(far, far2);
}

}  // namespace

extern "C" {

// Status codes: 0 = ok, 1 = no solution, 2 = bad input.
int oracle_prunedpp(uint32_t V, const uint32_t* beg, const uint32_t* adj, const int32_t* w, int k,
                    const uint64_t* qptr, const uint32_t* qv, int ratio, int32_t* cost,
                    uint32_t* root, int32_t* n_edges, uint32_t* edges, int max_edges,
                    int64_t* stats) {
  if (k < 1 || k > 14) return 2;
  Csr g{V, beg, adj, w};
  Query q = make_query(g, k, qptr, qv);
  PrunedDP p(g, q);
  return p.run(ratio, cost, root, n_edges, edges, max_edges, stats);
}

int oracle_hop(uint32_t V, const uint32_t* beg, const uint32_t* adj, const int32_t* w, int k,
               const uint64_t* qptr, const uint32_t* qv, int D, int32_t* cost, uint32_t* root,
               int32_t* n_edges, uint32_t* edges, int max_edges, int64_t* stats) {
  if (k < 1 || k > 14 || D < 0) return 2;
  Csr g{V, beg, adj, w};
  Query q = make_query(g, k, qptr, qv);
  return run_hop(g, q, D, cost, root, n_edges, edges, max_edges, stats);
}

// HOP_cpu with the hop-budget bound against the upper bound ub (see run_hop).
int oracle_hop_budget(uint32_t V, const uint32_t* beg, const uint32_t* adj, const int32_t* w, int k,
                      const uint64_t* qptr, const uint32_t* qv, int D, int64_t ub, int32_t* cost,
                      int64_t* stats) {
  if (k < 1 || k > 14 || D < 0) return 2;
  Csr g{V, beg, adj, w};
  Query q = make_query(g, k, qptr, qv);
  std::vector<int32_t> hd = hop_limited_distances(g, q, D);
  uint32_t root = 0;
  int32_t ne = 0;
  return run_hop(g, q, D, cost, &root, &ne, nullptr, 0, stats, &hd, ub);
}

int oracle_dpbf(uint32_t V, const uint32_t* beg, const uint32_t* adj, const int32_t* w, int k,
                const uint64_t* qptr, const uint32_t* qv, int32_t* cost, uint32_t* root,
                int32_t* n_edges, uint32_t* edges, int max_edges, int64_t* stats) {
  if (k < 1 || k > 14) return 2;
  Csr g{V, beg, adj, w};
  Query q = make_query(g, k, qptr, qv);
  return run_dpbf(g, q, cost, root, n_edges, edges, max_edges, stats);
}

// Minimum-cost tree over all edge subsets (E <= 22), with hop diameter <= D
// when D >= 0.  A single vertex in every group is a tree of cost 0.
int oracle_brute(uint32_t V, const uint32_t* beg, const uint32_t* adj, const int32_t* w, int k,
                 const uint64_t* qptr, const uint32_t* qv, int D, int32_t* cost) {
  Csr g{V, beg, adj, w};
  Query q = make_query(g, k, qptr, qv);
  uint32_t full = (1u << k) - 1;
  std::vector<Edge3> E;
  for (uint32_t v = 0; v < V; v++)
    for (uint32_t a = beg[v]; a < beg[v + 1]; a++)
      if (v < adj[a]) E.push_back({v, adj[a], w[a]});
  if (E.size() > 22) return 2;
  int bestc = INT32_MAX;
  for (uint32_t v = 0; v < V; v++)
    if (q.mask[v] == full) bestc = 0;
  std::vector<int> par(V);
  std::function<int(int)> find = [&](int x) { return par[x] == x ? x : par[x] = find(par[x]); };
  for (uint32_t S = 1; S < (1u << E.size()); S++) {
    std::iota(par.begin(), par.end(), 0);
    int c = 0, ne = 0;
    bool cyc = false;
    std::vector<Edge3> es;
    for (size_t i = 0; i < E.size(); i++)
      if (S >> i & 1) {
        int a = find(E[i].a), b = find(E[i].b);
        if (a == b) {
          cyc = true;
          break;
        }
        par[a] = b;
        c += E[i].w;
        ne++;
        es.push_back(E[i]);
      }
    if (cyc || c >= bestc) continue;
    // connected: all endpoints share one root
    int r = find(es[0].a);
    bool conn = true;
    uint32_t cov = 0;
    for (auto& e : es) {
      if (find(e.a) != r || find(e.b) != r) conn = false;
      cov |= q.mask[e.a] | q.mask[e.b];
    }
    if (!conn || cov != full) continue;
    if (D >= 0 && tree_diameter(es, es[0].a) > D) continue;
    bestc = c;
  }
  *cost = bestc == INT32_MAX ? -1 : bestc;
  return bestc == INT32_MAX ? 1 : 0;
}

// Tree validator.  Returns 0 if valid, else a code:
//  1 edge absent / weight mismatch, 2 not connected or not a tree,
//  3 a query group is not covered, 4 weight sum != cost, 5 diameter > D.
int oracle_validate(uint32_t V, const uint32_t* beg, const uint32_t* adj, const int32_t* w, int k,
                    const uint64_t* qptr, const uint32_t* qv, int D, int32_t cost, uint32_t root,
                    int32_t n_edges, const uint32_t* edges) {
  Csr g{V, beg, adj, w};
  Query q = make_query(g, k, qptr, qv);
  std::vector<Edge3> es;
  int64_t sum = 0;
  for (int i = 0; i < n_edges; i++) {
    uint32_t a = edges[3 * i], b = edges[3 * i + 1];
    int ww = (int)edges[3 * i + 2];
    if (a >= V || b >= V || edge_weight(g, a, b) != ww) return 1;
    es.push_back({a, b, ww});
    sum += ww;
  }
  if (root >= V) return 2;
  int diam = tree_diameter(es, root);
  if (diam < 0) return 2;
  // a tree on n vertices has n-1 edges
  std::vector<uint32_t> vs{root};
  for (auto& e : es) {
    vs.push_back(e.a);
    vs.push_back(e.b);
  }
  std::sort(vs.begin(), vs.end());
  vs.erase(std::unique(vs.begin(), vs.end()), vs.end());
  if ((int64_t)vs.size() != (int64_t)n_edges + 1) return 2;
  uint32_t cov = 0;
  for (uint32_t v : vs) cov |= q.mask[v];
  if (cov != (1u << k) - 1) return 3;
  if (sum != cost) return 4;
  if (D >= 0 && diam > D) return 5;
  return 0;
}

}  // extern "C"
