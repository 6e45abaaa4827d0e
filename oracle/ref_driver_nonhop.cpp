// Project-written driver around the reference's own PrunedDP++ code
// (code/PrunedDP++/include/CPUNONHOP.h, included unchanged through the
// include path set by oracle/Makefile).  Reads the reference file formats
// with the reference's readers and prints one line per query:
//   RESULT <query index> <cost> <feasible 0/1> <seconds> <process_num> <counts>
// ratio is the reference's maximum_return_app_ratio (the reference driver
// hard-codes 1 at exp_CPU_nonHop.h:113; 0 keeps only the exact exits).
#include <algorithm>
#include <cstdint>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <iterator>
#include <queue>
#include <sstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>
// the reference headers expect std in scope (as its main.cpp provides)
using namespace std;
#include "exp_CPU_nonHop.h"

// Binary input (--bin <prefix>): the same graph and group structures the
// reference's text readers build (read_input_graph: per vertex the
// (neighbour, weight) pairs sorted by neighbour; read_Group: per group its
// (member, 1) pairs sorted by member), filled from raw arrays instead of
// parsed text.  <prefix>.beg u32[V+1], .adj u32[arcs], .w i32[arcs] (a
// symmetric CSR with each list sorted by neighbour), .gptr u64[n+1],
// .gv u32[members] (each group sorted), .q<T> u32[queries][T].  Only the
// loading differs; the timed call is the reference's own.
template <class X>
static std::vector<X> read_raw(const std::string& f) {
  std::ifstream in(f, std::ios::binary | std::ios::ate);
  if (!in) {
    fprintf(stderr, "cannot open %s\n", f.c_str());
    exit(2);
  }
  size_t n = (size_t)in.tellg() / sizeof(X);
  std::vector<X> v(n);
  in.seekg(0);
  in.read(reinterpret_cast<char*>(v.data()), n * sizeof(X));
  return v;
}

static void load_bin(const std::string& pre, int T, graph_v_of_v_idealID& G, graph_v_of_v_idealID& grp,
                     std::vector<std::vector<int>>& inq) {
  auto beg = read_raw<uint32_t>(pre + ".beg");
  auto adj = read_raw<uint32_t>(pre + ".adj");
  auto w = read_raw<int32_t>(pre + ".w");
  auto gptr = read_raw<uint64_t>(pre + ".gptr");
  auto gv = read_raw<uint32_t>(pre + ".gv");
  auto qq = read_raw<uint32_t>(pre + ".q" + std::to_string(T));
  G.assign(beg.size() - 1, {});
  for (size_t v = 0; v + 1 < beg.size(); v++) {
    G[v].reserve(beg[v + 1] - beg[v]);
    for (uint32_t a = beg[v]; a < beg[v + 1]; a++) G[v].push_back({(int)adj[a], (int)w[a]});
  }
  grp.assign(gptr.size() - 1, {});
  for (size_t g = 0; g + 1 < gptr.size(); g++)
    for (uint64_t t = gptr[g]; t < gptr[g + 1]; t++) grp[g].push_back({(int)gv[t], 1});
  for (size_t i = 0; i + T <= qq.size(); i += T) inq.push_back(std::vector<int>(qq.begin() + i, qq.begin() + i + T));
}

int main(int argc, char** argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: %s path name T start end ratio\n       %s --bin prefix T start end ratio\n",
            argv[0], argv[0]);
    return 2;
  }
  std::string path = argv[1], name = argv[2];
  int T = atoi(argv[3]), s = atoi(argv[4]), e = atoi(argv[5]), ratio = atoi(argv[6]);
  graph_v_of_v_idealID G, grp;
  std::vector<std::vector<int>> inq;
  if (path == "--bin") {
    load_bin(name, T, G, grp, inq);
  } else {
    read_input_graph(path + name + ".in", G);
    read_Group(path + name + ".g", G, grp);
    read_inquire(path + name + std::to_string(T) + ".csv", inq);
  }
  fprintf(stderr, "LOADED\n");
  for (int i = s; i <= e && i < (int)inq.size(); i++) {
    std::unordered_set<int> q(inq[i].begin(), inq[i].end());
    std::vector<int> qv = inq[i];
    int RAM = 0;
    double tr = 0;
    records ret{0, 0};
    auto t0 = std::chrono::high_resolution_clock::now();
    graph_hash_of_mixed_weighted solu = graph_v_of_v_idealID_PrunedDPPlusPlus(G, grp, q, ratio, RAM, tr, ret);
    auto t1 = std::chrono::high_resolution_clock::now();
    int cost = graph_hash_of_mixed_weighted_sum_of_ec(solu);
    bool ok = this_is_a_feasible_solution_gpu(solu, grp, qv);
    printf("RESULT %d %d %d %.6f %d %d\n", i, cost, ok ? 1 : 0,
           std::chrono::duration<double>(t1 - t0).count(), ret.process_queue_num, ret.counts);
    fflush(stdout);
  }
  return 0;
}
