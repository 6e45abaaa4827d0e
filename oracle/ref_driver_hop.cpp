// Project-written driver around the reference's own HOP_cpu code
// (code/D-PrunedDP++/include/CPUHOP.h, included unchanged).  Prints
//   RESULT <query index> <cost> <feasible 0/1> <seconds> <process_num> <counts>
#include <algorithm>
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
#include "exp_CPU_Hop.h"

int main(int argc, char** argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: %s path name T D start end\n", argv[0]);
    return 2;
  }
  std::string path = argv[1], name = argv[2];
  int T = atoi(argv[3]), D = atoi(argv[4]), s = atoi(argv[5]), e = atoi(argv[6]);
  graph_v_of_v_idealID G, grp;
  std::vector<std::vector<int>> inq;
  read_input_graph(path + name + ".in", G);
  read_Group(path + name + ".g", G, grp);
  read_inquire(path + name + std::to_string(T) + ".csv", inq);
  for (int i = s; i <= e && i < (int)inq.size(); i++) {
    std::unordered_set<int> q(inq[i].begin(), inq[i].end());
    std::vector<int> qv = inq[i];
    int RAM = 0;
    double tr = 0;
    records ret{0, 0};
    auto t0 = std::chrono::high_resolution_clock::now();
    graph_hash_of_mixed_weighted solu = HOP_cpu(q, grp, G, D, tr, RAM, ret);
    auto t1 = std::chrono::high_resolution_clock::now();
    int cost = graph_hash_of_mixed_weighted_sum_of_ec(solu);
    bool ok = this_is_a_feasible_solution_gpu(solu, grp, qv);
    printf("RESULT %d %d %d %.6f %d %d\n", i, cost, ok ? 1 : 0,
           std::chrono::duration<double>(t1 - t0).count(), ret.process_queue_num, ret.counts);
    fflush(stdout);
  }
  return 0;
}
