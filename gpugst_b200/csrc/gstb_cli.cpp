// gstb: command-line driver with the reference's argv and CSV output.
//
//   gstb 2 <path> <name> <k> <start> <end>          (GPUGST:   code/GPUGST/src/main.cpp:14-17)
//   gstb 2 <path> <name> <k> <D> <start> <end>      (D-GPUGST: code/D-GPUGST/src/main.cpp)
//
// Reads <path><name>.in (or the int64 <name>_beg_pos/_csr/_weight.bin CSR),
// <path><name>.g and <path><name><k>.csv, answers queries start..end through
// the C ABI and writes <path>result/exp_GPU1_nonHop_<name>_T<k>_<s>-<e>.csv
// (exp_GPU1_Hop_..._D<D>_... with a hop bound) with the reference's columns
// (exp_GPU_nonHop.h:85-87,128; exp_GPU_Hop.h:38-40,70):
//   task_ID,task,GPU1_nonHop_time,GPU_nonHop_cost,GPU_nonHop_memory,counts,process_num
// A query without a solution is written with cost 0, as the reference's GPU
// programs do (DPQ.cu:571-575).  GSTB_CLI_BATCH=1 answers the whole range in
// one gst_query_batch call instead of one gst_query per line.
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gstb.h"

namespace {

bool exists(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0;
}

// ".in": "V E" header, then "v1 v2 w" lines; each edge in both directions,
// adjacency sorted by neighbour (read_input_graph, read_for_GSTP.h:75-148).
bool read_in(const std::string& path, uint32_t& V, std::vector<uint32_t>& beg, std::vector<uint32_t>& adj,
             std::vector<int32_t>& w) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  if (!std::getline(f, line)) return false;
  V = (uint32_t)std::stod(line.substr(0, line.find(' ')));
  std::vector<std::vector<std::pair<uint32_t, int32_t>>> g(V);
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    std::vector<std::string> t;
    std::string x;
    while (ss >> x) t.push_back(x);
    if (t.size() != 3) continue;
    uint32_t a = (uint32_t)std::stoul(t[0]), b = (uint32_t)std::stoul(t[1]);
    int32_t ww = std::stoi(t[2]);
    if (a >= V || b >= V) return false;
    g[a].push_back({b, ww});
    g[b].push_back({a, ww});
  }
  beg.assign(V + 1, 0);
  for (uint32_t v = 0; v < V; v++) {
    std::sort(g[v].begin(), g[v].end());
    beg[v + 1] = beg[v] + (uint32_t)g[v].size();
  }
  adj.resize(beg[V]);
  w.resize(beg[V]);
  for (uint32_t v = 0; v < V; v++)
    for (size_t i = 0; i < g[v].size(); i++) {
      adj[beg[v] + i] = g[v][i].first;
      w[beg[v] + i] = g[v][i].second;
    }
  return true;
}

// int64 CSR files of GPUGST+ (code/GPUGST+/include/graph.hpp:12-118)
bool read_bin(const std::string& prefix, uint32_t& V, std::vector<uint32_t>& beg, std::vector<uint32_t>& adj,
              std::vector<int32_t>& w) {
  auto load = [](const std::string& p, std::vector<int64_t>& out) {
    FILE* f = fopen(p.c_str(), "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long n = ftell(f) / 8;
    fseek(f, 0, SEEK_SET);
    out.resize(n);
    bool ok = fread(out.data(), 8, n, f) == (size_t)n;
    fclose(f);
    return ok;
  };
  std::vector<int64_t> b, c, ww;
  if (!load(prefix + "_beg_pos.bin", b) || !load(prefix + "_csr.bin", c) || !load(prefix + "_weight.bin", ww))
    return false;
  if (b.empty() || (int64_t)c.size() != b.back() || c.size() != ww.size()) return false;
  V = (uint32_t)(b.size() - 1);
  beg.assign(b.begin(), b.end());
  adj.assign(c.begin(), c.end());
  w.assign(ww.begin(), ww.end());
  return true;
}

// ".g": "g<id>:v v v" per line; group index = id - 1 (read_Group, :190-239)
bool read_groups(const std::string& path, std::vector<uint64_t>& ptr, std::vector<uint32_t>& mem) {
  std::ifstream f(path);
  if (!f) return false;
  std::vector<std::vector<uint32_t>> gs;
  std::string line;
  while (std::getline(f, line)) {
    while (!line.empty() && (line.back() == ' ' || line.back() == '\r')) line.pop_back();
    size_t c = line.find(':');
    if (line.empty() || c == std::string::npos) continue;
    long id = (long)std::stod(line.substr(1, c - 1)) - 1;
    if (id < 0) return false;
    if ((size_t)id >= gs.size()) gs.resize(id + 1);
    std::istringstream ss(line.substr(c + 1));
    uint32_t v;
    while (ss >> v) gs[id].push_back(v);
    std::sort(gs[id].begin(), gs[id].end());
  }
  ptr.assign(1, 0);
  for (auto& g : gs) {
    mem.insert(mem.end(), g.begin(), g.end());
    ptr.push_back(mem.size());
  }
  return true;
}

// "<name><k>.csv": k group indices per line (read_inquire, :240-286)
bool read_queries(const std::string& path, std::vector<std::vector<uint32_t>>& q) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    std::vector<uint32_t> row;
    uint32_t x;
    while (ss >> x) row.push_back(x);
    if (!row.empty()) q.push_back(row);
  }
  return true;
}

int usage() {
  fprintf(stderr,
          "usage: gstb 2 <path> <name> <k> <start> <end>\n"
          "       gstb 2 <path> <name> <k> <D> <start> <end>\n");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 7 && argc != 8) return usage();
  if (atoi(argv[1]) != 2) return usage();
  const std::string path = argv[2], name = argv[3];
  const int k = atoi(argv[4]);
  const bool hop = argc == 8;
  const int D = hop ? atoi(argv[5]) : -1;
  const int s = atoi(argv[hop ? 6 : 5]), e = atoi(argv[hop ? 7 : 6]);

  uint32_t V = 0;
  std::vector<uint32_t> beg, adj;
  std::vector<int32_t> w;
  bool ok = exists(path + name + ".in") ? read_in(path + name + ".in", V, beg, adj, w)
                                        : read_bin(path + name, V, beg, adj, w);
  if (!ok) {
    fprintf(stderr, "gstb: cannot read the graph %s%s(.in | _*.bin)\n", path.c_str(), name.c_str());
    return 1;
  }
  std::vector<uint64_t> gptr;
  std::vector<uint32_t> gmem;
  if (!read_groups(path + name + ".g", gptr, gmem)) {
    fprintf(stderr, "gstb: cannot read %s%s.g\n", path.c_str(), name.c_str());
    return 1;
  }
  std::vector<std::vector<uint32_t>> inq;
  if (!read_queries(path + name + std::to_string(k) + ".csv", inq)) {
    fprintf(stderr, "gstb: cannot read %s%s%d.csv\n", path.c_str(), name.c_str(), k);
    return 1;
  }
  gst_graph* G = nullptr;
  gst_status st = gst_graph_create(beg.data(), adj.data(), w.data(), V, adj.size(), &G);
  if (st != GST_OK) {
    fprintf(stderr, "gstb: gst_graph_create: %s\n", gst_status_string(st));
    return 1;
  }
  st = gst_groups_set(G, gptr.data(), gmem.data(), (uint32_t)(gptr.size() - 1));
  if (st != GST_OK) {
    fprintf(stderr, "gstb: gst_groups_set: %s\n", gst_status_string(st));
    return 1;
  }
  const int last = std::min(e, (int)inq.size() - 1);
  std::string out = path + "result/exp_GPU1_" + (hop ? "Hop_" : "nonHop_") + name + "_T" + std::to_string(k) + "_" +
                    (hop ? "D" + std::to_string(D) + "_" : std::string()) + std::to_string(s) + "-" +
                    std::to_string(e) + ".csv";
  mkdir((path + "result").c_str(), 0755);
  FILE* of = fopen(out.c_str(), "w");
  if (!of) {
    fprintf(stderr, "gstb: cannot write %s\n", out.c_str());
    return 1;
  }
  fprintf(of, hop ? "task_ID,task,GPU1_Hop_time,GPU1_Hop_cost,GPU1_Hop_memory,counts,process_num\n"
                  : "task_ID,task,GPU1_nonHop_time,GPU_nonHop_cost,GPU_nonHop_memory,counts,process_num\n");
  const int n = std::max(0, last - s + 1);
  std::vector<gst_result> res(n);
  std::vector<int32_t> sts(n, GST_BAD_INPUT);
  std::vector<std::vector<uint32_t>> ebuf(n, std::vector<uint32_t>(3 * 4096));
  for (int i = 0; i < n; i++) {
    memset(&res[i], 0, sizeof(gst_result));
    res[i].edges = ebuf[i].data();
    res[i].max_edges = 4096;
  }
  const char* bm = getenv("GSTB_CLI_BATCH");
  if (bm && atoi(bm) == 1) {
    std::vector<uint32_t> groups((size_t)n * 8, 0);
    std::vector<int32_t> ks(n), Ds(n, D);
    for (int i = 0; i < n; i++) {
      const auto& q = inq[s + i];
      ks[i] = (int32_t)q.size();
      for (size_t j = 0; j < q.size() && j < 8; j++) groups[(size_t)i * 8 + j] = q[j];
    }
    st = gst_query_batch(G, n, groups.data(), ks.data(), Ds.data(), res.data(), sts.data(), 0);
    if (st != GST_OK) {
      fprintf(stderr, "gstb: gst_query_batch: %s\n", gst_status_string(st));
      return 1;
    }
  } else {
    for (int i = 0; i < n; i++) {
      const auto& q = inq[s + i];
      sts[i] = gst_query(G, q.data(), (int)q.size(), D, &res[i]);
    }
  }
  for (int i = 0; i < n; i++) {
    const auto& q = inq[s + i];
    std::string task;
    for (uint32_t x : q) task += std::to_string(x) + " ";
    const gst_result& r = res[i];
    int cost = sts[i] == GST_OK ? r.cost : 0;
    if (sts[i] != GST_OK && sts[i] != GST_NO_SOLUTION)
      fprintf(stderr, "gstb: query %d: %s\n", s + i, gst_status_string((gst_status)sts[i]));
    fprintf(of, "%d,%s,%.8f,%d,%llu,%llu,%llu\n", s + i, task.c_str(), r.latency_ms / 1e3, cost,
            (unsigned long long)(r.stats[GST_STAT_TABLE_BYTES] / 8),
            (unsigned long long)r.stats[GST_STAT_ENQUEUED], (unsigned long long)r.stats[GST_STAT_EXPANDED]);
    printf("query %d cost %d\n", s + i, cost);
  }
  fprintf(of, "\n");
  fclose(of);
  gst_graph_destroy(G);
  return 0;
}
