/*
 * gstb -- B200-native exact group Steiner tree (GST) engine, C ABI.
 *
 * Drop-in for the query path of the reference (toziki/GPUGST).  The reference
 * exposes no library API: its query surface is the C++ function
 *
 *   void DPBF_GPU(node** host_tree, node* host_tree_one_d, CSR_graph& graph,
 *                 std::vector<int>& query_groups, graph_v_of_v_idealID& group_graph,
 *                 graph_v_of_v_idealID& input_graph, int& real_cost,
 *                 non_overlapped_group_sets s, double& rt, int& RAM, records& ret);
 *                                                  (code/GPUGST/include/DPQ.cuh:63)
 *   graph_hash_of_mixed_weighted DPBF_gpu(CSR_graph&, std::vector<int>& query_groups,
 *                 graph_v_of_v_idealID& group_graph, graph_v_of_v_idealID& input_graph,
 *                 int D, double* rt, int& real_cost, int& RAM, records&);
 *                                                  (code/D-GPUGST/include/DPQ.cuh:63)
 *
 * called once per query from the experiment drivers
 * (code/GPUGST/include/exp_GPU_nonHop.h:124, code/D-GPUGST/include/exp_GPU_Hop.h).
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions: plain pointers and sizes only; the caller owns every host
 * buffer; the library owns every device buffer.  Costs are int32 edge-weight
 * sums; vertex ids are uint32; a query names k (1..7) group indices (0-based,
 * i.e. the `.g` file id minus one, as read_Group does at
 * graph_hash_of_mixed_weighted_read_for_GSTP.h:206).  D < 0 means no hop bound;
 * 0 <= D <= 7 bounds the tree's hop diameter (the recurrence of
 * code/D-PrunedDP++/include/CPUHOP.h:192-227: grow d -> d+1 while d < D, merge
 * with d1 + d2 <= D into max(d1, d2)).
 */
#ifndef GSTB_H
#define GSTB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Replace the reference's exit(1) / "can not find" prints
 * (DPQ.cuh:24-41, DPQ.cu:495-500,571-575) and its two conflicting "no
 * solution" encodings (cost 0 on GPU, 100000 on CPU). */
typedef enum gst_status {
  GST_OK = 0,
  GST_NO_SOLUTION = 1,      /* the query groups are not connected */
  GST_BAD_INPUT = 2,        /* malformed graph / group index / query */
  GST_OOM = 3,              /* device memory for the state table not available */
  GST_DEVICE_TIMEOUT = 4,   /* a bounded device wait expired */
  GST_CUDA_ERROR = 5,       /* a CUDA runtime call failed */
  GST_QUEUE_OVERFLOW = 6,   /* a frontier exceeded its capacity: gst_query_noalloc only; the
                               other entry points rerun the query with 4x larger lists */
  GST_TRUNCATED = 7,        /* tree has more edges than the caller's buffer */
  GST_INTERNAL = 8,         /* internal consistency check failed */
  GST_BUSY = 9,             /* serving: no free slot right now (submit again) */
  GST_NOT_FOUND = 10,       /* serving: unknown request id */
  GST_SCRATCH_TOO_SMALL = 11, /* gst_query_noalloc: workspace exceeds the static scratch */
  GST_CANCELLED = 12        /* serving: the request was withdrawn by gst_serve_cancel */
} gst_status;

typedef struct gst_graph gst_graph;

/* Statistics of one query (the reference's CSV columns `counts` and
 * `process_num`, exp_GPU_nonHop.h:87, plus device counters). */
enum {
  GST_STAT_EXPANDED = 0,    /* DP states expanded (reference process_num, DPQ.cu:514) */
  GST_STAT_SSSP_ITEMS = 1,  /* distance items expanded */
  GST_STAT_ARCS = 2,        /* arcs scanned by DP grows */
  GST_STAT_UPDATES = 3,     /* successful DP state lowerings */
  GST_STAT_ENQUEUED = 4,    /* DP frontier insertions */
  GST_STAT_ROUNDS = 5,      /* device rounds */
  GST_STAT_MERGES = 6,      /* merge candidates evaluated */
  GST_STAT_TABLE_BYTES = 7, /* bytes of the state table */
  GST_STAT_SSSP_ARCS = 8,   /* arcs scanned by distance items */
  GST_STAT_SSSP_UPDATES = 9,  /* successful distance lowerings */
  GST_STAT_SSSP_ENQUEUED = 10, /* distance frontier insertions */
  GST_STAT_RETRIES = 11,    /* runs repeated with 4x larger frontier lists after GST_QUEUE_OVERFLOW */
  GST_STAT_LOWER_BOUND = 12,  /* proven lower bound on the optimum (= cost for an exact answer) */
  GST_NSTATS = 13
};

typedef struct gst_result {
  int32_t cost;            /* optimal cost (valid when status == GST_OK) */
  uint32_t root;           /* root vertex of the returned tree */
  int32_t n_edges;         /* number of tree edges (may exceed max_edges: TRUNCATED) */
  int32_t max_edges;       /* capacity of `edges` in edges (caller sets) */
  uint32_t* edges;         /* caller buffer, 3*max_edges uint32: (u, v, w) triples */
  uint64_t stats[GST_NSTATS];
  double device_ms;        /* device time of the call that ran this query (CUDA
                              events around all of that call's rounds) */
  double latency_ms;       /* host time from submission to completion */
} gst_result;

/* Replaces toCSR (code/GPUGST/include/graph_v_of_v_idealID/csr_graph.hpp:39-128):
 * copies a symmetric CSR (beg_pos[V+1], csr[arcs], w[arcs]; both directions
 * of every undirected edge present; weights >= 1) to the device.  The library
 * keeps its own device copy with each adjacency list re-sorted by weight.
 * Costs are summed in 32 bits: a graph whose V-1 heaviest arcs weigh 2^30 or
 * more in total (the bound on any shortest path or tree) is GST_BAD_INPUT. */
gst_status gst_graph_create(const uint32_t* beg_pos, const uint32_t* csr, const int32_t* w,
                            uint32_t V, uint64_t arcs, gst_graph** out);

/* Replaces read_Group's group_graph (graph_hash_of_mixed_weighted_read_for_GSTP.h:190-239):
 * group g has members grp_v[grp_ptr[g] .. grp_ptr[g+1]).  Copied to the device. */
gst_status gst_groups_set(gst_graph* g, const uint64_t* grp_ptr, const uint32_t* grp_v,
                          uint32_t n_groups);

void gst_graph_destroy(gst_graph* g);

uint32_t gst_graph_num_vertices(const gst_graph* g);
uint64_t gst_graph_num_arcs(const gst_graph* g);

/* Replaces DPBF_GPU (code/GPUGST/include/DPQ.cuh:63, DPQ.cu:275-624) when D < 0
 * and DPBF_gpu (code/D-GPUGST/include/DPQ.cuh:63, D-GPUGST/src/DPQ.cu:149-269)
 * when D >= 0.  One synchronous query; returns the exact optimum cost and a
 * tree (the reference's GPU path returns the cost only; its extraction is
 * commented out at DPQ.cu:577-606). */
gst_status gst_query(gst_graph* g, const uint32_t* groups, int k, int D, gst_result* out);

/* Progressive mode (the reference's maximum_return_app_ratio,
 * code/PrunedDP++/include/CPUNONHOP.h:499,730-755): the query may stop before
 * the DP has proven optimality, once the best tree recorded costs at most
 * `ratio` times a proven lower bound on the optimum.  The returned cost is
 * then at most ratio x the optimum, and stats[GST_STAT_LOWER_BOUND] holds the
 * bound.  The comparison is exact integer arithmetic (ratio is taken in
 * steps of 1/1024, rounded down), unlike the reference's integer division
 * (CPUNONHOP.h:733), which returns up to 2x the optimum at ratio 1.  The tree
 * is the minimum spanning tree of the recorded derivation's edges, as the
 * reference post-processes its incumbent.  ratio <= 1 is the exact query.
 * Hop-bounded queries (D >= 0) are always exact: the reference's hop program
 * (CPUHOP.h) has no ratio exit either. */
gst_status gst_query_ratio(gst_graph* g, const uint32_t* groups, int k, int D, double ratio, gst_result* out);

/* Allocation-free variant of gst_query.  It has no counterpart in the
 * reference.  Some callers cannot allocate device memory while they answer a
 * query: a host program that reserves all of the GPU's memory for its own
 * pool at start-up, so a cudaMalloc from this library would fail or take
 * memory the host has already promised elsewhere; and a latency-critical
 * loop in which cudaMalloc / cudaFree, which may synchronise the device,
 * are not allowed.  This entry point runs the same kernels as gst_query but
 * keeps every per-query buffer (state table, distances, frontier lists,
 * control blocks, tree output) in one static device array of
 * GST_NOALLOC_SCRATCH_BYTES (64 MiB) compiled into this library.  Every GPU
 * on which the library is loaded holds that array until the process exits.
 * The call allocates no device or pinned host memory and issues its work on
 * the legacy default stream; it returns when the GPU work is done.
 *   - A query whose workspace does not fit returns GST_SCRATCH_TOO_SMALL
 *     (roughly: V * 2^k * (D+1) states need 8 + 16 + 2^-2 bytes each).
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current; make that first call
 *     before any stream capture.
 *   - All calls share the array; each call re-initialises what must start
 *     empty.  Calls that overlapped on the GPU would race on it, so the
 *     library serialises its own calls with a mutex.  A call also holds the
 *     graph's lock, so on one graph it waits for (and holds off)
 *     gst_query, gst_query_batch, gst_tuning_set and gst_autotune, and it
 *     reads the group index under the lock gst_groups_set takes.
 * Trees are returned with up to 4096 edges (GST_TRUNCATED beyond).  The
 * call switches to the graph's device for its duration and restores the
 * caller's current device before returning. */
#define GST_NOALLOC_SCRATCH_BYTES (64ull << 20)
gst_status gst_query_noalloc(gst_graph* g, const uint32_t* groups, int k, int D, gst_result* out);

/* Launch parameters of a graph's engine (no reference counterpart: the
 * reference fixes its block sizes and thresholds at compile time, DPQ.cuh:43
 * and GPUGST+/include/util.h:19-33).  Defaults, overridable at
 * gst_graph_create by GSTB_DELTA_SSSP / GSTB_DELTA_DP / GSTB_HUB_MIN_DEG /
 * GSTB_SSSP_CAP_PCT / GSTB_PERSIST / GSTB_ROUNDS_PER_SYNC / GSTB_DP_WMAX /
 * GSTB_SSSP_WMAX / GSTB_MERGE_STAGE / GSTB_BLOCK_THREADS: 16, 8, 256, 60, 0,
 * 4, 32, 32, 14, 256.  None
 * of them changes a result, only the work schedule and how tight the lower
 * bounds are. */
typedef struct gst_tuning {
  uint32_t delta_sssp;   /* width of the distance rounds' near-far window */
  uint32_t delta_dp;     /* width of the DP rounds' near-far window */
  uint32_t hub_min_deg;  /* a vertex with this many arcs to relax hands them out in chunks (>= 32) */
  uint32_t cap_pct;      /* distances are computed exactly up to this percentage of the incumbent (1..100) */
  uint32_t persistent;   /* 1: each block of rounds is one persistent cooperative launch (the round
                            loop runs on the device, every block resident); 0: a CUDA graph of
                            control / light / heavy launches per round */
  uint32_t rounds_per_launch; /* rounds per block (1..64); between blocks the host retires finished
                                 queries and admits new ones */
  uint32_t dp_wmax;      /* most DP states per warp task: 1, 2, 4, 8, 16 or 32 */
  uint32_t sssp_wmax;    /* most distance items (vertices) per warp task: 4, 8, 16 or 32 */
  uint32_t merge_stage;  /* merge tile: a DP state with at least this many merge partners first
                            stages its vertex's table and bound rows in shared memory (0: never) */
  uint32_t block_threads; /* threads per block of the round kernels: 128 or 256 (24 warps per SM
                             either way) */
} gst_tuning;

gst_status gst_tuning_get(gst_graph* g, gst_tuning* out);
gst_status gst_tuning_set(gst_graph* g, const gst_tuning* t);
/* Autotuner for the graph's degree profile: times a sample of n queries
 * (laid out as for gst_query_batch) under candidate settings (cap_pct 50/60/
 * 67/75, delta_sssp 8..64, delta_dp 2..16, hub_min_deg 128..1024, persistent
 * 0/1, rounds_per_launch 2..16, dp_wmax 4..32, sssp_wmax 8..32, merge_stage
 * 0/6/14/30, block_threads 128/256), one parameter at a time, and keeps the
 * fastest.  objective 0 = batch throughput
 * (gst_query_batch), 1 = one query at a time (gst_query).  The chosen
 * settings stay on the graph; out (may be null) receives them. */
gst_status gst_autotune(gst_graph* g, int n, const uint32_t* groups, const int32_t* ks, const int32_t* Ds,
                        int objective, gst_tuning* out);

/* Row stride of the groups array of gst_query_batch. */
#define GST_GROUPS_STRIDE 8

/* Batched launch: n queries share the device rounds.  groups[i*8 .. i*8+ks[i])
 * lists query i's groups.  results[i].edges/max_edges set by the caller.
 * statuses[i] receives each query's status.  Queries are admitted by the HBM
 * bytes of their state tables; at most max_concurrent run at once (0 = as
 * many as fit). */
gst_status gst_query_batch(gst_graph* g, int n, const uint32_t* groups, const int32_t* ks,
                           const int32_t* Ds, gst_result* results, int32_t* statuses,
                           int max_concurrent);
/* gst_query_batch with a progressive-mode ratio per query (ratios may be
 * null: every query exact; see gst_query_ratio). */
gst_status gst_query_batch_ratio(gst_graph* g, int n, const uint32_t* groups, const int32_t* ks,
                                 const int32_t* Ds, const double* ratios, gst_result* results,
                                 int32_t* statuses, int max_concurrent);

/* Serving loop (continuous batching).  A background host thread keeps the
 * graph resident, admits submitted queries as device memory frees up, and
 * runs every admitted query's rounds together.  No reference counterpart
 * (the reference runs queries serially, exp_GPU_nonHop.h:97-138). */
typedef struct gst_server gst_server;

/* hbm_budget_bytes: device bytes the admitted queries' workspaces may hold
 * at once (0 = 80% of the free memory at open), reserved in one allocation
 * at open (GSTB_SERVE_RESERVE_MB caps the reservation; beyond it the loop
 * allocates as requests need); max_inflight: queries on the device at once
 * (0 = up to 1023).  Each result's latency_ms is the time from submission to
 * completion. */
gst_status gst_serve_open(gst_graph* g, uint64_t hbm_budget_bytes, int max_inflight,
                          gst_server** out);
/* Never blocks.  Copies the groups.  GST_BUSY if the pending queue is full. */
gst_status gst_serve_submit(gst_server* s, uint64_t req_id, const uint32_t* groups, int k, int D);
/* gst_serve_submit in progressive mode (see gst_query_ratio). */
gst_status gst_serve_submit_ratio(gst_server* s, uint64_t req_id, const uint32_t* groups, int k, int D,
                                  double ratio);
/* Returns up to max_results finished requests; *n_out set.  Tree edges are
 * copied into each result's caller buffer (edges/max_edges preset by the
 * caller; pass max_edges 0 to skip trees).  ids[i] and statuses[i] filled. */
gst_status gst_serve_poll(gst_server* s, uint64_t* ids, int32_t* statuses, gst_result* results,
                          int max_results, int* n_out);
/* Withdraws a request.  A pending request (not yet on the device) finishes at
 * once; an admitted one is ended by the device at its next round.  Either way
 * it is reported by gst_serve_poll with status GST_CANCELLED, unless it
 * finished first (then it keeps its own result).  GST_NOT_FOUND if no pending
 * or admitted request has this id.  No reference counterpart. */
gst_status gst_serve_cancel(gst_server* s, uint64_t req_id);
/* Largest number of pending (submitted, not yet admitted) requests; a submit
 * beyond it returns GST_BUSY (load shedding).  Default 2^20. */
gst_status gst_serve_set_max_pending(gst_server* s, uint64_t max_pending);
/* Occupancy and counters of a server (the quantities a front-end routes on). */
typedef struct gst_serve_info {
  uint64_t pending;            /* submitted, waiting for admission */
  uint64_t inflight;           /* admitted, on the device */
  uint64_t finished_unpolled;  /* finished, not yet returned by gst_serve_poll */
  uint64_t budget_bytes;       /* HBM budget of the admitted workspaces */
  uint64_t in_use_bytes;       /* workspace bytes of the admitted requests */
  uint64_t submitted, completed, rejected_busy, cancelled, oom;  /* totals since open */
} gst_serve_info;
gst_status gst_serve_stats(gst_server* s, gst_serve_info* out);
/* Stops the loop after the submitted requests finish and frees everything;
 * results not polled by then are discarded. */
gst_status gst_serve_close(gst_server* s);

/* Fault injection for tests (no reference counterpart): the next n workspace
 * allocations of this graph's engines fail as if the device were full.  A
 * query that cannot be admitted while nothing else runs returns GST_OOM;
 * with others running it waits for their memory. */
gst_status gst_debug_fail_allocs(gst_graph* g, int n);
/* Test hook for the persistent round launch's bounded waits: while hold is 1
 * its control steps are not published, so every wait of a launch expires
 * after timeout_ms (0: the default, GSTB_WAIT_MS or 30000) and the admitted
 * queries end with GST_DEVICE_TIMEOUT; the device stays usable.  hold 0 and
 * timeout_ms 0 restore normal running. */
gst_status gst_debug_hold_rounds(gst_graph* g, int hold, uint32_t timeout_ms);

const char* gst_status_string(gst_status st);
/* The CUDA runtime's description of the last CUDA error any gstb call in this
 * process met (the detail behind GST_CUDA_ERROR); "no error" if none. */
const char* gst_last_cuda_error(void);

/* Diagnostics (no reference counterpart).  Kernel launches issued by this
 * graph's engine so far, and, when profiling is on (gst_query_batch calls
 * only), the accumulated device time of the round kernels
 * (kernel_ms[0] = k_light: distance items, splits, seeds, tours,
 * extraction, DP states; kernel_ms[1] = k_heavy: arc chunks, lower-bound
 * rows, snapshots; when the rounds ran as persistent launches,
 * kernel_ms[0] = k_rounds, all of the round, and kernel_ms[1] = 0), the
 * number of rounds, and the summed GST_STAT_* counters of finished queries. */
uint64_t gst_kernel_launches(const gst_graph* g);
void gst_profile_enable(gst_graph* g, int on);
void gst_profile_read(const gst_graph* g, double kernel_ms[2], uint64_t* rounds,
                      uint64_t stats_totals[GST_NSTATS]);
void gst_profile_reset(gst_graph* g);

#ifdef __cplusplus
}
#endif

#endif /* GSTB_H */
