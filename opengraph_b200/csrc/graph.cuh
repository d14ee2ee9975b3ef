// graph.cuh -- device-resident GraphCSR (both directions) and the entry
// points of the hot-path modules (build, BFS, PageRank).
#pragma once
#include "common.cuh"
#include "sort.cuh"

#include <vector>

namespace ogb {

// One direction of a CSR on the device.  Field meaning follows the
// reference's struct Vertex + struct EdgeList (vertex.h:13-18,
// edgeList.h:8-23): src/dst/w are the sorted edge arrays, edges_idx the first
// edge of each vertex (0 when it has none), out_degree the run length;
// rows packs {edges_idx, out_degree} for one 8-byte load per vertex.
struct DevCSR {
  DevBuf src, dst, w;
  DevBuf out_degree, in_degree, edges_idx;
  DevBuf rows;  // uint2 per vertex
  uint32_t* d_src() const { return src.as<uint32_t>(); }
  uint32_t* d_dst() const { return dst.as<uint32_t>(); }
  float* d_w() const { return w.as<float>(); }
  uint32_t* d_out_degree() const { return out_degree.as<uint32_t>(); }
  uint32_t* d_in_degree() const { return in_degree.as<uint32_t>(); }
  uint32_t* d_edges_idx() const { return edges_idx.as<uint32_t>(); }
  uint2* d_rows() const { return rows.as<uint2>(); }
};

struct BfsWork;  // bfs.cu
struct PrWork;   // pagerank.cu
struct MsWork;   // batch.cu
struct PprWork;  // batch.cu
void bfs_work_free(BfsWork* w);
void pr_work_free(PrWork* w);
void ms_work_free(MsWork* w);
void ppr_work_free(PprWork* w);

struct BfsLevel {
  uint32_t direction;  // 0 top-down, 1 bottom-up
  uint32_t discovered; // vertices discovered by this step
  uint32_t frontier;   // frontier size entering the step
  uint32_t mf, mu;     // switch state after the step (top-down) / entering it
  uint64_t edges;      // edges examined by the step
  float ms;            // device time of the step (when timed)
};

struct DevGraph {
  uint32_t V = 0;
  uint32_t E = 0;
  bool weighted = false;
  uint32_t sort_type = 0;
  DevCSR fwd, inv;
  SortWorkspace sort_ws;
  DevBuf input_src, input_dst, input_w;  // staging of host uploads
  DevBuf err;                            // u32 error word of the build kernels
  DevBuf range_q;                        // scratch of the partitioned BFS steps (bfs_range.cu)
  uint32_t build_id = 0;  // bumped whenever the edges change (caches key on it)
  BfsWork* bfs = nullptr;
  PrWork* pr = nullptr;
  MsWork* ms = nullptr;
  PprWork* ppr = nullptr;
  // traces of the last BFS / PageRank run through the device API
  std::vector<BfsLevel> bfs_trace;  // the last BFS's steps (up to the trace capacity)
  std::vector<float> bfs_feat;      // learned-switch inputs before each of those steps, 8 per step
  uint32_t pr_last_executed = 0;
  double pr_err_hist[1024];
  uint32_t pr_active_hist[1024];
  ~DevGraph();
};

// Sort the device edge list (in_src, in_dst[, in_w]) with SORT_TYPE
// semantics (0/2 by src, 1/3 by (src, dst)) and build both CSR directions.
// All ids must be < V <= 2^30.  Inputs are not modified.
int graph_build(DevGraph& g, const uint32_t* in_src, const uint32_t* in_dst, const float* in_w,
                uint32_t E, uint32_t V, uint32_t sort_type, cudaStream_t s);

// Fill the per-vertex arrays of one direction from its sorted src array
// (the reference's mapVerticesWithInOutDegree, vertex.c:204-325), and the
// in_degree array of the other direction.
int csr_map(DevCSR& c, DevCSR& other, uint32_t V, uint32_t E, uint32_t* d_err, cudaStream_t s);

// Rebuild the packed rows of one direction from edges_idx/out_degree (used
// after an upload of a host GraphCSR).
int csr_pack_rows(DevCSR& c, uint32_t V, cudaStream_t s);

int sort_check(SortWorkspace& ws, cudaStream_t stream);

// out[0..n] = exclusive scan of in[0..n) followed by the total (out holds
// n + 1 entries); tmp holds scan_tmp_words(n) words.  scan.cu.
int scan_exclusive_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t s);
size_t scan_tmp_words(uint32_t n);
int graph_check(DevGraph& g, cudaStream_t s);

// ---- BFS -------------------------------------------------------------------
// BFS_PULL_DENSE: pull-only with every bottom-up step over all vertices (no
// unvisited list) -- a cost probe for the learned switch's training data.
enum BfsMode : uint32_t { BFS_PULL = 0, BFS_PUSH = 1, BFS_DO = 2, BFS_LEARNED = 3, BFS_PULL_DENSE = 4 };



struct BfsResult {
  uint32_t iteration = 0;        // BFSStats.iteration
  uint32_t processed_nodes = 0;  // BFSStats.processed_nodes
  uint32_t td_steps = 0, bu_steps = 0;
  uint64_t edges_examined = 0;
  uint64_t reached_out_edges = 0;  // sum of out-degrees of reached vertices
  uint32_t reached = 0;
  uint32_t launches = 0;  // kernels launched by the traversal
  double ms = 0.0;
  int nlevels = 0;                // steps taken
  std::vector<BfsLevel> levels;   // per-step trace (when asked for; at most the trace capacity)
  std::vector<float> feat;        // the learned switch's 8 inputs before each traced step
};

// Learned direction switch (mode BFS_LEARNED): fp32 parameters of the
// 8 -> 64 -> 64 -> 1 policy network (host; stored as bf16), or null to remove.
int bfs_set_policy(const float* params_host);

// Direction switch policy: plain rule (alpha/beta) unless a policy callback
// is installed (learned switch).  Returns 1 for bottom-up.
struct BfsSwitchState {
  uint32_t nf, nf_prev, mf, mu, n, E, level, direction;
};

// Run one BFS from `root` on the device graph; parents/distances are device
// arrays of V entries.  bu_entry_nf selects the nf value at the start of a
// bottom-up phase: 0 as the array-queue DO-BFS (BFS.c:550-551), or the
// frontier size as the bitmap DO-BFS.  want_trace: also copy the per-step
// trace and switch inputs back into res.  want_reached: count the reached
// vertices and their out-edges into res (one more pass over V).
int bfs_run(DevGraph& g, uint32_t root, uint32_t mode, int32_t* parents, uint32_t* distances,
            BfsResult* res, bool want_trace, bool bu_entry_nf_frontier, cudaStream_t s, bool want_reached = true);
// The same from several roots at once (host array): on a disjoint union of
// graphs with one root each, every vertex gets its depth from its own
// graph's root.  The switch state covers the whole union.
int bfs_run_roots(DevGraph& g, const uint32_t* roots, uint32_t nroots, uint32_t mode, int32_t* parents,
                  uint32_t* distances, BfsResult* res, bool want_trace, bool bu_entry_nf_frontier, cudaStream_t s,
                  bool want_reached = true);

// ---- multi-source BFS (batch.cu) -------------------------------------------
struct MsResult {
  uint32_t levels = 0, push_levels = 0, pull_levels = 0, launches = 0;
  unsigned long long reached = 0;         // (vertex, lane) pairs reached, roots included
  unsigned long long edges_examined = 0;  // edges read by the levels
  double ms = 0.0;                        // device time of the levels
  double init_ms = 0.0;                   // device time of the initialisation before them
};
// Up to 64 BFS searches at once, one lane per root; depth[v * 64 + lane] =
// depth of v in that lane's search, 0xFFFF when unreached (V * 64 u16).
int msbfs_run(DevGraph& g, const uint32_t* roots, uint32_t nroots, uint16_t* depth, MsResult* res, cudaStream_t s);

// ---- PageRank over many graphs at once (a disjoint union) -------------------
struct PrBatchDev {
  const uint32_t* voff;   // ngraphs + 1 vertex offsets
  const uint32_t* gid;    // graph of every vertex
  uint32_t* frozen;       // per graph: stopped
  uint32_t* stop_iter;    // per graph: iteration at which it stopped (~0u: did not)
  uint32_t* executed;     // per graph: iterations run
  uint32_t* active_last;  // per graph: active vertices of its last iteration
  double* err_last;       // per graph: error_total of its last iteration
  float* delta;           // per vertex: change in the last iteration
};
int pagerank_batch_run(DevGraph& g, const PrBatchDev& b, uint32_t ngraphs, uint32_t max_iters, double epsilon,
                       float* ranks, cudaGraphExec_t* exec, bool* rebuilt, cudaStream_t s);

// ---- many graphs in one disjoint union (batch.cu) ---------------------------
struct GraphBatch;
struct BatchPrGraph {
  uint32_t iterations, executed, activeVertices, converged;
  double error_total;
};
struct TuneResult {
  uint32_t n = 0, best = 0;
  uint32_t warp_thr[16] = {}, cta_thr[16] = {};
  double ms[16] = {};
};
GraphBatch* batch_new();
void batch_free(GraphBatch* b);
uint32_t batch_ngraphs(const GraphBatch* b);
const uint32_t* batch_voff(const GraphBatch* b);
DevGraph& batch_graph(GraphBatch* b);
// Graphs given by local-id edge lists back to back (edges of graph i at
// [eoff[i], eoff[i+1]) of src/dst, host arrays); nv[i] vertices each.
int batch_create(GraphBatch& b, uint32_t ngraphs, const uint32_t* nv, const uint64_t* eoff, const uint32_t* src,
                 const uint32_t* dst, uint32_t sort_type, cudaStream_t s);
// DO-BFS of every graph from its root (local ids, host array): parents
// (local ids) and distances of all vertices, graph after graph.
int batch_bfs(GraphBatch& b, const uint32_t* roots, int32_t* parents, uint32_t* distances, BfsResult* res,
              cudaStream_t s);
int batch_pagerank(GraphBatch& b, uint32_t max_iters, double epsilon, float* ranks, BatchPrGraph* per_graph,
                   double* ms, uint32_t* captured, cudaStream_t s);
int batch_autotune(GraphBatch& b, uint32_t iters, TuneResult* out, cudaStream_t s);

// ---- the learned parts' networks (mlp.cu) -----------------------------------
int mlp_nparams_host(int in, int h);
int mlp_grad(int in, int h, int loss, const float* X, const float* T, int B, const float* params_host,
             float* grad_host, float* loss_host, cudaStream_t s);
int mlp_train(int in, int h, int loss, const float* X, const float* T, int N, int epochs, int batch, float lr,
              uint32_t seed, float* params_host, float* loss_hist, cudaStream_t s);
int mlp_infer(int in, int h, const float* params_host, const float* X, int N, float* Y, cudaStream_t s);
int pr_warm_start(DevGraph& g, int h, const float* params_host, float* init, cudaStream_t s);

// ---- batched personalized PageRank (batch.cu) -------------------------------
struct PprResult {
  uint32_t executed = 0, converged = 0, launches = 0;
  double ms = 0.0;
  double err_last[32] = {};  // L1 change of each seed's vector in the last iteration
};
// Up to 32 one-hot seeds; ranks (may be null) receives V * 32 floats, row v
// = v's rank in each seed's vector (unnormalized, as the reference's pull).
int ppr_run(DevGraph& g, const uint32_t* seeds, uint32_t nseeds, uint32_t max_iters, double epsilon, float* ranks,
            PprResult* res, cudaStream_t s);

// Depths as bytes (out: V bytes, rounded up to a multiple of 4), for the host
// copy of a search of fewer than 255 levels.  bfs.cu.
int bfs_depth_bytes(uint32_t V, const uint32_t* distances, uint8_t* out, cudaStream_t s);

}  // namespace ogb

// One top-down / bottom-up level over HOST state (the reference's
// topDownStepGraphCSR / bottomUpStepGraphCSR signatures): host arrays are
// copied in, the level runs on the device, results are copied back.
int bfs_td_step_host(ogb::DevGraph& g, const uint32_t* q, uint32_t qsize, int32_t* parents, uint32_t* distances,
                     uint32_t* next_q, uint32_t* next_size, uint32_t* mf, cudaStream_t s);
int bfs_bu_step_host(ogb::DevGraph& g, const uint32_t* bm_cur, uint32_t* bm_next, int32_t* parents,
                     uint32_t* distances, uint32_t* nf, cudaStream_t s);

namespace ogb {

// ---- PageRank ----------------------------------------------------------------
struct PrResult {
  uint32_t iterations = 0;       // PageRankStats.iterations
  uint32_t executed = 0;         // iterations actually run
  uint32_t activeVertices = 0;
  double error_total = 0.0;
  double ms = 0.0;
  uint32_t launches = 0;
  int converged = 0;
  double err_hist[1024];
  uint32_t active_hist[1024];
};

// The reference's PULL_PUSH numbers: 0 pull, 1 push, 6 data-driven pull, 7
// data-driven push, 8 data-driven pull-push.
enum PrMode : uint32_t { PR_PULL = 0, PR_PUSH = 1, PR_DD_PULL = 6, PR_DD_PUSH = 7, PR_DD_PULLPUSH = 8 };

// PageRank with the reference semantics (pageRank.c:939-1186): unnormalized
// start at 1-d, stop when no vertex changes by >= epsilon or after
// max_iters, ranks divided by V at the end.  `ranks` is a device array of V
// floats; `init` (optional, device) replaces the uniform start.
int pagerank_run(DevGraph& g, uint32_t mode, uint32_t max_iters, double epsilon, float* ranks,
                 const float* init, PrResult* res, cudaStream_t s);

// Data-driven PageRank (modes PR_DD_*; pageRank.c:2405-2919), same result
// fields as pagerank_run.  dd.cu.
int pagerank_dd_run(DevGraph& g, uint32_t mode, uint32_t max_iters, double epsilon, float* ranks, PrResult* res,
                    cudaStream_t s);
// SPMV (SPMV.c:588-811): mode 0 pull, 1 push; x receives the input vector
// (1 / out_degree, 0.001 without out-edges), y the output accumulated over
// `iterations` passes.  Device arrays of V floats.  dd.cu.
int spmv_run(DevGraph& g, uint32_t mode, uint32_t iterations, float* x, float* y, double* ms, cudaStream_t s);
// radixSortEdgesByPageRank (reorder.c:165-221) on device arrays: labels
// stably sorted ascending by (uint32_t)(rank * 2^20 + 0.5f).  dd.cu.
int rank_sort(const float* ranks, uint32_t* labels, uint32_t n, cudaStream_t s);
void dd_work_free(const DevGraph* g);
// One pull PageRank iteration over the destination vertices [lo, hi) (a rank
// of a 1-D partition): ranks and contrib_next are written on [lo, hi) only;
// |change| / V and the changes >= epsilon are added to d_err / d_active
// (device, zeroed by the caller).  init: ranks = 1 - 0.85, contrib = that /
// out_degree on all V; finish: ranks /= V.  dd.cu.
int pagerank_range_init(DevGraph& g, float* ranks, float* contrib, cudaStream_t s);
// peers (device array of npeers buffers of V floats, optional): contrib_next
// on [lo, hi) is also stored into each of them.
int pagerank_range_step(DevGraph& g, uint32_t lo, uint32_t hi, const float* contrib, float* ranks,
                        float* contrib_next, double epsilon, double* d_err, uint32_t* d_active, cudaStream_t s,
                        float* const* peers = nullptr, uint32_t npeers = 0);
int pagerank_range_finish(DevGraph& g, float* ranks, cudaStream_t s);
void range_work_free(const DevGraph* g);
// Stable split of an edge-list shard by vertex owner (ranges
// [bounds[r], bounds[r+1]), bounds on the host): each edge to its source's
// owner and, if another, to its destination's owner; out_* hold up to 2 E
// edges, grouped by owner in rank order; counts (host) the edges per owner.
// partition.cu.
int partition_edges(const uint32_t* src, const uint32_t* dst, const float* w, uint32_t E, const uint32_t* bounds,
                    uint32_t nparts, uint32_t* out_src, uint32_t* out_dst, float* out_w, uint32_t* counts,
                    cudaStream_t s);
// One rank's share of a 1-D partitioned DO-BFS over the vertices [lo, hi)
// (ogb_bfs_range_* in ogb200_device.h).  bfs_range.cu.
int bfs_range_init(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t root, int32_t* parents, uint32_t* dist,
                   uint8_t* frontier, uint8_t* visited, int32_t* cand, unsigned long long* counts, cudaStream_t s);
int bfs_range_expand(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                     const uint8_t* frontier, const uint8_t* visited, uint8_t* next, int32_t* cand,
                     int32_t* parents, uint32_t* dist, unsigned long long* counts, cudaStream_t s);
int bfs_range_expand_peers(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                           const uint8_t* frontier, const uint8_t* visited, uint8_t* next, int32_t* const* cand_peers,
                           const uint32_t* bounds, uint32_t nparts, int32_t* parents, uint32_t* dist,
                           unsigned long long* counts, cudaStream_t s);
int bfs_range_claim_peers(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth, int32_t* cand,
                          uint8_t* next, uint8_t* const* next_peers, uint32_t npeers, int32_t* parents,
                          uint32_t* dist, unsigned long long* counts, cudaStream_t s);
int bfs_range_settle(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth, int32_t* cand,
                     uint8_t* next, uint8_t* visited, int32_t* parents, uint32_t* dist, unsigned long long* counts,
                     cudaStream_t s);

// Row-length thresholds of the PageRank work split (light rows per thread,
// heavy rows per warp, very heavy rows per CTA of cta_threads threads).
void pagerank_set_bins(uint32_t warp_thr, uint32_t cta_thr);
void pagerank_get_bins(uint32_t* warp_thr, uint32_t* cta_thr, uint32_t* cta_threads, uint32_t* chunk);

}  // namespace ogb
