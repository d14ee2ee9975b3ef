/*
 * ogb200_device.h -- status-returning device API of libogb200 (no OpenGraph
 * counterpart: this is the layer under the drop-in symbols of ogb200.h).
 *
 * Every function returns 0 on success or a nonzero status (see
 * OGB_ERR_*), with a message in ogb_last_error().  Pointers named d_* are
 * device pointers of the current CUDA device; `stream` is a cudaStream_t
 * (NULL = the legacy default stream, so a call is ordered after the caller's
 * default-stream copies into its inputs).  Nothing here exits the process.
 */
#ifndef OGB200_DEVICE_H
#define OGB200_DEVICE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OGB_OK 0
#define OGB_ERR_CUDA 1
#define OGB_ERR_ARG 2
#define OGB_ERR_SPIN 3
#define OGB_ERR_RANGE 4
#define OGB_ERR_NOMEM 5
#define OGB_ERR_UNSUPPORTED 6
#define OGB_ERR_STATE 7 /* a device-side consistency check failed */

typedef struct ogb_graph ogb_graph; /* device-resident CSR, both directions */

/* One direction of a device CSR (the device image of struct Vertex plus the
 * sorted edge arrays of struct EdgeList). */
typedef struct ogb_csr_view
{
    uint32_t num_vertices;
    uint32_t num_edges;
    uint32_t *src;        /* sorted source ids (E)                    */
    uint32_t *dst;        /* neighbour ids (E)                        */
    float *weight;        /* E, or NULL when unweighted               */
    uint32_t *out_degree; /* V                                        */
    uint32_t *in_degree;  /* V                                        */
    uint32_t *edges_idx;  /* V, 0 for vertices without edges          */
} ogb_csr_view;

typedef struct ogb_bfs_info
{
    uint32_t iteration;        /* BFSStats.iteration                    */
    uint32_t processed_nodes;  /* BFSStats.processed_nodes              */
    uint32_t td_steps;
    uint32_t bu_steps;
    uint32_t reached;          /* vertices with a parent               */
    uint32_t levels;           /* steps recorded in the level trace     */
    uint64_t reached_out_edges;/* sum of out-degrees of reached vertices */
    uint64_t edges_examined;   /* edges read by the steps               */
    double ms;                 /* device time of the traversal          */
    uint32_t launches;         /* kernels launched by the traversal     */
    uint32_t pad;
} ogb_bfs_info;

/* One step of the BFS level trace (ogb_bfs_trace). */
typedef struct ogb_bfs_level
{
    uint32_t direction;  /* 0 top-down, 1 bottom-up */
    uint32_t discovered;
    uint32_t frontier;
    uint32_t mf;
    uint32_t mu;
    uint32_t pad;
    uint64_t edges;
    float ms;
    float pad2;
} ogb_bfs_level;

typedef struct ogb_pr_info
{
    uint32_t iterations;     /* PageRankStats.iterations              */
    uint32_t executed;       /* iterations actually run               */
    uint32_t activeVertices; /* of the last iteration                 */
    uint32_t converged;      /* 1 if an iteration had no active vertex */
    double error_total;      /* of the last iteration                 */
    double ms;               /* device time, init to normalization    */
    uint32_t launches;       /* kernels launched (early-exit ones included) */
    uint32_t pad;
} ogb_pr_info;

const char *ogb_last_error(void);
/* 1 when this build's struct layouts are the WEIGHTED=1 ones. */
int ogb_weighted_layout(void);
/* Silence the reference-style progress tables printed by ogb200.h calls. */
void ogb_set_quiet(int quiet);

/* No counterpart in the reference.  Wall-clock phases, in seconds, of the
 * last breadthFirstSearchGraphCSR-family call: [0] the whole call, [1] stats
 * allocation and the device copy lookup, [2] the device search as the
 * calling thread sees it (launch to result header), [3] writing the DualOrder
 * parent copy's sentinels (host threads, during the search), [4] both of
 * those together, [5] the device-to-host copy of the result into the
 * reference's arrays (depths as bytes, widened on the host; parents whole).  Writes min(n, OGB_DROPIN_BFS_PHASES) values. */
#define OGB_DROPIN_BFS_PHASES 6
int ogb_dropin_bfs_phases(double *seconds, uint32_t n);

int ogb_graph_create(ogb_graph **g);
void ogb_graph_destroy(ogb_graph *g);
/* Sort (SORT_TYPE semantics) and build both CSR directions from device edge
 * arrays; all ids < V <= 2^30.  Inputs are read only.  d_w may be NULL. */
int ogb_graph_build(ogb_graph *g, const uint32_t *d_src, const uint32_t *d_dst, const float *d_w,
                    uint32_t num_edges, uint32_t num_vertices, uint32_t sort_type, void *stream);
int ogb_graph_view(ogb_graph *g, int inverse, ogb_csr_view *view);
/* The device copy the drop-in layer keeps for a host GraphCSR (uploaded on
 * first use); NULL with an error message when it cannot be made. */
ogb_graph *ogb_graph_of(const void *graphCSR);

/* Stable device sort of an edge list with SORT_TYPE semantics. */
int ogb_sort_edges(const uint32_t *d_src, const uint32_t *d_dst, const float *d_w, uint32_t num_edges,
                   uint32_t sort_type, uint32_t *d_out_src, uint32_t *d_out_dst, float *d_out_w, void *stream);

/* BFS from root; mode 0 pull, 1 push, 2 direction-optimized, 3
 * direction-optimized with the learned switch (ogb_bfs_set_policy; depths
 * are the same, the step directions and counts are the policy's), 4 pull
 * with every bottom-up step over all vertices (a cost probe: the learned
 * switch's training data).  d_parents (int32) and d_distances (u32) hold V
 * entries each. */
int ogb_bfs(ogb_graph *g, uint32_t root, uint32_t mode, int32_t *d_parents, uint32_t *d_distances,
            ogb_bfs_info *info, void *stream);
/* Level trace of the last ogb_bfs on g (up to max_levels entries). */
int ogb_bfs_trace(ogb_graph *g, ogb_bfs_level *levels, uint32_t max_levels, uint32_t *count);

/* Learned parts (no reference counterpart).  Networks have one shape: in
 * (<= 8) -> hidden (<= 64, ReLU) -> hidden (ReLU) -> 1; fp32 parameters
 * (host arrays of ogb_mlp_nparams floats) packed as W1[h][in], b1[h],
 * W2[h][h], b2[h], w3[h], b3; inference rounds them to bf16 and accumulates
 * in fp32.  loss 0 = squared error, 1 = binary cross-entropy on the logit.
 * ogb_mlp_grad: the batch-mean loss and its gradient (host) for d_X (batch
 * x in) and d_T (batch).  ogb_mlp_train: Adam on shuffled mini-batches,
 * params in/out; loss_hist (may be NULL) gets the mean loss per epoch. */
uint32_t ogb_mlp_nparams(uint32_t in, uint32_t hidden);
int ogb_mlp_grad(uint32_t in, uint32_t hidden, uint32_t loss, const float *d_X, const float *d_T, uint32_t batch,
                 const float *params, float *grad, float *loss_out, void *stream);
int ogb_mlp_train(uint32_t in, uint32_t hidden, uint32_t loss, const float *d_X, const float *d_T, uint32_t n,
                  uint32_t epochs, uint32_t batch, float lr, uint32_t seed, float *params, float *loss_hist,
                  void *stream);
int ogb_mlp_infer(uint32_t in, uint32_t hidden, const float *params, const float *d_X, uint32_t n, float *d_Y,
                  void *stream);
/* The learned direction switch used by ogb_bfs mode 3.  params holds the
 * 8 -> 64 -> 64 -> 1 network in the ogb_mlp packing (4801 floats) followed by
 * a linear prior: 8 coefficients, a bias and a bound B (4811 floats in all).
 * A step runs bottom-up when  prior . x + bias + clamp(network(x), -B, B) > 0,
 * so the network is a bounded correction of the prior; NULL removes it.  The
 * inputs x, before every step (L(x) = log2(1 + x)): L(frontier vertices),
 * L(frontier out-edges), L(unexplored out-edges), L(bottom-up candidates:
 * the list a bottom-up step would walk -- the graph's vertices with in-edges
 * before the first bottom-up step, the unvisited list after it; V in mode 4),
 * L(V), L(frontier) - L(previous frontier), visited fraction, 1 when a
 * bottom-up step would walk a list (else 0). */
int ogb_bfs_set_policy(const float *params);
/* Those inputs for every step of the last ogb_bfs on g (count x 8 floats). */
int ogb_bfs_features(ogb_graph *g, float *features, uint32_t max_levels, uint32_t *count);
/* PageRank warm start: a 2 -> hidden -> hidden -> 1 network of
 * log2(1 + in_degree), log2(1 + out_degree) predicts log2 of each vertex's
 * unnormalized rank; d_init (V floats) = 2^prediction, for ogb_pagerank's
 * d_init. */
int ogb_pagerank_warm_start(ogb_graph *g, uint32_t hidden, const float *params, float *d_init, void *stream);

/* Multi-source BFS (no reference counterpart: a batch of the reference's
 * single-root searches, BFS.c:476-626).  Up to 64 roots (host array), one
 * bit-lane each; d_depths (device, V * 64 uint16) receives, for vertex v and
 * lane i, d_depths[v * 64 + i] = v's depth in the search from roots[i], or
 * 0xFFFF when unreached.  Every lane's depths equal the single-root BFS
 * distances of that root. */
typedef struct ogb_msbfs_info
{
    uint32_t levels;           /* levels until every frontier emptied     */
    uint32_t push_levels;
    uint32_t pull_levels;
    uint32_t launches;
    uint64_t reached_pairs;    /* (vertex, lane) pairs reached, roots too */
    uint64_t edges_examined;
    double ms;                 /* device time of the levels (the search)  */
    double init_ms;            /* device time of the initialisation before
                                  it: depth fill, per-vertex words cleared,
                                  roots set (as the single-root search's
                                  initialisation precedes its timed part) */
} ogb_msbfs_info;
int ogb_msbfs(ogb_graph *g, const uint32_t *roots, uint32_t nroots, uint16_t *d_depths, ogb_msbfs_info *info,
              void *stream);

/* Batched personalized PageRank (no reference counterpart: the reference's
 * pull PageRank, pageRank.c:984-1044, with the teleport term replaced by
 * (1 - 0.85) on the seed vertex only).  Up to 32 seeds (host array), one
 * vector each, started from the seed's one-hot vector; d_ranks (device, may
 * be NULL) receives V * 32 floats, d_ranks[v * 32 + k] = v's (unnormalized)
 * rank in seed k's vector.  Stops after an iteration in which every vector
 * changed by < epsilon (L1), or after max_iterations. */
typedef struct ogb_ppr_info
{
    uint32_t executed;         /* iterations run                          */
    uint32_t converged;        /* 1 when the epsilon rule stopped the run */
    uint32_t launches;
    uint32_t pad;
    double ms;                 /* device time                             */
    double err_last[32];       /* last L1 change of each seed's vector    */
} ogb_ppr_info;
int ogb_ppr(ogb_graph *g, const uint32_t *seeds, uint32_t nseeds, uint32_t max_iterations, double epsilon,
            float *d_ranks, ogb_ppr_info *info, void *stream);

/* Many graphs in one (no reference counterpart: each graph's results equal
 * the reference path run on that graph alone).  The graphs are packed into
 * one disjoint union on the device; BFS of all of them is one launch and
 * PageRank of all of them one CUDA graph, each graph with its own stop rule
 * and normalization.  Edge lists use local ids, back to back: graph i's
 * edges are src/dst[edge_offsets[i] .. edge_offsets[i+1]) (host arrays),
 * ids < num_vertices[i].  Vertex arrays of the batch (parents, distances,
 * ranks) hold the graphs' vertices back to back (ogb_batch_offsets). */
typedef struct ogb_batch ogb_batch;
ogb_batch *ogb_batch_create(uint32_t num_graphs, const uint32_t *num_vertices, const uint64_t *edge_offsets,
                            const uint32_t *src, const uint32_t *dst, uint32_t sort_type);
void ogb_batch_free(ogb_batch *b);
/* vertex_offsets: num_graphs + 1 entries (host) */
int ogb_batch_offsets(ogb_batch *b, uint32_t *vertex_offsets);
typedef struct ogb_batch_bfs_info
{
    uint32_t levels;           /* steps of the joint search              */
    uint32_t td_steps;
    uint32_t bu_steps;
    uint32_t reached;          /* vertices reached, all graphs           */
    double ms;                 /* device time of the search              */
} ogb_batch_bfs_info;
/* DO-BFS of every graph from roots[i] (local id, host array); d_parents
 * (local ids, sentinel -out_degree / -1 for unreached) and d_distances. */
int ogb_batch_bfs(ogb_batch *b, const uint32_t *roots, int32_t *d_parents, uint32_t *d_distances,
                  ogb_batch_bfs_info *info, void *stream);
typedef struct ogb_batch_pr_graph
{
    uint32_t iterations;       /* PageRankStats.iterations of the graph   */
    uint32_t executed;
    uint32_t activeVertices;
    uint32_t converged;
    double error_total;
} ogb_batch_pr_graph;
typedef struct ogb_batch_pr_info
{
    double ms;                 /* device time of the graph launch         */
    uint32_t captured;         /* 1 when this call (re)built the graph    */
    uint32_t pad;
} ogb_batch_pr_info;
/* Pull PageRank of every graph; d_ranks receives the normalized ranks of all
 * vertices; per_graph (host, num_graphs entries, may be NULL). */
int ogb_batch_pagerank(ogb_batch *b, uint32_t max_iterations, double epsilon, float *d_ranks,
                       ogb_batch_pr_graph *per_graph, ogb_batch_pr_info *info, void *stream);
typedef struct ogb_tune_info
{
    uint32_t ncandidates;
    uint32_t best;             /* index of the chosen candidate           */
    uint32_t warp_thr[16];
    uint32_t cta_thr[16];
    double ms[16];             /* pull ms per iteration of each candidate */
} ogb_tune_info;
/* Times the pull PageRank bin thresholds on this batch and keeps the
 * fastest (ogb_pagerank_set_bins). */
int ogb_batch_autotune(ogb_batch *b, ogb_tune_info *info);

/* PageRank; mode = the reference's PULL_PUSH value: 0 pull, 1 push, 6
 * data-driven pull, 7 data-driven push, 8 data-driven pull-push
 * (pageRank.c:939-1186, 2405-2919).  d_ranks receives V normalized ranks;
 * d_init (may be NULL; modes 0 and 1 only) replaces the uniform unnormalized
 * start 1-0.85. */
int ogb_pagerank(ogb_graph *g, uint32_t mode, uint32_t max_iterations, double epsilon, float *d_ranks,
                 const float *d_init, ogb_pr_info *info, void *stream);

typedef struct ogb_spmv_info
{
    uint32_t iterations;
    uint32_t weighted; /* 1: the graph's edge weights were used, 0: 0.0001 each */
    double ms;         /* device time of the iterations */
} ogb_spmv_info;
/* SPMV (SPMV.c:588-811); mode 0 pull, 1 push.  d_x receives the input
 * vector (1 / out_degree, 0.001 without out-edges), d_y the output summed
 * over `iterations` passes (never reset between them, as the reference).
 * Device arrays of V floats. */
int ogb_spmv(ogb_graph *g, uint32_t mode, uint32_t iterations, float *d_x, float *d_y, ogb_spmv_info *info,
             void *stream);
/* 1-D partitioned PageRank pull (no counterpart in the reference; its
 * iteration is pageRank.c:984-1044).  A rank owns the destination vertices
 * [lo, hi).  range_init: d_ranks = 1 - 0.85 and d_contrib = that /
 * out_degree on all V.  range_step: one iteration over [lo, hi) with the
 * whole previous d_contrib; writes d_ranks and d_contrib_next on [lo, hi)
 * only and adds |change| / V and the count of changes >= epsilon to the
 * DEVICE scalars *d_err / *d_active (zeroed by the caller).  Each row is
 * summed in the same order as ogb_pagerank pull at its default thresholds,
 * so any partition gives the same ranks bit for bit.  range_finish: d_ranks
 * /= V.  The caller all-gathers d_contrib_next's slices between steps
 * (opengraph_b200.parallel does this over torch.distributed). */
int ogb_pagerank_range_init(ogb_graph *g, float *d_ranks, float *d_contrib, void *stream);
int ogb_pagerank_range_step(ogb_graph *g, uint32_t lo, uint32_t hi, const float *d_contrib, float *d_ranks,
                            float *d_contrib_next, double epsilon, double *d_err, uint32_t *d_active, void *stream);
int ogb_pagerank_range_finish(ogb_graph *g, float *d_ranks, void *stream);
/* range_step with the all-gather fused in: d_peers is a DEVICE array of
 * npeers addresses of V-float buffers (the ranks' next-contrib buffers,
 * e.g. symmetric memory mapped over NVLink; this rank's own may be among
 * them); every contrib of [lo, hi) is stored into each of them as it is
 * computed, then ordered by a system-scope fence, so the caller needs only a
 * barrier across the ranks before the next step reads them. */
int ogb_pagerank_range_step_peers(ogb_graph *g, uint32_t lo, uint32_t hi, const float *d_contrib, float *d_ranks,
                                  float *d_contrib_next, const uint64_t *d_peers, uint32_t npeers, double epsilon,
                                  double *d_err, uint32_t *d_active, void *stream);
/* Graph build across several GPUs (no counterpart in the reference, which
 * sorts one edge list: radixsort.c:46-335, graphCSR.c:107-248).  Ranks own
 * the vertex ranges [bounds[r], bounds[r+1]) (bounds: nparts + 1 ascending
 * HOST values from 0; nparts <= 64).  ogb_partition_edges splits a rank's
 * edge-list shard (device arrays of E, d_w may be NULL): every edge goes to
 * its source's owner and, when that is another rank, to its destination's
 * owner.  d_out_* (capacity 2 E) receive, per owner in rank order, first the
 * edges it owns by source then those it owns by destination only, each in
 * shard order; counts (HOST, nparts) the edges per owner.  After an
 * all-to-all of these segments, ogb_graph_build on the received edges (in
 * sender order, with the global V) gives every owned vertex the out-row and
 * in-row, in the same order, of the graph of the whole edge list (the
 * shards concatenated in rank order).  ERR_RANGE if an id is >= bounds[nparts].
 * Synchronizes the stream. */
int ogb_partition_edges(const uint32_t *d_src, const uint32_t *d_dst, const float *d_w, uint32_t E,
                        const uint32_t *bounds, uint32_t nparts, uint32_t *d_out_src, uint32_t *d_out_dst,
                        float *d_out_w, uint32_t *counts, void *stream);
/* 1-D partitioned direction-optimizing BFS (no counterpart in the
 * reference; its loop is BFS.c:476-626).  A rank owns the vertices [lo, hi):
 * their parents and depths (d_parents, d_dist: V entries, written on
 * [lo, hi) only), their out-rows for top-down steps and in-rows for
 * bottom-up steps.  d_frontier, d_next and d_visited are V bytes (0/1) and
 * d_cand V int32, the same on every rank.
 * bfs_range_init: d_frontier = d_visited = {root}; d_cand = 0x7F7F7F7F
 * everywhere (it is so again after every step); d_parents / d_dist on
 * [lo, hi) as the reference initialises them (BFS.c:58-74: -out_degree, or
 * -1 without out-edges; depth 0; the root its own parent); d_counts =
 * {1, out_degree(root), 0, 0} on the rank that owns the root and zeros on
 * the others (summed over the ranks: the first frontier's size and mf,
 * BFS.c:511).  g may hold the whole graph or, built from
 * ogb_partition_edges' output, only the rows of the owned vertices.
 * A step at depth `depth` (1 for the first) in `direction` (0 top-down,
 * 1 bottom-up) is bfs_range_expand, an all-reduce by the caller across the
 * ranks (top-down: MIN over d_cand; bottom-up: MAX over d_next), then
 * bfs_range_settle; d_next is then the next frontier.
 * expand zeroes d_counts (4 u64, device).  Top-down: d_cand[w] =
 * min(d_cand[w], u) for every unvisited
 * out-neighbour w of an owned frontier vertex u.  Bottom-up: d_next zeroed;
 * each owned unvisited vertex takes its first in-neighbour in the frontier,
 * in CSR order, as parent (BFS.c:703-754), sets its d_next byte and adds
 * itself to d_counts[0] and its examined in-edges to d_counts[2].
 * settle: top-down, d_next[v] = (d_cand[v] != 0x7F7F7F7F), and each owned
 * such vertex takes d_cand[v] as parent (its smallest frontier
 * in-neighbour) and the depth, adding itself to d_counts[0] and
 * max(out_degree, 1) to d_counts[1] (the mf of BFS.c:675), and d_cand is
 * reset to 0x7F7F7F7F; both
 * directions: d_visited |= d_next.  d_counts[3] != 0 reports an overflow of
 * the library's step queue (sized for the worst case).  Neither call
 * synchronizes its stream.  opengraph_b200.parallel holds the direction
 * switch of BFS.c:546-587. */
int ogb_bfs_range_init(ogb_graph *g, uint32_t lo, uint32_t hi, uint32_t root, int32_t *d_parents, uint32_t *d_dist,
                       uint8_t *d_frontier, uint8_t *d_visited, int32_t *d_cand, uint64_t *d_counts, void *stream);
int ogb_bfs_range_expand(ogb_graph *g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                         const uint8_t *d_frontier, const uint8_t *d_visited, uint8_t *d_next, int32_t *d_cand,
                         int32_t *d_parents, uint32_t *d_dist, uint64_t *d_counts, void *stream);
int ogb_bfs_range_settle(ogb_graph *g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                         int32_t *d_cand, uint8_t *d_next, uint8_t *d_visited, int32_t *d_parents,
                         uint32_t *d_dist, uint64_t *d_counts, void *stream);
/* The same search with the exchange fused into the steps (no all-reduce of
 * cand or next).  d_cand and the two next buffers are memory every rank maps
 * (e.g. symmetric memory over NVLink), 4-byte aligned; d_cand_peers /
 * d_next_peers are DEVICE arrays of every rank's address of them (rank
 * order), d_bounds a DEVICE array of the nparts + 1 range bounds.  A step:
 * ogb_bfs_range_expand_peers (top-down: each candidate goes straight to the
 * cand array of its vertex's owner by atomicMin; bottom-up: as
 * ogb_bfs_range_expand, zeroing only the owned next bytes), then for a
 * top-down step a barrier across the ranks, then ogb_bfs_range_claim_peers
 * (top-down: the owned vertices with a candidate are reached -- parent =
 * the smallest frontier in-neighbour, depth, d_counts -- and d_cand is put
 * back; both: the owned next bytes are stored into every rank's next
 * buffer), a barrier, and ogb_bfs_range_settle with direction 1 (visited |=
 * next).  Both calls end with a system-scope fence; the caller's barrier
 * must order them across the GPUs. */
int ogb_bfs_range_expand_peers(ogb_graph *g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                               const uint8_t *d_frontier, const uint8_t *d_visited, uint8_t *d_next,
                               const uint64_t *d_cand_peers, const uint32_t *d_bounds, uint32_t nparts,
                               int32_t *d_parents, uint32_t *d_dist, uint64_t *d_counts, void *stream);
int ogb_bfs_range_claim_peers(ogb_graph *g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                              int32_t *d_cand, uint8_t *d_next, const uint64_t *d_next_peers, uint32_t npeers,
                              int32_t *d_parents, uint32_t *d_dist, uint64_t *d_counts, void *stream);
/* radixSortEdgesByPageRank (reorder.c:165-221) on device arrays: d_labels
 * stably sorted in place, ascending by (uint32_t)(rank * 2^20 + 0.5f). */
int ogb_sort_by_rank(const float *d_ranks, uint32_t *d_labels, uint32_t n, void *stream);
/* Work split of the PageRank kernels by row length: rows of at most warp_thr
 * edges are reduced by one thread in CSR order (the reference's summation
 * order), longer rows by a warp, rows above cta_thr by a CTA of cta_threads
 * threads (fixed-order butterfly sums).  Defaults 32 / 2048 / 256. */
void ogb_pagerank_set_bins(uint32_t warp_thr, uint32_t cta_thr);
void ogb_pagerank_get_bins(uint32_t *warp_thr, uint32_t *cta_thr, uint32_t *cta_threads, uint32_t *chunk_edges);
/* Per-iteration L1 error and active count of the last ogb_pagerank on g. */
int ogb_pagerank_history(ogb_graph *g, double *errors, uint32_t *active, uint32_t max_entries, uint32_t *count);

/* No counterpart in the reference.  PageRank pull that allocates no memory,
 * for callers that cannot allocate device memory when they need the result:
 * another allocator or pool owns the device memory, or their request path
 * must not call cudaMalloc (it synchronizes the device and can fail when
 * memory is fragmented).  All scratch is one fixed __device__ array inside
 * the library, about 12.6 MB held on every GPU that loads the library until
 * the process exits; so num_vertices is limited to OGB_NOALLOC_MAX_VERTICES
 * and a larger graph is rejected with OGB_ERR_RANGE.
 * Inputs (device arrays): the inverse CSR -- row starts d_in_edges_idx,
 * in-degrees d_in_degree, in-neighbour ids d_in_neighbors -- and the forward
 * out-degrees.  Outputs: d_ranks (V normalized ranks) and, if d_info is not
 * NULL, a DEVICE ogb_pr_info (ms and launches are 0).  Same semantics as
 * ogb_pagerank pull; rows of at most 2048 in-edges are summed in the same
 * order as its default thresholds give, longer rows by one 256-thread CTA
 * (ogb_pagerank cuts them into chunks), so the ranks can differ in the last
 * bits: they agree with ogb_pagerank and with the reference's sequential
 * order within 1e-6 L1 at the same iteration count.
 * The work is enqueued on `stream` (NULL = the default stream) and the call
 * returns without waiting.  The first call on each device looks up the
 * scratch address: make that first call before any stream capture.  Every
 * call shares the one scratch array and overwrites what the last call left
 * in it, so calls that overlap on the GPU race with each other. */
#define OGB_NOALLOC_MAX_VERTICES (1u << 20)
int ogb_pagerank_pull_noalloc(uint32_t num_vertices, const uint32_t *d_in_edges_idx, const uint32_t *d_in_degree,
                              const uint32_t *d_in_neighbors, const uint32_t *d_out_degree, uint32_t max_iterations,
                              double epsilon, float *d_ranks, ogb_pr_info *d_info, void *stream);

/* ---- synthetic inputs (host, multi-threaded, deterministic) ------------- */

/* RMAT (a, b, c; d = 1-a-b-c) with 2^scale vertices and edge_factor*2^scale
 * edges, counter-based RNG keyed by seed, ids relabelled by a seeded random
 * permutation when permute != 0.  Weights (if w != NULL) uniform in [1,256). */
int ogb_generate_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b, double c,
                      int permute, uint32_t *src, uint32_t *dst, float *w);
/* Erdos-Renyi: num_edges uniform (src, dst) pairs over num_vertices ids. */
int ogb_generate_uniform(uint32_t num_vertices, uint64_t num_edges, uint64_t seed, uint32_t *src, uint32_t *dst,
                         float *w);
/* side x side 4-neighbour grid (both directions) plus, per vertex with
 * probability p, a diagonal shortcut to (r+1, c+1) and back.  Returns the edge count in
 * *num_edges; call with src == NULL to get the capacity needed. */
int ogb_generate_grid(uint32_t side, double p, uint64_t seed, uint32_t *src, uint32_t *dst, float *w,
                      uint64_t *num_edges);
/* Write {u32 src, u32 dst[, f32 w]} records (the reference .bin / .wbin). */
int ogb_write_edge_file(const char *path, const uint32_t *src, const uint32_t *dst, const float *w,
                        uint64_t num_edges);

#ifdef __cplusplus
}
#endif

#endif /* OGB200_DEVICE_H */
