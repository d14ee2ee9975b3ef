/*
 * og_oracle.h -- CPU restatement of the OpenGraph CSR hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg compare the GPU library against.  Nothing in
 * opengraph_b200/ links, loads or calls it.
 *
 * Sequential, plain-array restatement of the reference functions cited at
 * each entry point (paths relative to the OpenGraph tree).  Pinned against
 * the reference's own build (oracle/_ref) by tests/test_oracle.py, and
 * against the committed fixtures under tests/golden/.
 */
#ifndef OG_ORACLE_H
#define OG_ORACLE_H

#include <stdint.h>

/* Stable sort of (src, dst[, w]) -- mode 0: by src (radixsort.c:231-278,
 * countsort.c:28-140), 1: by (src, dst) (radixsort.c:282-335,
 * countsort.c:262-270), 2: by dst (countsort.c:143-259).  w may be NULL. */
void orc_sort(uint32_t E, const uint32_t *src, const uint32_t *dst, const float *w, int mode,
              uint32_t *osrc, uint32_t *odst, float *ow);

/* mapVerticesWithInOutDegree (vertex.c:204-325) for one direction: run
 * lengths and run starts of the sorted src array (edges_idx = 0 for vertices
 * without edges).  Returns -1 if a source id is >= V. */
int orc_csr_map(uint32_t E, uint32_t V, const uint32_t *sorted_src, uint32_t *out_degree, uint32_t *edges_idx);

/* graphCSRPreProcessingStep's sort + map + inverse (graphCSR.c:164-248)
 * without file I/O: f_* forward arrays, i_* inverse arrays (E or V each);
 * in_degree arrays are the other direction's out_degree (vertex.c:291-311).
 * sort_type as SORT_TYPE (0/2 by src, 1/3 by (src,dst)).  w may be NULL, then
 * f_w/i_w are ignored. */
int orc_build(uint32_t E, uint32_t V, const uint32_t *src, const uint32_t *dst, const float *w, int sort_type,
              uint32_t *f_src, uint32_t *f_dst, float *f_w, uint32_t *f_outdeg, uint32_t *f_indeg, uint32_t *f_idx,
              uint32_t *i_src, uint32_t *i_dst, float *i_w, uint32_t *i_outdeg, uint32_t *i_indeg, uint32_t *i_idx);

/* removeDulpicatesSelfLoopEdges (edgeList.c:138-211) on a sorted list;
 * truncate_w reproduces the WEIGHTED layout's uint32 temporary.  Returns the
 * kept count. */
uint32_t orc_dedup(uint32_t E, const uint32_t *s, const uint32_t *d, const float *w, uint32_t *os, uint32_t *od,
                   float *ow, int truncate_w);

typedef struct orc_bfs_stats
{
    uint32_t iteration;       /* BFSStats.iteration       */
    uint32_t processed_nodes; /* BFSStats.processed_nodes */
    uint32_t td_steps;
    uint32_t bu_steps;
    uint32_t reached;
    uint64_t reached_out_edges;
} orc_bfs_stats;

/* BFS over both CSRs (BFS.c:281-754): mode 0 pull, 1 push, 2 direction-
 * optimized (alpha 15, beta 18).  bu_entry_nf_frontier = 0 follows the
 * array-queue DO-BFS (nf = 0 entering bottom-up), 1 the bitmap variant.
 * Top-down parents are the first discoverer in queue order.  dirs (may be
 * NULL) receives the direction of each step (0 TD, 1 BU), up to max_dirs. */
int orc_bfs(uint32_t V, uint32_t E, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
            const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, uint32_t root, int mode,
            int bu_entry_nf_frontier, int32_t *parents, uint32_t *dist, orc_bfs_stats *st, uint8_t *dirs,
            uint32_t max_dirs);

/* PageRank fp32 (pageRank.c:939-1186): mode 0 pull (sequential sums in CSR
 * order), 1 push (sequential scatter in vertex order), 2 pull in the GPU
 * kernel's reduction order (orc_set_gpu_order).  init (may be NULL)
 * replaces the start 1-0.85f.  ranks receives the normalized ranks;
 * err_hist/active_hist (may be NULL) one entry per executed iteration.
 * Returns the number of executed iterations. */
uint32_t orc_pagerank(uint32_t V, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
                      const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, int mode,
                      uint32_t max_iters, double epsilon, const float *init, float *ranks,
                      uint32_t *iterations_out, double *error_out, double *err_hist, uint32_t *active_hist);

/* mode 2 of orc_pagerank: pull with the GPU kernel's reduction order for
 * rows above the given in-degree thresholds (see og_oracle.c). */
void orc_set_gpu_order(uint32_t warp_thr, uint32_t cta_thr, uint32_t cta_threads, uint32_t chunk);

/* The same pull iteration in double precision throughout (the FP64 oracle the
 * fp32 error is stated against).  Runs exactly `iters` iterations. */
void orc_pagerank_f64(uint32_t V, const uint32_t *f_outdeg, const uint32_t *i_outdeg, const uint32_t *i_idx,
                      const uint32_t *i_dst, uint32_t iters, const double *init, double *ranks);

/* generateRandomRootGraphCSR (graphRun.c:537-556) with MT19937 seeded as
 * initializeMersenneState (mt19937.c:54-67): n roots drawn in sequence. */
void orc_random_roots(uint32_t seed, uint32_t V, uint32_t avg_degree, const uint32_t *out_degree, uint32_t n,
                      uint32_t *roots);

/* The benchmark's seeded RMAT edge list (the product's ogb_generate_rmat,
 * restated so the timed reference arm needs no product library).  Returns -1
 * on bad sizes. */
int orc_generate_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b, double c,
                      int permute, uint32_t *src, uint32_t *dst, float *w);

/* Data-driven PageRank (pageRank.c:2405-2919): mode 6 pull, 7 push, 8
 * pull-push, sequential in vertex order; gpu_order (mode 6) sums long
 * in-rows in the GPU kernels' order.  Ranks normalized; returns the executed
 * iterations. */
uint32_t orc_pagerank_dd(uint32_t V, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
                         const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, int mode,
                         int gpu_order, uint32_t max_iters, double epsilon, float *pr, uint32_t *iterations_out,
                         double *error_out, uint32_t *active_hist);

/* SPMV (SPMV.c:616-810): mode 0 pull, 1 push; w may be NULL (0.0001). */
void orc_spmv(uint32_t V, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
              const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, const float *w, int mode,
              int gpu_order, uint32_t iters, float *x, float *y);

/* One pull iteration over the destination range [lo, hi) of a 1-D
 * partition (pageRank.c:984-1044 restricted to the range). */
void orc_pull_range_step(uint32_t V, const uint32_t *f_outdeg, const uint32_t *i_outdeg, const uint32_t *i_idx,
                         const uint32_t *i_dst, uint32_t lo, uint32_t hi, const float *contrib, float *pr,
                         float *contrib_next, double epsilon, int gpu_order, double *err, uint32_t *active);

/* One rank's share of a 1-D partitioned DO-BFS step over the owned
 * vertices [lo, hi) (the steps of BFS.c:639-687 and BFS.c:703-754
 * restricted to the range); frontier, next and visited are V bytes, cand
 * V int32.  init: parents / dist on [lo, hi) as BFS.c:58-74; frontier =
 * visited = {root}; cand = 0x7F7F7F7F (and again after every step).
 * expand: counts zeroed; top-down, cand[w] = min(cand[w], u) over the
 * unvisited out-neighbours w of
 * owned frontier vertices u; bottom-up, next zeroed, each owned unvisited
 * vertex takes its first frontier in-neighbour in CSR order (counts[0]
 * found, counts[2] in-edges examined).  settle (after the exchange: MIN of
 * cand, or MAX of next): top-down, next = cand set, the owned such vertices
 * take cand as parent (counts[0] found, counts[1] sum of
 * max(out_degree, 1), the mf of BFS.c:675), cand reset; visited |= next. */
void orc_bfs_range_init(uint32_t V, const uint32_t *f_outdeg, uint32_t lo, uint32_t hi, uint32_t root,
                        int32_t *parents, uint32_t *dist, uint8_t *frontier, uint8_t *visited, int32_t *cand);
void orc_bfs_range_expand(uint32_t V, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
                          const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, uint32_t lo,
                          uint32_t hi, int direction, uint32_t depth, const uint8_t *frontier, const uint8_t *visited,
                          uint8_t *next, int32_t *cand, int32_t *parents, uint32_t *dist, uint64_t *counts);
void orc_bfs_range_settle(uint32_t V, const uint32_t *f_outdeg, uint32_t lo, uint32_t hi, int direction,
                          uint32_t depth, int32_t *cand, uint8_t *next, uint8_t *visited, int32_t *parents,
                          uint32_t *dist, uint64_t *counts);

/* radixSortEdgesByPageRank (reorder.c:165-221), in place. */
void orc_rank_sort(uint32_t n, const float *ranks, uint32_t *labels);

#endif
