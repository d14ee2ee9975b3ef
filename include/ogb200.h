/*
 * ogb200.h -- C ABI of the B200 CSR hot path (drop-in for OpenGraph's C API).
 *
 * Every struct below has the byte layout of the OpenGraph struct of the same
 * name, and every function has the OpenGraph signature it replaces, so an
 * OpenGraph driver links against libogb200.so without a source change.  The
 * struct layouts are an interface that has to be identical: the field order
 * and types follow the cited reference headers, nothing else is shared.
 *
 * Layout switch: OGB200_WEIGHTED selects the WEIGHTED=1 layout of OpenGraph
 * (00_graph_bench/include/config/graphConfig.h:7).  libogb200.so is built
 * with OGB200_WEIGHTED=0 and libogb200_w.so with OGB200_WEIGHTED=1.
 * DIRECTED=1 (graphConfig.h:8) is the only supported layout.
 *
 * Ownership: every struct and array returned here is allocated with malloc
 * and released by the caller with free() (or the matching free* function),
 * as in OpenGraph (00_graph_bench/src/utils/myMalloc.c:54-66).  Device copies
 * of a GraphCSR are cached by the library and released by graphCSRFree().
 *
 * Errors: as in OpenGraph there are no return codes at this layer.  I/O
 * failures print a message and exit(1); a CUDA failure prints the CUDA error
 * and exits(1).  The status-returning device API is in ogb200_device.h.
 */
#ifndef OGB200_H
#define OGB200_H

#include <stdint.h>

#ifndef OGB200_WEIGHTED
#define OGB200_WEIGHTED 0
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- structs (layout-identical to OpenGraph) --------------------------- */

/* 00_graph_bench/include/utils/mt19937.h:56-60 (unsigned long words). */
typedef struct mt19937_stateStruct
{
    unsigned long mt[624];
    int mti;
} mt19937state;

/* 00_graph_bench/include/config/graphConfig.h:11-44 */
struct Arguments
{
    int wflag;
    int xflag;
    int sflag;
    int Sflag;
    int dflag;                 /* remove duplicates + self loops            */
    uint32_t binSize;
    uint32_t verbosity;
    uint32_t iterations;       /* NUM_ITERATIONS                            */
    uint32_t trials;
    double epsilon;            /* TOLERANCE                                 */
    int source;                /* ROOT                                      */
    uint32_t algorithm;
    uint32_t datastructure;
    uint32_t pushpull;         /* PULL_PUSH                                 */
    uint32_t sort;             /* SORT_TYPE                                 */
    uint32_t lmode;
    uint32_t lmode_l2;
    uint32_t lmode_l3;
    uint32_t mmode;
    uint32_t symmetric;
    uint32_t weighted;
    uint32_t delta;
    int pre_numThreads;
    int algo_numThreads;
    int ker_numThreads;
    char *fnameb;
    char *fnamel;
    uint32_t fnameb_format;
    uint32_t convert_format;
    mt19937state mt19937var;
    uint32_t cache_size;
};

/* 00_graph_bench/include/structures/edgeList.h:8-23 */
struct EdgeList
{
    uint32_t num_edges;
    uint32_t num_vertices;
    uint32_t avg_degree;
#if OGB200_WEIGHTED
    float max_weight;
    float *edges_array_weight;
#endif
    uint32_t *edges_array_src;
    uint32_t *edges_array_dest;
    uint32_t *mask_array;
    uint32_t *label_array;
    uint32_t *inverse_label_array;
};

/* 00_graph_bench/include/structures/vertex.h:13-18 */
struct Vertex
{
    uint32_t *out_degree;
    uint32_t *in_degree;
    uint32_t *edges_idx;
};

/* 00_graph_bench/include/structures/graphCSR.h:12-29 (DIRECTED=1) */
struct GraphCSR
{
    uint32_t num_edges;
    uint32_t num_vertices;
    uint32_t avg_degree;
#if OGB200_WEIGHTED
    float max_weight;
#endif
    struct Vertex *vertices;
    struct EdgeList *sorted_edges_array;
    struct Vertex *inverse_vertices;
    struct EdgeList *inverse_sorted_edges_array;
};

/* 00_graph_bench/include/algorithms/openmp/BFS.h:19-29 */
struct BFSStats
{
    uint32_t *distances;
    int *parents;
    uint32_t *distances_DualOrder;
    int *parents_DualOrder;
    uint32_t processed_nodes;
    uint32_t num_vertices;
    uint32_t iteration;
    double time_total;
};

/* 00_graph_bench/include/algorithms/openmp/pageRank.h:19-30 */
struct PageRankStats
{
    float damp;
    float base_pr;
    uint32_t iterations;
    uint32_t num_vertices;
    uint32_t activeVertices;
    uint32_t *realRanks;
    float *pageRanks;
    double time_total;
    double error_total;
};

/* 00_graph_bench/include/algorithms/openmp/SPMV.h:19-27 */
struct SPMVStats
{
    uint32_t iterations;
    struct Arguments *arguments;
    uint32_t num_vertices;
    float *vector_output;
    float *vector_input;
    double time_total;
};

/* 00_graph_bench/include/structures/bitmap.h:19-26 */
struct Bitmap
{
    uint32_t real_size;
    uint32_t size;
    uint32_t numSetBits;
    uint32_t *bitarray;
};

/* 00_graph_bench/include/structures/arrayQueue.h:7-16 */
struct ArrayQueue
{
    uint32_t head;
    uint32_t tail;
    uint32_t tail_next;
    uint32_t size;
    uint32_t *queue;
    struct Bitmap *q_bitmap;
    struct Bitmap *q_bitmap_next;
};

/* ---- edge lists (host side of the path) ------------------------------- */

/* 00_graph_bench/include/structures/edgeList.h:30 ; edgeList.c:336-594.
 * mmap reader of {u32 src, u32 dst[, f32 w]} records; V = max id + 1. */
struct EdgeList *readEdgeListsbin(const char *fname, uint8_t inverse,
                                  uint32_t symmetric, uint32_t weighted);
/* edgeList.h:31 ; edgeList.c:597-745.  Copy (inverse=1: src/dst swapped). */
struct EdgeList *readEdgeListsMem(struct EdgeList *edgeListmem, uint8_t inverse,
                                  uint32_t symmetric, uint32_t weighted);
/* edgeList.h:32 ; edgeList.c:98-135.  Zero-filled list of num_edges edges. */
struct EdgeList *newEdgeList(uint32_t num_edges);
/* edgeList.h:27 ; edgeList.c:213-239. */
void freeEdgeList(struct EdgeList *edgeList);
/* edgeList.h:34 ; edgeList.c:138-211.  GPU stream compaction; consumes the
 * input list and returns a new one. */
struct EdgeList *removeDulpicatesSelfLoopEdges(struct EdgeList *edgeList);

/* ---- sorting (GPU) ----------------------------------------------------- */

/* 00_graph_bench/include/preprocess/sortRun.h:7 ; sortRun.c:26-63.
 * sort: 0 radix by src, 1 radix by (src,dst), 2 count by src,
 * 3 count by (src,dst), other = 0.  Stable; sorts the arrays of the list in
 * place and returns the same list. */
struct EdgeList *sortRunAlgorithms(struct EdgeList *edgeList, uint32_t sort);
/* radixsort.h:9 ; radixsort.c:231-278 */
struct EdgeList *radixSortEdgesBySource(struct EdgeList *edgeList);
/* radixsort.h:10 ; radixsort.c:282-335 */
struct EdgeList *radixSortEdgesBySourceAndDestination(struct EdgeList *edgeList);
/* countsort.h:10 ; countsort.c:28-140 (same output as the radix sort) */
struct EdgeList *countSortEdgesBySource(struct EdgeList *edgeList);
/* countsort.h:11 ; countsort.c:143-259 */
struct EdgeList *countSortEdgesByDestination(struct EdgeList *edgeList);
/* countsort.h:12 ; countsort.c:262-270 */
struct EdgeList *countSortEdgesBySourceAndDestination(struct EdgeList *edgeList);

/* ---- CSR (GPU build, host result) ------------------------------------- */

/* 00_graph_bench/include/structures/vertex.h:24 ; vertex.c:26-49 */
struct Vertex *newVertexArray(uint32_t num_vertices);
/* vertex.h:25 ; vertex.c:406-419 */
void freeVertexArray(struct Vertex *vertices);
/* vertex.h:22 ; vertex.c:204-325.  out_degree = run lengths of the sorted
 * src array, edges_idx = first index of each run (0 when the vertex has no
 * edges), in_degree of the other direction mirrored. */
struct GraphCSR *mapVerticesWithInOutDegree(struct GraphCSR *graph, uint8_t inverse);
/* graphCSR.h:34 ; graphCSR.c:107-134 */
struct GraphCSR *graphCSRNew(uint32_t V, uint32_t E, uint8_t inverse);
/* graphCSR.h:33 ; graphCSR.c:137-161 */
struct GraphCSR *graphCSRAssignEdgeList(struct GraphCSR *graphCSR,
                                        struct EdgeList *edgeList, uint8_t inverse);
/* graphCSR.h:35 ; graphCSR.c:164-248.  Read, GPU sort, [dedup], GPU CSR in
 * both directions; keeps a device copy of the result for the algorithms. */
struct GraphCSR *graphCSRPreProcessingStep(struct Arguments *arguments);
/* graphCSR.h:31 ; graphCSR.c:42-64.  Also releases the device copy. */
void graphCSRFree(struct GraphCSR *graphCSR);
/* graphCSR.h:32 ; graphCSR.c:66-104 */
void graphCSRPrint(struct GraphCSR *graphCSR);

/* ---- BFS (GPU) ---------------------------------------------------------- */

/* 00_graph_bench/include/algorithms/openmp/BFS.h:31 ; BFS.c:42-78 */
struct BFSStats *newBFSStatsGraphCSR(struct GraphCSR *graph);
/* BFS.h:36 ; BFS.c:163-180 */
void freeBFSStats(struct BFSStats *stats);
/* BFS.h:42 ; BFS.c:238-268.  pushpull 0 pull, 1 push, 2 direction-optimized,
 * 3/4 bitmap-frontier variants (same depths, GPU), default DO. */
struct BFSStats *breadthFirstSearchGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:44 ; BFS.c:281-362 (bottom-up only) */
struct BFSStats *breadthFirstSearchPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:45 ; BFS.c:375-463 (top-down only) */
struct BFSStats *breadthFirstSearchPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:46 ; BFS.c:476-626 (alpha = 15, beta = 18) */
struct BFSStats *breadthFirstSearchDirectionOptimizedGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:55 ; BFS.c:785-... (GPU: the top-down path) */
struct BFSStats *breadthFirstSearchPushBitmapGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:56 ; BFS.c (GPU: the direction-optimized path) */
struct BFSStats *breadthFirstSearchPushDirectionOptimizedBitmapGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:48 ; BFS.c:639-687.  One top-down level over host queues: the
 * current window [head, tail) of the shared queue is expanded on the GPU and
 * the discovered vertices are appended after tail_next (localFrontierQueues
 * is accepted and unused).  Returns mf = sum over discovered vertices of
 * max(out_degree, 1). */
uint32_t topDownStepGraphCSR(struct GraphCSR *graph, struct ArrayQueue *sharedFrontierQueue,
                             struct ArrayQueue **localFrontierQueues, struct BFSStats *stats);
/* BFS.h:49 ; BFS.c:703-754.  One bottom-up level over host bitmaps on the
 * GPU; returns the number of discovered vertices. */
uint32_t bottomUpStepGraphCSR(struct GraphCSR *graph, struct Bitmap *bitmapCurr,
                              struct Bitmap *bitmapNext, struct BFSStats *stats);

/* 00_graph_bench/include/structures/graphCSR.h:39 ; graphCSR.c:439-558.  Host
 * decode of the .csr file; with a GPU present the device copy used by the
 * algorithms is built while the file decodes.  Label arrays stay NULL. */
struct GraphCSR *readFromBinFileGraphCSR(const char *fname);
/* graphCSR.h:40 ; graphCSR.c:380-437.  Writes fname + ".csr". */
void writeToBinFileGraphCSR(const char *fname, struct GraphCSR *graph);

/* ---- BFS DualOrder (GPU) ------------------------------------------------
 * The DualOrder variants translate the frontier and parents between the
 * forward and inverse CSRs' vertex orders at direction changes.  Provided for
 * graphs whose two orders are the same (no reordering); after a
 * direction-optimized search parents_DualOrder holds the parents as they
 * stood when the last bottom-up phase ended (sentinels if none ran).
 * Graphs with reordered labels: message + NULL. */
/* 00_graph_bench/include/structures/graphCSR.h:36 ; graphCSR.c:250-335 (no -l/-L/-O/-M) */
struct GraphCSR *graphCSRPreProcessingStepDualOrder(struct Arguments *arguments);
/* graphCSR.h:37 ; graphCSR.c:337-377 */
void graphCSRVertexLabelRemappingDualOrder(struct GraphCSR *graphCSR);
/* 00_graph_bench/include/algorithms/openmp/BFS.h:63 ; BFS.c:1045-1068 */
struct BFSStats *breadthFirstSearchGraphCSRDualOrder(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:65 ; BFS.c:1082-1164 */
struct BFSStats *breadthFirstSearchPullGraphCSRDualOrder(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:66 ; BFS.c:1178-1267 */
struct BFSStats *breadthFirstSearchPushGraphCSRDualOrder(struct Arguments *arguments, struct GraphCSR *graph);
/* BFS.h:67 ; BFS.c:1279-1430 */
struct BFSStats *breadthFirstSearchDirectionOptimizedGraphCSRDualOrder(struct Arguments *arguments,
                                                                       struct GraphCSR *graph);
/* BFS.h:69 ; BFS.c:1442-1490 (the code of topDownStepGraphCSR) */
uint32_t topDownStepGraphCSRDualOrder(struct GraphCSR *graph, struct ArrayQueue *sharedFrontierQueue,
                                      struct ArrayQueue **localFrontierQueues, struct BFSStats *stats);
/* BFS.h:70 ; BFS.c:1505-1562 (the code of bottomUpStepGraphCSR) */
uint32_t bottomUpStepGraphCSRDualOrder(struct GraphCSR *graph, struct Bitmap *bitmapCurr,
                                       struct Bitmap *bitmapNext, struct BFSStats *stats);

/* ---- PageRank (GPU) ----------------------------------------------------- */

/* 00_graph_bench/include/algorithms/openmp/pageRank.h:32 ; pageRank.c:47-75 */
struct PageRankStats *newPageRankStatsGraphCSR(struct GraphCSR *graph);
/* pageRank.h:37 ; pageRank.c:167-177 */
void freePageRankStats(struct PageRankStats *stats);
/* pageRank.h:69 ; pageRank.c:871-936.  pushpull 0 pull, 1 push, 6
 * data-driven pull, 7 data-driven push, 8 data-driven pull-push; 2-5 and
 * 9-13 are the reference's fixed-point / quantized variants, which this
 * library does not provide (message + NULL); larger values pull. */
struct PageRankStats *pageRankGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.h:70 ; pageRank.c:939-1062 */
struct PageRankStats *pageRankPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.h:71 ; pageRank.c:1064-1186 */
struct PageRankStats *pageRankPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.h:84 ; pageRank.c:2405-2564 */
struct PageRankStats *pageRankDataDrivenPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.h:85 ; pageRank.c:2566-2721 */
struct PageRankStats *pageRankDataDrivenPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* pageRank.h:86 ; pageRank.c:2723-2919 */
struct PageRankStats *pageRankDataDrivenPullPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* 00_graph_bench/include/preprocess/reorder.h:68 ; reorder.c:165-221.  The
 * labels are sorted in place (ascending fixed-point rank) and returned. */
uint32_t *radixSortEdgesByPageRank(float *pageRanks, uint32_t *labels, uint32_t num_vertices);

/* ---- SPMV (GPU) --------------------------------------------------------- */

/* 00_graph_bench/include/algorithms/openmp/SPMV.h:30 ; SPMV.c:45-66 */
struct SPMVStats *newSPMVStatsGraphCSR(struct GraphCSR *graph);
/* SPMV.h:35 ; SPMV.c:139-154 */
void freeSPMVStats(struct SPMVStats *stats);
/* SPMV.h:51 ; SPMV.c:588-614.  pushpull 0 pull, 1 push; 2 and 3 are the
 * reference's fixed-point variants (message + NULL); other values pull. */
struct SPMVStats *SPMVGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* SPMV.h:52 ; SPMV.c:616-713 */
struct SPMVStats *SPMVPullGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);
/* SPMV.h:53 ; SPMV.c:715-810 */
struct SPMVStats *SPMVPushGraphCSR(struct Arguments *arguments, struct GraphCSR *graph);

/* ---- roots and RNG ------------------------------------------------------ */

/* 00_graph_bench/include/utils/mt19937.h:62-69 ; mt19937.c:54-114 */
void initializeMersenneState(mt19937state *m, unsigned long seed);
unsigned long generateRandInt(mt19937state *m);
float generateRandFloat(mt19937state *m);
/* 00_graph_bench/include/utils/graphRun.h:27 ; graphRun.c:537-556 */
uint32_t generateRandomRootGraphCSR(mt19937state *mt19937var, struct GraphCSR *graph);

#ifdef __cplusplus
}
#endif

#endif /* OGB200_H */
