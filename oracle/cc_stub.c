/* Stand-ins for the connected-components entry points that graphRun.c
 * references (00_graph_bench/src/utils/graphRun.c:766-808, :1300).  Their
 * implementation (connectedComponents.c) needs libJudy, which this image
 * does not have; nothing on the BFS/PageRank path calls them. */
#include <stdio.h>
#include <stddef.h>

struct CCStats;

static void *cc_unavailable(void)
{
    fprintf(stderr, "connected components: not built (libJudy unavailable)\n");
    return NULL;
}

struct CCStats *connectedComponentsGraphCSR(void *arguments, void *graph) { (void)arguments; (void)graph; return cc_unavailable(); }
struct CCStats *connectedComponentsGraphGrid(void *arguments, void *graph) { (void)arguments; (void)graph; return cc_unavailable(); }
struct CCStats *connectedComponentsGraphAdjArrayList(void *arguments, void *graph) { (void)arguments; (void)graph; return cc_unavailable(); }
struct CCStats *connectedComponentsGraphAdjLinkedList(void *arguments, void *graph) { (void)arguments; (void)graph; return cc_unavailable(); }
void freeCCStats(struct CCStats *stats) { (void)stats; }
