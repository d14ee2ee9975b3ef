/* Prints sizeof/offsetof of the reference structs that cross the drop-in
 * boundary, compiled against the reference headers (or the WEIGHTED=1
 * shadow).  tests/test_abi.py compares this with the ctypes layouts of
 * include/ogb200.h.  Output: one "Struct.field offset" line per field and
 * one "Struct sizeof" line per struct. */
#include <stdio.h>
#include <stddef.h>
#include <stdint.h>
#include "graphConfig.h"
#include "edgeList.h"
#include "vertex.h"
#include "graphCSR.h"
#include "BFS.h"
#include "pageRank.h"
#include "bitmap.h"
#include "arrayQueue.h"

#define F(S, f) printf(#S "." #f " %zu\n", offsetof(struct S, f))
#define Z(S) printf(#S " %zu\n", sizeof(struct S))

int main(void)
{
    Z(Arguments); F(Arguments, epsilon); F(Arguments, source); F(Arguments, pushpull); F(Arguments, sort);
    F(Arguments, fnameb); F(Arguments, fnamel); F(Arguments, fnameb_format); F(Arguments, mt19937var);
    F(Arguments, cache_size);
    Z(EdgeList); F(EdgeList, num_edges); F(EdgeList, num_vertices); F(EdgeList, avg_degree);
#if WEIGHTED
    F(EdgeList, max_weight); F(EdgeList, edges_array_weight);
#endif
    F(EdgeList, edges_array_src); F(EdgeList, edges_array_dest); F(EdgeList, mask_array);
    F(EdgeList, label_array); F(EdgeList, inverse_label_array);
    Z(Vertex); F(Vertex, out_degree); F(Vertex, in_degree); F(Vertex, edges_idx);
    Z(GraphCSR); F(GraphCSR, num_edges); F(GraphCSR, vertices); F(GraphCSR, sorted_edges_array);
#if WEIGHTED
    F(GraphCSR, max_weight);
#endif
    F(GraphCSR, inverse_vertices); F(GraphCSR, inverse_sorted_edges_array);
    Z(BFSStats); F(BFSStats, distances); F(BFSStats, parents); F(BFSStats, processed_nodes);
    F(BFSStats, iteration); F(BFSStats, time_total);
    Z(PageRankStats); F(PageRankStats, iterations); F(PageRankStats, activeVertices); F(PageRankStats, realRanks);
    F(PageRankStats, pageRanks); F(PageRankStats, time_total); F(PageRankStats, error_total);
    Z(Bitmap); F(Bitmap, bitarray);
    Z(ArrayQueue); F(ArrayQueue, queue); F(ArrayQueue, q_bitmap_next);
    printf("mt19937state %zu\n", sizeof(mt19937state));
    return 0;
}
