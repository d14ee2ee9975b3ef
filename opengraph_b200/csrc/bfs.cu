// bfs.cu -- direction-optimizing BFS over the device CSR.
//
// Reference: breadthFirstSearchDirectionOptimizedGraphCSR
// (00_graph_bench/src/algorithms/openmp/BFS.c:476-626) with
// topDownStepGraphCSR (:639-687) and bottomUpStepGraphCSR (:703-754);
// pull-only (:281-362) and push-only (:375-463) are the same loop with the
// direction fixed.
//
// Semantics kept exactly (they decide which steps run, hence the depths):
//  * parents start at -out_degree (or -1), so a top-down step's mf is the
//    sum of max(out_degree, 1) over the vertices it discovers (BFS.c:58-74,
//    :675);
//  * switch to bottom-up when mf > mu / alpha (u32 division, alpha = 15);
//    stay while nf > nf_prev or nf > n / beta (beta = 18); nf is 0 when a
//    bottom-up phase starts, because the reference reads the queue size
//    after arrayQueueToBitmap emptied it (BFS.c:550-551, arrayQueue.c:303);
//    mf = 1 after a bottom-up phase, mu -= mf before each top-down step;
//  * the loop runs while the queue holds any vertex, including vertices
//    without out-edges (one more, empty, top-down step then runs);
//  * bottom-up scans the in-edges of each unvisited vertex in CSR order and
//    takes the first in-neighbour in the frontier (deterministic parent);
//  * top-down claims a vertex with a CAS on its parent (racy parent choice,
//    as in the reference; depths are exact).
//
// Device design:
//  * the frontier is kept twice: its logical size (every vertex discovered
//    by the last step, which drives the loop) and an expansion list of the
//    frontier vertices WITH out-edges -- a vertex without out-edges is never
//    expanded top-down and never probed bottom-up (it is nobody's
//    in-neighbour), so it needs no slot;
//  * top-down is load-balanced by edges: a chained scan over the list's
//    out-degrees gives each vertex its edge offset and scatters, for every
//    tile of kExpTile edges, the list index where the tile starts; the expand
//    kernel then gives each CTA whole edge tiles (coalesced neighbour reads,
//    independent of the degree skew);
//  * bottom-up: the first bottom-up level of a search walks all vertices (a
//    warp's ballot is one whole word of the next bitmap), later levels walk
//    the compacted list of still-unvisited vertices;
//  * bitmaps: bit v = word v>>5, bit v&31 (bitmap.h:7-9).
#include "graph.cuh"

#include <algorithm>

namespace ogb {

constexpr int kScanT = 256;            // threads of the degree scan
constexpr int kScanI = 8;              // list entries per thread
constexpr int kScanTile = kScanT * kScanI;
constexpr int kExpT = 256;             // threads of the expand kernel
constexpr uint32_t kExpTile = 1024;    // edges per expand tile
constexpr unsigned long long kLbAgg = 1ull << 32;
constexpr unsigned long long kLbInc = 2ull << 32;

struct BfsCtl {
  uint32_t qnext;            // logical size of the next frontier
  uint32_t lnext;            // size of the next expansion list
  uint32_t mf;               // top-down: sum of max(out_degree, 1) of discovered
  uint32_t nf;               // bottom-up: discovered count
  uint32_t ul_size;          // bottom-up: size of the next unvisited list
  uint32_t total_edges;      // top-down: out-edges of the expansion list
  uint32_t scan_tiles;       // tile counter of the degree scan
  uint32_t err;
  unsigned long long edges;  // edges examined
  unsigned long long reached_edges;
  uint32_t reached;
  uint32_t all_count;        // host-state step: entries written to all_out
};

struct BfsWork {
  uint32_t V = 0, E = 0;
  DevBuf q0, q1, bm0, bm1, ul0, ul1, ctl;
  DevBuf offs, fstart, fdist, tile_i0, scan_status, all_out;
  BfsCtl* h_ctl = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr, ev_a = nullptr, ev_b = nullptr;
  ~BfsWork() {
    if (h_ctl) cudaFreeHost(h_ctl);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
    if (ev_a) cudaEventDestroy(ev_a);
    if (ev_b) cudaEventDestroy(ev_b);
  }
};

void bfs_work_free(BfsWork* w) { delete w; }

static int bfs_work_get(DevGraph& g, BfsWork** out) {
  if (!g.bfs) g.bfs = new BfsWork();
  BfsWork* w = g.bfs;
  const uint32_t V = g.V, E = g.E;
  const size_t words = ((size_t)V + 31) / 32;
  if (w->V != V || w->E != E || !w->q0.p) {
    OGB_TRY(w->q0.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->q1.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->bm0.alloc(words * 4 + 16));
    OGB_TRY(w->bm1.alloc(words * 4 + 16));
    OGB_TRY(w->ul0.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->ul1.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->offs.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->fstart.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->fdist.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->tile_i0.alloc(((size_t)E / kExpTile + 4) * 4));
    OGB_TRY(w->scan_status.alloc(((size_t)V / kScanTile + 4) * 8));
    OGB_TRY(w->ctl.alloc(sizeof(BfsCtl)));
    w->V = V;
    w->E = E;
  }
  if (!w->h_ctl) OGB_CUDA(cudaMallocHost(&w->h_ctl, sizeof(BfsCtl)));
  if (!w->ev_start) {
    OGB_CUDA(cudaEventCreate(&w->ev_start));
    OGB_CUDA(cudaEventCreate(&w->ev_stop));
    OGB_CUDA(cudaEventCreate(&w->ev_a));
    OGB_CUDA(cudaEventCreate(&w->ev_b));
  }
  *out = w;
  return OK;
}

// parents[v] = -out_degree[v] (or -1), distances[v] = 0 (BFS.c:58-74);
// the root gets itself as parent; it starts the expansion list when it has
// out-edges.
__global__ void __launch_bounds__(256) bfs_init_kernel(uint32_t V, const uint32_t* __restrict__ out_degree,
                                                       int32_t* __restrict__ parents,
                                                       uint32_t* __restrict__ distances, uint32_t root,
                                                       uint32_t* __restrict__ list) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = out_degree[v];
    parents[v] = (v == root) ? (int32_t)root : (d ? -(int32_t)d : -1);
    distances[v] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) list[0] = root;
}

__device__ __forceinline__ uint32_t scan_block_excl(uint32_t v, uint32_t* s_w, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_w[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < kScanT / 32 ? s_w[lane] : 0;
#pragma unroll
    for (int o = 1; o < kScanT / 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < kScanT / 32) s_w[lane] = t;
  }
  __syncthreads();
  *total = s_w[kScanT / 32 - 1];
  return (warp ? s_w[warp - 1] : 0) + x - v;
}

// Top-down, phase 1: exclusive scan of the out-degrees of the expansion list
// (single pass, decoupled look-back).  Writes offs[i] (first edge of entry i
// in the level's edge range), fstart[i] (its first CSR edge), fdist[i] (its
// depth + 1), the total into ctl, and for every edge tile the list index of
// the entry holding the tile's first edge.
__global__ void __launch_bounds__(kScanT) bfs_td_scan_kernel(
    const uint32_t* __restrict__ list, uint32_t n, const uint2* __restrict__ rows,
    const uint32_t* __restrict__ distances, uint32_t* __restrict__ offs, uint32_t* __restrict__ fstart,
    uint32_t* __restrict__ fdist, uint32_t* __restrict__ tile_i0, unsigned long long* __restrict__ status,
    BfsCtl* __restrict__ ctl) {
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ uint32_t s_w[kScanT / 32];
  if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->scan_tiles, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanI;
  uint32_t deg[kScanI], sum = 0;
#pragma unroll
  for (int k = 0; k < kScanI; k++) {
    const uint64_t i = base + k;
    deg[k] = 0;
    if (i < n) {
      const uint32_t v = list[i];
      const uint2 r = rows[v];
      deg[k] = r.y;
      fstart[i] = r.x;
      fdist[i] = distances[v] + 1;
      sum += r.y;
    }
  }
  uint32_t tile_total = 0;
  const uint32_t excl = scan_block_excl(sum, s_w, &tile_total);
  if (threadIdx.x == 0) {
    uint32_t prefix = 0;
    unsigned long long* st = status + tile;
    if (tile == 0) {
      st_volatile_u64(st, kLbInc | tile_total);
    } else {
      st_volatile_u64(st, kLbAgg | tile_total);
      int64_t p = (int64_t)tile - 1;
      uint32_t spins = 0;
      while (p >= 0) {
        const unsigned long long v = ld_volatile_u64(status + p);
        const unsigned long long f = v & ~0xFFFFFFFFull;
        if (f == 0) {
          if (++spins > kSpinLimit) {
            atomicExch(&ctl->err, (uint32_t)ERR_SPIN);
            break;
          }
          continue;
        }
        prefix += (uint32_t)v;
        if (f == kLbInc) break;
        --p;
      }
      st_volatile_u64(st, kLbInc | (unsigned long long)(prefix + tile_total));
    }
    s_prefix = prefix;
    if ((uint64_t)(tile + 1) * kScanTile >= n) ctl->total_edges = prefix + tile_total;
  }
  __syncthreads();
  uint32_t o = s_prefix + excl;
#pragma unroll
  for (int k = 0; k < kScanI; k++) {
    const uint64_t i = base + k;
    if (i < n) {
      offs[i] = o;
      // edge tiles whose first edge lies in [o, o + deg)
      for (uint32_t t = (o + kExpTile - 1) / kExpTile; (uint64_t)t * kExpTile < (uint64_t)o + deg[k]; t++)
        tile_i0[t] = (uint32_t)i;
      o += deg[k];
    }
  }
}

// Top-down, phase 2: each CTA takes whole tiles of kExpTile edges of the
// level; the list entries overlapping a tile are staged in shared memory and
// each edge finds its entry by binary search there.
__global__ void __launch_bounds__(kExpT) bfs_td_expand_kernel(
    const uint32_t* __restrict__ list, uint32_t n, const uint32_t* __restrict__ offs,
    const uint32_t* __restrict__ fstart, const uint32_t* __restrict__ fdist, const uint32_t* __restrict__ tile_i0,
    const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ out_degree, int32_t* __restrict__ parents,
    uint32_t* __restrict__ distances, uint32_t* __restrict__ next_list, uint32_t* __restrict__ all_out,
    BfsCtl* __restrict__ ctl) {
  __shared__ uint32_t s_off[kExpTile + 2], s_start[kExpTile + 2], s_v[kExpTile + 2], s_d[kExpTile + 2];
  __shared__ BlockAppend<kExpTile> q_list, q_all;
  ba_init(q_list);
  ba_init(q_all);
  const uint32_t total = ctl->total_edges;
  const uint32_t ntiles = (total + kExpTile - 1) / kExpTile;
  uint32_t mf = 0, found = 0;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t e0 = t * kExpTile;
    const uint32_t e1 = min(e0 + kExpTile, total);
    const uint32_t i0 = tile_i0[t];
    const uint32_t i1 = (t + 1 < ntiles) ? tile_i0[t + 1] : n - 1;
    const uint32_t cnt = i1 - i0 + 1;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < cnt; k += kExpT) {
      s_off[k] = offs[i0 + k];
      s_start[k] = fstart[i0 + k];
      s_v[k] = list[i0 + k];
      s_d[k] = fdist[i0 + k];
    }
    __syncthreads();
    for (uint32_t e = e0 + threadIdx.x; e < e1; e += kExpT) {
      uint32_t lo = 0, hi = cnt - 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (s_off[mid] <= e)
          lo = mid;
        else
          hi = mid - 1;
      }
      const uint32_t u = nbr[s_start[lo] + (e - s_off[lo])] & 0x3FFFFFFFu;
      const int32_t p = parents[u];
      if (p < 0 && atomicCAS(&parents[u], p, (int32_t)s_v[lo]) == p) {
        distances[u] = s_d[lo];
        mf += (uint32_t)(-p);
        found++;
        if (all_out) ba_push(q_all, u);
        if (out_degree[u]) ba_push(q_list, u);
      }
    }
    // at most kExpTile discoveries per tile: flush every tile
    ba_flush(q_list, next_list, &ctl->lnext);
    if (all_out) ba_flush(q_all, all_out, &ctl->all_count);
  }
  warp_atomic_add_total(&ctl->mf, mf);
  warp_atomic_add_total(&ctl->qnext, found);
}

// Keep the entries of a queue that have out-edges (host-state step API).
__global__ void bfs_filter_list_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                       const uint32_t* __restrict__ out_degree, uint32_t* __restrict__ out,
                                       uint32_t* __restrict__ count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = in[i];
    if (out_degree[v]) out[warp_atomic_inc(count)] = v;
  }
}

// One bottom-up level over all vertices (first bottom-up level of a search):
// a warp covers 32 consecutive vertices, so its ballot is a whole word of
// the next bitmap (no atomics, no clearing).  Vertices left unvisited go to
// the unvisited list.
template <bool OR_INTO>
__global__ void __launch_bounds__(256) bfs_bu_dense_kernel(uint32_t V, const uint2* __restrict__ rows,
                                                           const uint32_t* __restrict__ nbr,
                                                           const uint32_t* __restrict__ bm_cur,
                                                           uint32_t* __restrict__ bm_next,
                                                           int32_t* __restrict__ parents,
                                                           uint32_t* __restrict__ distances,
                                                           uint32_t* __restrict__ ul_next,
                                                           BfsCtl* __restrict__ ctl) {
  constexpr uint32_t kRound = 1024;  // vertices per block round (4 bitmap words per warp)
  __shared__ BlockAppend<2 * kRound> q_ul;
  ba_init(q_ul);
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t nf = 0;
  unsigned long long edges = 0;
  for (uint32_t rbase = blockIdx.x * kRound; rbase < V; rbase += gridDim.x * kRound) {
#pragma unroll
    for (uint32_t k = 0; k < kRound / 256; k++) {
      const uint32_t base = rbase + k * 256 + warp * 32;
      const uint32_t v = base + lane;
      bool found = false;
      bool unvisited = false;
      if (v < V && parents[v] < 0) {
        const uint2 row = rows[v];
        uint32_t j = row.x;
        const uint32_t end = row.x + row.y;
        for (; j < end; j++) {
          const uint32_t u = nbr[j] & 0x3FFFFFFFu;
          if ((bm_cur[u >> 5] >> (u & 31)) & 1u) {
            parents[v] = (int32_t)u;
            distances[v] = distances[u] + 1;
            found = true;
            j++;
            break;
          }
        }
        edges += j - row.x;
        unvisited = !found;
      }
      const uint32_t word = __ballot_sync(0xffffffffu, found);
      if (lane == 0 && base < V) {
        if (OR_INTO)
          bm_next[base >> 5] |= word;
        else
          bm_next[base >> 5] = word;
      }
      nf += found;
      if (unvisited) ba_push(q_ul, v);
    }
    if (ba_size(q_ul) > kRound) ba_flush(q_ul, ul_next, &ctl->ul_size);
  }
  ba_flush(q_ul, ul_next, &ctl->ul_size);
  warp_atomic_add_total(&ctl->nf, nf);
  warp_atomic_add_total64(&ctl->edges, (uint32_t)edges);
}

// One bottom-up level over the unvisited list (bm_next must be cleared).
__global__ void __launch_bounds__(256) bfs_bu_list_kernel(const uint32_t* __restrict__ list, uint32_t count,
                                                          const uint2* __restrict__ rows,
                                                          const uint32_t* __restrict__ nbr,
                                                          const uint32_t* __restrict__ bm_cur,
                                                          uint32_t* __restrict__ bm_next,
                                                          int32_t* __restrict__ parents,
                                                          uint32_t* __restrict__ distances,
                                                          uint32_t* __restrict__ ul_next,
                                                          BfsCtl* __restrict__ ctl) {
  constexpr uint32_t kRound = 1024;  // list entries per block round
  __shared__ BlockAppend<2 * kRound> q_ul;
  ba_init(q_ul);
  uint32_t nf = 0;
  unsigned long long edges = 0;
  for (uint32_t rbase = blockIdx.x * kRound; rbase < count; rbase += gridDim.x * kRound) {
#pragma unroll
    for (uint32_t k = 0; k < kRound / 256; k++) {
      const uint32_t t = rbase + k * 256 + threadIdx.x;
      if (t >= count) continue;
      const uint32_t v = list[t];
      if (parents[v] >= 0) continue;  // visited by a top-down step since the list was made
      const uint2 row = rows[v];
      uint32_t j = row.x;
      const uint32_t end = row.x + row.y;
      bool found = false;
      for (; j < end; j++) {
        const uint32_t u = nbr[j] & 0x3FFFFFFFu;
        if ((bm_cur[u >> 5] >> (u & 31)) & 1u) {
          parents[v] = (int32_t)u;
          distances[v] = distances[u] + 1;
          found = true;
          j++;
          break;
        }
      }
      edges += j - row.x;
      if (found) {
        atomicOr(&bm_next[v >> 5], 1u << (v & 31));
        nf++;
      } else {
        ba_push(q_ul, v);
      }
    }
    if (ba_size(q_ul) > kRound) ba_flush(q_ul, ul_next, &ctl->ul_size);
  }
  ba_flush(q_ul, ul_next, &ctl->ul_size);
  warp_atomic_add_total(&ctl->nf, nf);
  warp_atomic_add_total64(&ctl->edges, (uint32_t)edges);
}

// arrayQueueToBitmap (arrayQueue.c:289-307) over the expansion list.
__global__ void __launch_bounds__(256) bfs_list_to_bitmap_kernel(const uint32_t* __restrict__ q, uint32_t n,
                                                                 uint32_t* __restrict__ bm) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = q[i];
    atomicOr(&bm[v >> 5], 1u << (v & 31));
  }
}

// bitmapToArrayQueue (arrayQueue.c:310-337): the logical size counts every
// set bit; the expansion list keeps the ones with out-edges.
__global__ void __launch_bounds__(256) bfs_bitmap_to_list_kernel(const uint32_t* __restrict__ bm, uint32_t words,
                                                                 const uint32_t* __restrict__ out_degree,
                                                                 uint32_t* __restrict__ list,
                                                                 BfsCtl* __restrict__ ctl) {
  constexpr uint32_t kRoundWords = 128;  // bitmap words per block round (<= 4096 bits)
  __shared__ BlockAppend<2 * kRoundWords * 32> q;
  ba_init(q);
  uint32_t cnt = 0;
  for (uint32_t rbase = blockIdx.x * kRoundWords; rbase < words; rbase += gridDim.x * kRoundWords) {
    const uint32_t w = rbase + threadIdx.x;
    if (threadIdx.x < kRoundWords && w < words) {
      uint32_t word = bm[w];
      cnt += __popc(word);
      while (word) {
        const int bit = __ffs(word) - 1;
        const uint32_t v = w * 32 + (uint32_t)bit;
        if (out_degree[v]) ba_push(q, v);
        word &= word - 1;
      }
    }
    if (ba_size(q) > kRoundWords * 32) ba_flush(q, list, &ctl->lnext);
  }
  ba_flush(q, list, &ctl->lnext);
  warp_atomic_add_total(&ctl->qnext, cnt);
}

// Number of reached vertices and the sum of their out-degrees (Graph500
// traversed edges).
__global__ void __launch_bounds__(256) bfs_reached_kernel(uint32_t V, const int32_t* __restrict__ parents,
                                                          const uint32_t* __restrict__ out_degree,
                                                          BfsCtl* __restrict__ ctl) {
  unsigned long long e = 0;
  uint32_t r = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    if (parents[v] >= 0) {
      r++;
      e += out_degree[v];
    }
  }
  for (int o = 16; o; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    r += __shfl_down_sync(0xffffffffu, r, o);
  }
  if (lane_id() == 0) {
    if (e) atomicAdd(&ctl->reached_edges, e);
    if (r) atomicAdd(&ctl->reached, r);
  }
}

static int read_ctl(BfsWork* w, cudaStream_t s) {
  OGB_CUDA(cudaMemcpyAsync(w->h_ctl, w->ctl.p, sizeof(BfsCtl), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  if (w->h_ctl->err) return fail((int)w->h_ctl->err, "bfs: a bounded device wait gave up");
  return OK;
}

// Launch one top-down level over `list` (n entries with out-edges).  The
// caller clears ctl before and reads it after.
static int td_level(DevGraph& g, BfsWork* w, const uint32_t* list, uint32_t n, int32_t* parents,
                    uint32_t* distances, uint32_t* next_list, uint32_t* all_out, cudaStream_t s,
                    uint32_t* launches) {
  if (n == 0) return OK;
  BfsCtl* d_ctl = w->ctl.as<BfsCtl>();
  const uint32_t tiles = ceil_div(n, kScanTile);
  OGB_CUDA(cudaMemsetAsync(w->scan_status.p, 0, (size_t)tiles * 8, s));
  bfs_td_scan_kernel<<<tiles, kScanT, 0, s>>>(list, n, g.fwd.d_rows(), distances, w->offs.as<uint32_t>(),
                                              w->fstart.as<uint32_t>(), w->fdist.as<uint32_t>(),
                                              w->tile_i0.as<uint32_t>(), w->scan_status.as<unsigned long long>(),
                                              d_ctl);
  OGB_CUDA(cudaGetLastError());
  bfs_td_expand_kernel<<<sm_count() * 8, kExpT, 0, s>>>(
      list, n, w->offs.as<uint32_t>(), w->fstart.as<uint32_t>(), w->fdist.as<uint32_t>(), w->tile_i0.as<uint32_t>(),
      g.fwd.d_dst(), g.fwd.d_out_degree(), parents, distances, next_list, all_out, d_ctl);
  OGB_CUDA(cudaGetLastError());
  *launches += 2;
  return OK;
}

int bfs_run(DevGraph& g, uint32_t root, uint32_t mode, int32_t* parents, uint32_t* distances, BfsResult* res,
            bool time_levels, bool bu_entry_nf_frontier, cudaStream_t s) {
  const uint32_t V = g.V;
  if (root >= V) return fail(ERR_ARG, "bfs: root %u out of range (V=%u)", root, V);
  BfsWork* w = nullptr;
  OGB_TRY(bfs_work_get(g, &w));
  const uint32_t words = (V + 31) / 32;
  const int sms = sm_count();
  const int grid_v = sms * 8;
  BfsCtl* d_ctl = w->ctl.as<BfsCtl>();

  uint32_t* l_cur = w->q0.as<uint32_t>();
  uint32_t* l_next = w->q1.as<uint32_t>();
  uint32_t* bm_cur = w->bm0.as<uint32_t>();
  uint32_t* bm_next = w->bm1.as<uint32_t>();
  uint32_t* ul_cur = w->ul0.as<uint32_t>();
  uint32_t* ul_next = w->ul1.as<uint32_t>();

  bfs_init_kernel<<<grid_v, 256, 0, s>>>(V, g.fwd.d_out_degree(), parents, distances, root, l_cur);
  OGB_CUDA(cudaGetLastError());
  uint32_t launches = 1;
  OGB_CUDA(cudaMemcpyAsync(&w->h_ctl->mf, g.fwd.d_out_degree() + root, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  const uint32_t root_deg = w->h_ctl->mf;

  const uint32_t alpha = 15, beta = 18;
  const uint32_t n = V;
  uint32_t mu = g.E, mf = root_deg, nf = 0, nf_prev = 0;
  uint32_t qcount = 1;                 // logical frontier size
  uint32_t lsize = root_deg ? 1 : 0;   // expansion list size
  uint32_t level = 0;
  bool ul_valid = false;
  uint32_t ul_size = 0;
  BfsResult r;
  r.iteration = 1;
  r.processed_nodes = 1;

  OGB_CUDA(cudaEventRecord(w->ev_start, s));
  auto push_level = [&](uint32_t dir, uint32_t disc, uint32_t fr, uint64_t edges, float ms) {
    if (r.nlevels < (int)(sizeof(r.levels) / sizeof(r.levels[0]))) {
      BfsLevel& L = r.levels[r.nlevels++];
      L.direction = dir;
      L.discovered = disc;
      L.frontier = fr;
      L.mf = mf;
      L.mu = mu;
      L.edges = edges;
      L.ms = ms;
    }
  };

  while (qcount > 0) {
    const bool bottom_up = (mode == BFS_PULL) || (mode == BFS_DO && mf > mu / alpha);
    if (bottom_up) {
      OGB_CUDA(cudaMemsetAsync(bm_cur, 0, (size_t)words * 4, s));
      if (lsize) {
        bfs_list_to_bitmap_kernel<<<std::min<uint32_t>(grid_v, ceil_div(lsize, 256)), 256, 0, s>>>(l_cur, lsize,
                                                                                                    bm_cur);
        OGB_CUDA(cudaGetLastError());
        launches++;
      }
      nf = bu_entry_nf_frontier ? qcount : 0;
      uint32_t frontier = qcount;
      do {
        nf_prev = nf;
        OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(BfsCtl), s));
        if (time_levels) OGB_CUDA(cudaEventRecord(w->ev_a, s));
        if (!ul_valid) {
          bfs_bu_dense_kernel<false><<<grid_v, 256, 0, s>>>(V, g.inv.d_rows(), g.inv.d_dst(), bm_cur, bm_next,
                                                            parents, distances, ul_next, d_ctl);
          launches++;
        } else {
          OGB_CUDA(cudaMemsetAsync(bm_next, 0, (size_t)words * 4, s));
          if (ul_size) {
            bfs_bu_list_kernel<<<std::min<uint32_t>(grid_v, ceil_div(ul_size, 256)), 256, 0, s>>>(
                ul_cur, ul_size, g.inv.d_rows(), g.inv.d_dst(), bm_cur, bm_next, parents, distances, ul_next, d_ctl);
            launches++;
          }
        }
        OGB_CUDA(cudaGetLastError());
        if (time_levels) OGB_CUDA(cudaEventRecord(w->ev_b, s));
        OGB_TRY(read_ctl(w, s));
        float ms = 0.f;
        if (time_levels) cudaEventElapsedTime(&ms, w->ev_a, w->ev_b);
        nf = w->h_ctl->nf;
        ul_size = w->h_ctl->ul_size;
        ul_valid = true;
        std::swap(ul_cur, ul_next);
        std::swap(bm_cur, bm_next);
        level++;
        r.iteration++;
        r.processed_nodes += nf;
        r.bu_steps++;
        r.edges_examined += w->h_ctl->edges;
        push_level(1, nf, frontier, w->h_ctl->edges, ms);
        frontier = nf;
      } while (mode == BFS_PULL ? (nf > 0) : ((nf > nf_prev) || (nf > (n / beta))));
      OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(BfsCtl), s));
      bfs_bitmap_to_list_kernel<<<std::min<uint32_t>(grid_v, ceil_div(words, 256)), 256, 0, s>>>(
          bm_cur, words, g.fwd.d_out_degree(), l_cur, d_ctl);
      OGB_CUDA(cudaGetLastError());
      launches++;
      OGB_TRY(read_ctl(w, s));
      qcount = w->h_ctl->qnext;
      lsize = w->h_ctl->lnext;
      mf = 1;
    } else {
      mu -= mf;
      OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(BfsCtl), s));
      if (time_levels) OGB_CUDA(cudaEventRecord(w->ev_a, s));
      OGB_TRY(td_level(g, w, l_cur, lsize, parents, distances, l_next, nullptr, s, &launches));
      if (time_levels) OGB_CUDA(cudaEventRecord(w->ev_b, s));
      OGB_TRY(read_ctl(w, s));
      float ms = 0.f;
      if (time_levels) cudaEventElapsedTime(&ms, w->ev_a, w->ev_b);
      const uint32_t frontier = qcount;
      mf = w->h_ctl->mf;
      qcount = w->h_ctl->qnext;
      lsize = w->h_ctl->lnext;
      std::swap(l_cur, l_next);
      level++;
      r.iteration++;
      r.processed_nodes += qcount;
      r.td_steps++;
      r.edges_examined += w->h_ctl->total_edges;
      push_level(0, qcount, frontier, w->h_ctl->total_edges, ms);
    }
  }
  OGB_CUDA(cudaEventRecord(w->ev_stop, s));
  OGB_CUDA(cudaEventSynchronize(w->ev_stop));
  float total_ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&total_ms, w->ev_start, w->ev_stop));
  r.ms = total_ms;
  r.launches = launches;

  OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(BfsCtl), s));
  bfs_reached_kernel<<<grid_v, 256, 0, s>>>(V, parents, g.fwd.d_out_degree(), d_ctl);
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(read_ctl(w, s));
  r.reached = w->h_ctl->reached;
  r.reached_out_edges = w->h_ctl->reached_edges;
  if (res) *res = r;
  return OK;
}

}  // namespace ogb

using namespace ogb;

int bfs_td_step_host(DevGraph& g, const uint32_t* q, uint32_t qsize, int32_t* parents, uint32_t* distances,
                     uint32_t* next_q, uint32_t* next_size, uint32_t* mf, cudaStream_t s) {
  BfsWork* w = nullptr;
  OGB_TRY(bfs_work_get(g, &w));
  const uint32_t V = g.V;
  DevBuf d_par, d_dist, d_all;
  OGB_TRY(d_par.alloc((size_t)V * 4 + 4));
  OGB_TRY(d_dist.alloc((size_t)V * 4 + 4));
  OGB_TRY(d_all.alloc((size_t)V * 4 + 4));
  OGB_CUDA(cudaMemcpyAsync(d_par.p, parents, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(d_dist.p, distances, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->ul0.p, q, (size_t)qsize * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemsetAsync(w->ctl.p, 0, sizeof(BfsCtl), s));
  uint32_t launches = 0;
  if (qsize) {
    bfs_filter_list_kernel<<<std::min<uint32_t>(sm_count() * 8, ceil_div(qsize, 256)), 256, 0, s>>>(
        w->ul0.as<uint32_t>(), qsize, g.fwd.d_out_degree(), w->q0.as<uint32_t>(), &w->ctl.as<BfsCtl>()->lnext);
    OGB_CUDA(cudaGetLastError());
  }
  OGB_TRY(read_ctl(w, s));
  const uint32_t n = w->h_ctl->lnext;
  OGB_CUDA(cudaMemsetAsync(w->ctl.p, 0, sizeof(BfsCtl), s));
  OGB_TRY(td_level(g, w, w->q0.as<uint32_t>(), n, d_par.as<int32_t>(), d_dist.as<uint32_t>(), w->q1.as<uint32_t>(),
                   d_all.as<uint32_t>(), s, &launches));
  OGB_TRY(read_ctl(w, s));
  *next_size = w->h_ctl->qnext;
  *mf = w->h_ctl->mf;
  OGB_CUDA(cudaMemcpyAsync(next_q, d_all.p, (size_t)(*next_size) * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(parents, d_par.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(distances, d_dist.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

int bfs_bu_step_host(DevGraph& g, const uint32_t* bm_cur, uint32_t* bm_next, int32_t* parents, uint32_t* distances,
                     uint32_t* nf, cudaStream_t s) {
  BfsWork* w = nullptr;
  OGB_TRY(bfs_work_get(g, &w));
  const uint32_t V = g.V;
  const size_t words = ((size_t)V + 31) / 32;
  DevBuf d_par, d_dist;
  OGB_TRY(d_par.alloc((size_t)V * 4 + 4));
  OGB_TRY(d_dist.alloc((size_t)V * 4 + 4));
  OGB_CUDA(cudaMemcpyAsync(d_par.p, parents, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(d_dist.p, distances, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->bm0.p, bm_cur, words * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->bm1.p, bm_next, words * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemsetAsync(w->ctl.p, 0, sizeof(BfsCtl), s));
  bfs_bu_dense_kernel<true><<<sm_count() * 8, 256, 0, s>>>(V, g.inv.d_rows(), g.inv.d_dst(), w->bm0.as<uint32_t>(),
                                                           w->bm1.as<uint32_t>(), d_par.as<int32_t>(),
                                                           d_dist.as<uint32_t>(), w->ul0.as<uint32_t>(),
                                                           w->ctl.as<BfsCtl>());
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(read_ctl(w, s));
  *nf = w->h_ctl->nf;
  OGB_CUDA(cudaMemcpyAsync(bm_next, w->bm1.p, words * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(parents, d_par.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(distances, d_dist.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}
