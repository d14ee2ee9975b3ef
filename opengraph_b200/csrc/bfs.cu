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
//  * bottom-up scans the in-edges of each unvisited vertex in CSR order and
//    takes the first in-neighbour in the frontier (deterministic parent);
//  * top-down claims a vertex with a CAS on its parent (racy parent choice,
//    as in the reference; depths are exact).
//
// Device layout: frontier queue (u32 ids), frontier bitmaps (bit v = word
// v>>5, bit v&31, as bitmap.h:7-9), and a compacted list of unvisited
// vertices so that bottom-up levels after the first only visit candidates.
#include "graph.cuh"

#include <algorithm>

namespace ogb {

struct BfsCtl {
  uint32_t qnext;            // size of the next queue / converted queue
  uint32_t mf;               // top-down: sum of max(out_degree, 1) of discovered
  uint32_t nf;               // bottom-up: discovered count
  uint32_t ul_size;          // bottom-up: size of the next unvisited list
  unsigned long long edges;  // edges examined
  unsigned long long reached_edges;
  uint32_t reached;
  uint32_t err;
};

struct BfsWork {
  uint32_t V = 0;
  DevBuf q0, q1, bm0, bm1, ul0, ul1, ctl;
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
  const uint32_t V = g.V;
  const size_t words = ((size_t)V + 31) / 32;
  if (w->V != V || !w->q0.p) {
    OGB_TRY(w->q0.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->q1.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->bm0.alloc(words * 4 + 16));
    OGB_TRY(w->bm1.alloc(words * 4 + 16));
    OGB_TRY(w->ul0.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->ul1.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->ctl.alloc(sizeof(BfsCtl)));
    w->V = V;
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
// the root gets itself as parent and is the only queue entry.
__global__ void __launch_bounds__(256) bfs_init_kernel(uint32_t V, const uint32_t* __restrict__ out_degree,
                                                       int32_t* __restrict__ parents,
                                                       uint32_t* __restrict__ distances, uint32_t root,
                                                       uint32_t* __restrict__ queue) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = out_degree[v];
    parents[v] = (v == root) ? (int32_t)root : (d ? -(int32_t)d : -1);
    distances[v] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) queue[0] = root;
}

// One top-down level: a warp per frontier vertex, lanes over its out-edges.
__global__ void __launch_bounds__(256) bfs_td_kernel(const uint2* __restrict__ rows,
                                                     const uint32_t* __restrict__ nbr,
                                                     const uint32_t* __restrict__ queue, uint32_t qsize,
                                                     uint32_t* __restrict__ next_queue,
                                                     int32_t* __restrict__ parents,
                                                     uint32_t* __restrict__ distances, BfsCtl* __restrict__ ctl) {
  const uint32_t lane = lane_id();
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t mf = 0;
  unsigned long long edges = 0;
  for (uint32_t i = gwarp; i < qsize; i += nwarps) {
    const uint32_t v = queue[i];
    const uint2 row = rows[v];
    const uint32_t next_level = distances[v] + 1;
    edges += row.y;
    for (uint32_t j = row.x + lane; j < row.x + row.y; j += 32) {
      const uint32_t u = nbr[j] & 0x3FFFFFFFu;
      const int32_t p = parents[u];
      if (p < 0) {
        if (atomicCAS(&parents[u], p, (int32_t)v) == p) {
          distances[u] = next_level;
          next_queue[warp_atomic_inc(&ctl->qnext)] = u;
          mf += (uint32_t)(-p);
        }
      }
    }
  }
  mf = __reduce_add_sync(0xffffffffu, mf);
  if (lane == 0) {
    if (mf) atomicAdd(&ctl->mf, mf);
    if (edges) atomicAdd(&ctl->edges, edges);
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
  const uint32_t lane = lane_id();
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t nf = 0;
  unsigned long long edges = 0;
  for (uint32_t base = gwarp * 32; base < V; base += nwarps * 32) {
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
    if (lane == 0) {
      if (OR_INTO)
        bm_next[base >> 5] |= word;
      else
        bm_next[base >> 5] = word;
    }
    nf += found;
    if (unvisited) ul_next[warp_atomic_inc(&ctl->ul_size)] = v;
  }
  nf = __reduce_add_sync(0xffffffffu, nf);
  if (lane == 0) {
    if (nf) atomicAdd(&ctl->nf, nf);
    if (edges) atomicAdd(&ctl->edges, edges);
  }
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
  uint32_t nf = 0;
  unsigned long long edges = 0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
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
      ul_next[warp_atomic_inc(&ctl->ul_size)] = v;
    }
  }
  warp_atomic_add_total(&ctl->nf, nf);
  if (edges) atomicAdd(&ctl->edges, edges);
}

// arrayQueueToBitmap (arrayQueue.c:289-307).
__global__ void __launch_bounds__(256) bfs_queue_to_bitmap_kernel(const uint32_t* __restrict__ q, uint32_t n,
                                                                  uint32_t* __restrict__ bm) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = q[i];
    atomicOr(&bm[v >> 5], 1u << (v & 31));
  }
}

// bitmapToArrayQueue (arrayQueue.c:310-337): compaction of the set bits.
__global__ void __launch_bounds__(256) bfs_bitmap_to_queue_kernel(const uint32_t* __restrict__ bm, uint32_t words,
                                                                  uint32_t* __restrict__ q,
                                                                  uint32_t* __restrict__ qsize) {
  const uint32_t lane = lane_id();
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t base = gwarp * 32; base < words; base += nwarps * 32) {
    const uint32_t w = base + lane;
    uint32_t word = (w < words) ? bm[w] : 0u;
    const uint32_t c = __popc(word);
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, x, 31);
    uint32_t b = 0;
    if (lane == 31 && total) b = atomicAdd(qsize, total);
    b = __shfl_sync(0xffffffffu, b, 31);
    uint32_t pos = b + x - c;
    while (word) {
      const int bit = __ffs(word) - 1;
      q[pos++] = w * 32 + (uint32_t)bit;
      word &= word - 1;
    }
  }
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

  uint32_t* q_cur = w->q0.as<uint32_t>();
  uint32_t* q_next = w->q1.as<uint32_t>();
  uint32_t* bm_cur = w->bm0.as<uint32_t>();
  uint32_t* bm_next = w->bm1.as<uint32_t>();
  uint32_t* ul_cur = w->ul0.as<uint32_t>();
  uint32_t* ul_next = w->ul1.as<uint32_t>();

  bfs_init_kernel<<<grid_v, 256, 0, s>>>(V, g.fwd.d_out_degree(), parents, distances, root, q_cur);
  OGB_CUDA(cudaGetLastError());
  uint32_t launches = 1;
  uint32_t root_deg = 0;
  OGB_CUDA(cudaMemcpyAsync(&w->h_ctl->mf, g.fwd.d_out_degree() + root, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  root_deg = w->h_ctl->mf;

  const uint32_t alpha = 15, beta = 18;
  const uint32_t n = V;
  uint32_t mu = g.E, mf = root_deg, nf = 0, nf_prev = 0;
  uint32_t qsize = 1, level = 0;
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

  while (qsize > 0) {
    const bool bottom_up = (mode == BFS_PULL) || (mode == BFS_DO && mf > mu / alpha);
    if (bottom_up) {
      OGB_CUDA(cudaMemsetAsync(bm_cur, 0, (size_t)words * 4, s));
      bfs_queue_to_bitmap_kernel<<<std::min<uint32_t>(grid_v, ceil_div(qsize, 256)), 256, 0, s>>>(q_cur, qsize, bm_cur);
      OGB_CUDA(cudaGetLastError());
      launches++;
      nf = bu_entry_nf_frontier ? qsize : 0;
      uint32_t frontier = qsize;
      do {
        nf_prev = nf;
        OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(BfsCtl), s));
        if (time_levels) OGB_CUDA(cudaEventRecord(w->ev_a, s));
        launches++;
        if (!ul_valid) {
          bfs_bu_dense_kernel<false><<<grid_v, 256, 0, s>>>(V, g.inv.d_rows(), g.inv.d_dst(), bm_cur, bm_next,
                                                            parents, distances, ul_next, d_ctl);
        } else {
          OGB_CUDA(cudaMemsetAsync(bm_next, 0, (size_t)words * 4, s));
          if (ul_size)
            bfs_bu_list_kernel<<<std::min<uint32_t>(grid_v, ceil_div(ul_size, 256)), 256, 0, s>>>(
                ul_cur, ul_size, g.inv.d_rows(), g.inv.d_dst(), bm_cur, bm_next, parents, distances, ul_next, d_ctl);
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
      bfs_bitmap_to_queue_kernel<<<std::min<uint32_t>(grid_v, ceil_div(words, 256)), 256, 0, s>>>(bm_cur, words,
                                                                                                    q_cur, &d_ctl->qnext);
      OGB_CUDA(cudaGetLastError());
      launches++;
      OGB_TRY(read_ctl(w, s));
      qsize = w->h_ctl->qnext;
      mf = 1;
    } else {
      mu -= mf;
      OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(BfsCtl), s));
      if (time_levels) OGB_CUDA(cudaEventRecord(w->ev_a, s));
      const uint32_t grid_td = std::min<uint32_t>(grid_v, ceil_div((uint64_t)qsize * 32, 256));
      bfs_td_kernel<<<grid_td, 256, 0, s>>>(g.fwd.d_rows(), g.fwd.d_dst(), q_cur, qsize, q_next, parents, distances,
                                             d_ctl);
      OGB_CUDA(cudaGetLastError());
      launches++;
      if (time_levels) OGB_CUDA(cudaEventRecord(w->ev_b, s));
      OGB_TRY(read_ctl(w, s));
      float ms = 0.f;
      if (time_levels) cudaEventElapsedTime(&ms, w->ev_a, w->ev_b);
      const uint32_t frontier = qsize;
      mf = w->h_ctl->mf;
      qsize = w->h_ctl->qnext;
      std::swap(q_cur, q_next);
      level++;
      r.iteration++;
      r.processed_nodes += qsize;
      r.td_steps++;
      r.edges_examined += w->h_ctl->edges;
      push_level(0, qsize, frontier, w->h_ctl->edges, ms);
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
  DevBuf d_par, d_dist;
  OGB_TRY(d_par.alloc((size_t)V * 4 + 4));
  OGB_TRY(d_dist.alloc((size_t)V * 4 + 4));
  OGB_CUDA(cudaMemcpyAsync(d_par.p, parents, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(d_dist.p, distances, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->q0.p, q, (size_t)qsize * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemsetAsync(w->ctl.p, 0, sizeof(BfsCtl), s));
  if (qsize) {
    const uint32_t grid = std::min<uint32_t>(sm_count() * 8, ceil_div((uint64_t)qsize * 32, 256));
    bfs_td_kernel<<<grid, 256, 0, s>>>(g.fwd.d_rows(), g.fwd.d_dst(), w->q0.as<uint32_t>(), qsize,
                                        w->q1.as<uint32_t>(), d_par.as<int32_t>(), d_dist.as<uint32_t>(),
                                        w->ctl.as<BfsCtl>());
    OGB_CUDA(cudaGetLastError());
  }
  OGB_TRY(read_ctl(w, s));
  *next_size = w->h_ctl->qnext;
  *mf = w->h_ctl->mf;
  OGB_CUDA(cudaMemcpyAsync(next_q, w->q1.p, (size_t)(*next_size) * 4, cudaMemcpyDeviceToHost, s));
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
