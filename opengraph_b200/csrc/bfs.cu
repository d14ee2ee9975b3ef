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
//  * the whole switch state lives in device memory (BfsDevState) and two
//    one-thread control kernels apply the reference's rules: `decide` before
//    a step (termination, direction, conversions) and `finish` after it
//    (counters, bottom-up continuation).  A search is therefore ONE CUDA
//    graph: a WHILE node whose body is [IF bitmap->list] decide [IF
//    list->bitmap] [IF top-down] [IF bottom-up first] [IF bottom-up list]
//    finish, the IF conditions set by the control kernels.  No host round
//    trip per level; the loop is bounded (max_steps) so it cannot run away.
//    A host-stepped driver launches the same kernels one by one (used when
//    per-level CUDA-event times are wanted);
//  * the frontier is kept twice: its logical size (every vertex discovered
//    by the last step, which drives the loop) and an expansion list of the
//    frontier vertices WITH out-edges -- a vertex without out-edges is never
//    expanded top-down and never probed bottom-up (it is nobody's
//    in-neighbour), so it needs no slot;
//  * top-down is load-balanced by edges: a chained scan over the list's
//    out-degrees gives each vertex its edge offset and scatters, for every
//    tile of kExpTile edges, the list index where the tile starts; the expand
//    kernel then gives each CTA whole edge tiles (coalesced neighbour reads,
//    independent of the degree skew).  The scan's look-back words carry the
//    step's epoch, so they never need clearing;
//  * bottom-up: the first bottom-up level of a search walks all vertices (a
//    warp's ballot is one whole word of the next bitmap), later levels walk
//    the compacted list of still-unvisited vertices;
//  * queue appends are staged per CTA in shared memory (one global atomic
//    per flush);
//  * bitmaps: bit v = word v>>5, bit v&31 (bitmap.h:7-9).
#include "graph.cuh"

#include <algorithm>
#include <vector>

namespace ogb {

constexpr int kScanT = 256;            // threads of the degree scan
constexpr int kScanI = 8;              // list entries per thread
constexpr int kScanTile = kScanT * kScanI;
constexpr int kExpT = 256;             // threads of the expand kernel
constexpr uint32_t kExpTile = 1024;    // edges per expand tile
constexpr int kMaxTrace = 512;
constexpr uint32_t kAlpha = 15, kBeta = 18;

struct BfsCtl {
  uint32_t qnext;            // logical size of the next frontier
  uint32_t lnext;            // size of the next expansion list
  uint32_t mf;               // top-down: sum of max(out_degree, 1) of discovered
  uint32_t nf;               // bottom-up: discovered count
  uint32_t ul_size;          // bottom-up: size of the next unvisited list
  uint32_t total_edges;      // top-down: out-edges of the expansion list
  uint32_t scan_tiles;       // tile counter of the degree scan
  uint32_t all_count;        // host-state step: entries written to all_out
  unsigned long long edges;  // bottom-up: edges examined
  unsigned long long reached_edges;
  uint32_t reached;
  uint32_t pad;
};

// Direction codes of BfsDevState::dir.
constexpr uint32_t kDirTD = 0, kDirBU = 1, kDirNone = 2;

struct BfsDevState {
  uint32_t mode, bu_entry_frontier, n, E;
  uint32_t max_steps, root;
  int32_t* parents;
  uint32_t* distances;
  uint32_t mu, mf, nf, nf_prev;          // the reference's switch state
  uint32_t qcount, lsize, frontier, dir;  // logical frontier, expansion list, step
  uint32_t in_bu, need_b2l, l2b_now, dense_now;
  uint32_t ul_valid, ul_size, par_l, par_bm;
  uint32_t par_ul, iteration, processed, td_steps;
  uint32_t bu_steps, nlevels, done, err;
  uint32_t epoch, pad;
  unsigned long long edges_examined;
  BfsCtl ctl;
  BfsLevel trace[kMaxTrace];
};

// Device buffers of one graph (fixed; passed by value to every kernel).
struct BfsBufs {
  const uint2* rows_f;
  const uint32_t* nbr_f;
  const uint2* rows_i;
  const uint32_t* nbr_i;
  const uint32_t* out_degree;
  uint32_t* list[2];
  uint32_t* bm[2];
  uint32_t* ul[2];
  uint32_t* offs;
  uint32_t* fstart;
  uint32_t* fdist;
  uint32_t* tile_i0;
  unsigned long long* status;
  uint32_t* all_out;  // host-state top-down step only
  uint32_t V, words;
};

struct BfsGraph {
  cudaGraphExec_t exec = nullptr;
};

struct BfsWork {
  uint32_t V = 0, E = 0;
  DevBuf q0, q1, bm0, bm1, ul0, ul1, state;
  DevBuf offs, fstart, fdist, tile_i0, scan_status, all_out;
  BfsDevState* h_state = nullptr;   // pinned copy
  cudaStream_t cap = nullptr;       // capture stream
  BfsGraph graphs[3][2];            // [mode][bu_entry_frontier]
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr, ev_a = nullptr, ev_b = nullptr;
  ~BfsWork() {
    for (auto& gm : graphs)
      for (auto& gg : gm)
        if (gg.exec) cudaGraphExecDestroy(gg.exec);
    if (h_state) cudaFreeHost(h_state);
    if (cap) cudaStreamDestroy(cap);
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
    for (auto& gm : w->graphs)
      for (auto& gg : gm)
        if (gg.exec) {
          cudaGraphExecDestroy(gg.exec);
          gg.exec = nullptr;
        }
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
    OGB_TRY(w->state.alloc(sizeof(BfsDevState)));
    OGB_CUDA(cudaMemset(w->scan_status.p, 0, ((size_t)V / kScanTile + 4) * 8));
    OGB_CUDA(cudaMemset(w->state.p, 0, sizeof(BfsDevState)));
    w->V = V;
    w->E = E;
  }
  if (!w->h_state) OGB_CUDA(cudaMallocHost(&w->h_state, sizeof(BfsDevState)));
  if (!w->ev_start) {
    OGB_CUDA(cudaEventCreate(&w->ev_start));
    OGB_CUDA(cudaEventCreate(&w->ev_stop));
    OGB_CUDA(cudaEventCreate(&w->ev_a));
    OGB_CUDA(cudaEventCreate(&w->ev_b));
  }
  if (!w->cap) OGB_CUDA(cudaStreamCreateWithFlags(&w->cap, cudaStreamNonBlocking));
  *out = w;
  return OK;
}

static BfsBufs make_bufs(DevGraph& g, BfsWork* w, uint32_t* all_out) {
  BfsBufs b;
  b.rows_f = g.fwd.d_rows();
  b.nbr_f = g.fwd.d_dst();
  b.rows_i = g.inv.d_rows();
  b.nbr_i = g.inv.d_dst();
  b.out_degree = g.fwd.d_out_degree();
  b.list[0] = w->q0.as<uint32_t>();
  b.list[1] = w->q1.as<uint32_t>();
  b.bm[0] = w->bm0.as<uint32_t>();
  b.bm[1] = w->bm1.as<uint32_t>();
  b.ul[0] = w->ul0.as<uint32_t>();
  b.ul[1] = w->ul1.as<uint32_t>();
  b.offs = w->offs.as<uint32_t>();
  b.fstart = w->fstart.as<uint32_t>();
  b.fdist = w->fdist.as<uint32_t>();
  b.tile_i0 = w->tile_i0.as<uint32_t>();
  b.status = w->scan_status.as<unsigned long long>();
  b.all_out = all_out;
  b.V = g.V;
  b.words = (g.V + 31) / 32;
  return b;
}

// ------------------------------------------------------------ init ---------

// parents[v] = -out_degree[v] (or -1), distances[v] = 0 (BFS.c:58-74); the
// root gets itself as parent; the state starts as the reference's loop does
// (mu = E, mf = out_degree(root), queue = {root}, iteration 1).
__global__ void __launch_bounds__(256) bfsk_init(BfsBufs b, BfsDevState* __restrict__ st, uint32_t root,
                                                 int32_t* __restrict__ parents, uint32_t* __restrict__ distances,
                                                 uint32_t mode, uint32_t bu_entry_frontier, uint32_t E) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < b.V; v += gridDim.x * blockDim.x) {
    const uint32_t d = b.out_degree[v];
    parents[v] = (v == root) ? (int32_t)root : (d ? -(int32_t)d : -1);
    distances[v] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t d = b.out_degree[root];
    const uint32_t epoch = st->epoch;  // keeps growing across searches
    char* raw = reinterpret_cast<char*>(st);
    for (size_t i = 0; i < offsetof(BfsDevState, trace); i++) raw[i] = 0;
    st->mode = mode;
    st->bu_entry_frontier = bu_entry_frontier;
    st->n = b.V;
    st->E = E;
    st->max_steps = b.V + 8;
    st->root = root;
    st->parents = parents;
    st->distances = distances;
    st->mu = E;
    st->mf = d;
    st->qcount = 1;
    st->lsize = d ? 1u : 0u;
    st->dir = kDirNone;
    st->iteration = 1;
    st->processed = 1;
    st->epoch = epoch;
    b.list[0][0] = root;
  }
}

// ------------------------------------------------------------ control ------

// Before a step: turns a finished bottom-up phase's bitmap count into the
// queue (mf = 1), stops on an empty queue, and otherwise picks the step's
// direction with the reference's rule.  Sets the IF conditions of the step
// (graph mode) and the matching flags (host-stepped mode).
__global__ void bfsk_decide(BfsDevState* __restrict__ st, int use_handles, cudaGraphConditionalHandle h_l2b,
                            cudaGraphConditionalHandle h_td, cudaGraphConditionalHandle h_bud,
                            cudaGraphConditionalHandle h_bul) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t l2b = 0, td = 0, bud = 0, bul = 0;
  if (!st->done) {
    if (st->need_b2l) {
      st->qcount = st->ctl.qnext;
      st->lsize = st->ctl.lnext;
      st->mf = 1;
      st->need_b2l = 0;
    }
    if (!st->in_bu && st->qcount == 0) {
      st->done = 1;
      st->dir = kDirNone;
    } else {
      const uint32_t epoch = st->epoch + 1;
      BfsCtl z = {};
      st->ctl = z;
      st->epoch = epoch;
      if (st->in_bu) {
        st->dir = kDirBU;
        st->frontier = st->nf;
        st->nf_prev = st->nf;
      } else {
        const bool bu = (st->mode == BFS_PULL) || (st->mode == BFS_DO && st->mf > st->mu / kAlpha);
        st->frontier = st->qcount;
        if (bu) {
          st->in_bu = 1;
          l2b = 1;
          st->nf = st->bu_entry_frontier ? st->qcount : 0u;
          st->nf_prev = st->nf;
          st->dir = kDirBU;
        } else {
          st->mu -= st->mf;
          st->dir = kDirTD;
        }
      }
      if (st->dir == kDirTD)
        td = 1;
      else if (!st->ul_valid)
        bud = 1;
      else
        bul = 1;
    }
  }
  st->l2b_now = l2b;
  st->dense_now = bud;
  if (use_handles) {
    cudaGraphSetConditional(h_l2b, l2b);
    cudaGraphSetConditional(h_td, td);
    cudaGraphSetConditional(h_bud, bud);
    cudaGraphSetConditional(h_bul, bul);
  }
}

// After a step: the step's counters into the switch state, the trace, the
// parities; decides whether the bottom-up phase continues (else the next
// iteration converts the bitmap to the queue) and whether the loop goes on.
__global__ void bfsk_finish(BfsDevState* __restrict__ st, int use_handles, cudaGraphConditionalHandle h_while,
                            cudaGraphConditionalHandle h_b2l) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t again = 0, b2l = 0;
  if (!st->done) {
    uint32_t discovered;
    unsigned long long edges;
    if (st->dir == kDirTD) {
      st->mf = st->ctl.mf;
      st->qcount = st->ctl.qnext;
      st->lsize = st->ctl.lnext;
      st->par_l ^= 1u;
      st->td_steps++;
      discovered = st->qcount;
      edges = st->ctl.total_edges;
    } else {
      st->nf = st->ctl.nf;
      st->ul_size = st->ctl.ul_size;
      st->ul_valid = 1;
      st->par_ul ^= 1u;
      st->par_bm ^= 1u;
      st->bu_steps++;
      discovered = st->nf;
      edges = st->ctl.edges;
      const bool cont = (st->mode == BFS_PULL) ? (st->nf > 0)
                                               : ((st->nf > st->nf_prev) || (st->nf > st->n / kBeta));
      if (!cont) {
        st->in_bu = 0;
        st->need_b2l = 1;
        st->ctl.qnext = 0;
        st->ctl.lnext = 0;
        b2l = 1;
      }
    }
    st->processed += discovered;
    st->edges_examined += edges;
    if (st->nlevels < (uint32_t)kMaxTrace) {
      BfsLevel& L = st->trace[st->nlevels];
      L.direction = st->dir;
      L.discovered = discovered;
      L.frontier = st->frontier;
      L.mf = st->mf;
      L.mu = st->mu;
      L.edges = edges;
      L.ms = 0.0f;
    }
    st->nlevels++;
    st->iteration++;
    if (st->dir == kDirTD && st->qcount == 0) {
      st->done = 1;
    } else if (st->iteration > st->max_steps) {
      st->err = ERR_SPIN;
      st->done = 1;
    } else {
      again = 1;
    }
  }
  if (use_handles) {
    cudaGraphSetConditional(h_b2l, b2l);
    cudaGraphSetConditional(h_while, again);
  }
}

// ------------------------------------------------------------ conversions --

__global__ void __launch_bounds__(256) bfsk_clear_bitmap(BfsBufs b, const BfsDevState* __restrict__ st,
                                                         int next) {
  uint32_t* bm = b.bm[st->par_bm ^ (uint32_t)next];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.words; i += gridDim.x * blockDim.x) bm[i] = 0;
}

// arrayQueueToBitmap (arrayQueue.c:289-307) over the expansion list (the
// bitmap was cleared by bfsk_clear_bitmap).
__global__ void __launch_bounds__(256) bfsk_list_to_bitmap(BfsBufs b, const BfsDevState* __restrict__ st) {
  const uint32_t* q = b.list[st->par_l];
  uint32_t* bm = b.bm[st->par_bm];
  const uint32_t n = st->lsize;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = q[i];
    atomicOr(&bm[v >> 5], 1u << (v & 31));
  }
}

// bitmapToArrayQueue (arrayQueue.c:310-337): the logical size counts every
// set bit; the expansion list keeps the ones with out-edges.
__global__ void __launch_bounds__(256) bfsk_bitmap_to_list(BfsBufs b, BfsDevState* __restrict__ st) {
  constexpr uint32_t kRoundWords = 128;  // bitmap words per block round (<= 4096 bits)
  __shared__ BlockAppend<2 * kRoundWords * 32> q;
  ba_init(q);
  const uint32_t* bm = b.bm[st->par_bm];
  uint32_t* list = b.list[st->par_l];
  uint32_t cnt = 0;
  for (uint32_t rbase = blockIdx.x * kRoundWords; rbase < b.words; rbase += gridDim.x * kRoundWords) {
    const uint32_t w = rbase + threadIdx.x;
    if (threadIdx.x < kRoundWords && w < b.words) {
      uint32_t word = bm[w];
      cnt += __popc(word);
      while (word) {
        const int bit = __ffs(word) - 1;
        const uint32_t v = w * 32 + (uint32_t)bit;
        if (b.out_degree[v]) ba_push(q, v);
        word &= word - 1;
      }
    }
    if (ba_size(q) > kRoundWords * 32) ba_flush(q, list, &st->ctl.lnext);
  }
  ba_flush(q, list, &st->ctl.lnext);
  warp_atomic_add_total(&st->ctl.qnext, cnt);
}

// ------------------------------------------------------------ top-down -----

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

// Look-back word: value (32 bits) | flag (bits 32-33: 1 aggregate, 2
// inclusive) | epoch (bits 34-63).  A word from an older step never matches.
__device__ __forceinline__ unsigned long long lb_word(uint32_t epoch, uint32_t flag, uint32_t value) {
  return ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | ((unsigned long long)flag << 32) | value;
}

// Top-down, phase 1: exclusive scan of the out-degrees of the expansion list
// (single pass, decoupled look-back; CTAs claim tiles in order until the
// list is done).  Writes offs[i] (first edge of entry i in the level's edge
// range), fstart[i] (its first CSR edge), fdist[i] (its depth + 1), the total
// into ctl, and for every edge tile the list index of the entry holding the
// tile's first edge.
__global__ void __launch_bounds__(kScanT) bfsk_td_scan(BfsBufs b, BfsDevState* __restrict__ st) {
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ uint32_t s_w[kScanT / 32];
  const uint32_t* list = b.list[st->par_l];
  const uint32_t n = st->lsize;
  const uint32_t epoch = st->epoch;
  const uint32_t* distances = st->distances;
  BfsCtl* ctl = &st->ctl;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->scan_tiles, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if ((uint64_t)tile * kScanTile >= n) break;
    const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanI;
    uint32_t deg[kScanI], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanI; k++) {
      const uint64_t i = base + k;
      deg[k] = 0;
      if (i < n) {
        const uint32_t v = list[i];
        const uint2 r = b.rows_f[v];
        deg[k] = r.y;
        b.fstart[i] = r.x;
        b.fdist[i] = distances[v] + 1;
        sum += r.y;
      }
    }
    uint32_t tile_total = 0;
    const uint32_t excl = scan_block_excl(sum, s_w, &tile_total);
    if (threadIdx.x == 0) {
      uint32_t prefix = 0;
      unsigned long long* sw = b.status + tile;
      if (tile == 0) {
        st_volatile_u64(sw, lb_word(epoch, 2, tile_total));
      } else {
        st_volatile_u64(sw, lb_word(epoch, 1, tile_total));
        int64_t p = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (p >= 0) {
          const unsigned long long v = ld_volatile_u64(b.status + p);
          const uint32_t ep = (uint32_t)(v >> 34), flag = (uint32_t)(v >> 32) & 3u;
          if (ep != (epoch & 0x3FFFFFFFu) || flag == 0) {
            if (++spins > kSpinLimit) {
              atomicExch(&st->err, (uint32_t)ERR_SPIN);
              break;
            }
            continue;
          }
          prefix += (uint32_t)v;
          if (flag == 2) break;
          --p;
        }
        st_volatile_u64(sw, lb_word(epoch, 2, prefix + tile_total));
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
        b.offs[i] = o;
        // edge tiles whose first edge lies in [o, o + deg)
        for (uint32_t t = (o + kExpTile - 1) / kExpTile; (uint64_t)t * kExpTile < (uint64_t)o + deg[k]; t++)
          b.tile_i0[t] = (uint32_t)i;
        o += deg[k];
      }
    }
    __syncthreads();
  }
}

// Top-down, phase 2: each CTA takes whole tiles of kExpTile edges of the
// level; the list entries overlapping a tile are staged in shared memory and
// each edge finds its entry by binary search there.  A vertex is claimed by
// CAS on its parent; the winner appends it to the next frontier.
__global__ void __launch_bounds__(kExpT) bfsk_td_expand(BfsBufs b, BfsDevState* __restrict__ st) {
  __shared__ uint32_t s_off[kExpTile + 2], s_start[kExpTile + 2], s_v[kExpTile + 2], s_d[kExpTile + 2];
  __shared__ BlockAppend<kExpTile> q_list, q_all;
  ba_init(q_list);
  ba_init(q_all);
  const uint32_t* list = b.list[st->par_l];
  uint32_t* next_list = b.list[st->par_l ^ 1u];
  const uint32_t n = st->lsize;
  int32_t* parents = st->parents;
  uint32_t* distances = st->distances;
  BfsCtl* ctl = &st->ctl;
  const uint32_t total = ctl->total_edges;
  const uint32_t ntiles = (total + kExpTile - 1) / kExpTile;
  uint32_t mf = 0, found = 0;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t e0 = t * kExpTile;
    const uint32_t e1 = min(e0 + kExpTile, total);
    const uint32_t i0 = b.tile_i0[t];
    const uint32_t i1 = (t + 1 < ntiles) ? b.tile_i0[t + 1] : n - 1;
    const uint32_t cnt = i1 - i0 + 1;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < cnt; k += kExpT) {
      s_off[k] = b.offs[i0 + k];
      s_start[k] = b.fstart[i0 + k];
      s_v[k] = list[i0 + k];
      s_d[k] = b.fdist[i0 + k];
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
      const uint32_t u = b.nbr_f[s_start[lo] + (e - s_off[lo])] & 0x3FFFFFFFu;
      const int32_t p = parents[u];
      if (p < 0 && atomicCAS(&parents[u], p, (int32_t)s_v[lo]) == p) {
        distances[u] = s_d[lo];
        mf += (uint32_t)(-p);
        found++;
        if (b.all_out) ba_push(q_all, u);
        if (b.out_degree[u]) ba_push(q_list, u);
      }
    }
    // at most kExpTile discoveries per tile: flush every tile
    ba_flush(q_list, next_list, &ctl->lnext);
    if (b.all_out) ba_flush(q_all, b.all_out, &ctl->all_count);
  }
  warp_atomic_add_total(&ctl->mf, mf);
  warp_atomic_add_total(&ctl->qnext, found);
}

// ------------------------------------------------------------ bottom-up ----

// Scan v's in-edges in CSR order for the first in-neighbour in the frontier.
__device__ __forceinline__ bool bu_probe(const BfsBufs& b, const uint32_t* __restrict__ bm_cur, uint32_t v,
                                         int32_t* __restrict__ parents, uint32_t* __restrict__ distances,
                                         unsigned long long& edges) {
  const uint2 row = b.rows_i[v];
  uint32_t j = row.x;
  const uint32_t end = row.x + row.y;
  bool found = false;
  for (; j < end; j++) {
    const uint32_t u = b.nbr_i[j] & 0x3FFFFFFFu;
    if ((bm_cur[u >> 5] >> (u & 31)) & 1u) {
      parents[v] = (int32_t)u;
      distances[v] = distances[u] + 1;
      found = true;
      j++;
      break;
    }
  }
  edges += j - row.x;
  return found;
}

// First bottom-up level of a search: a warp covers 32 consecutive vertices,
// so its ballot is a whole word of the next bitmap (no atomics, no
// clearing).  Vertices left unvisited go to the unvisited list.
template <bool OR_INTO>
__global__ void __launch_bounds__(256) bfsk_bu_dense(BfsBufs b, BfsDevState* __restrict__ st) {
  constexpr uint32_t kRound = 1024;  // vertices per block round (4 bitmap words per warp)
  __shared__ BlockAppend<2 * kRound> q_ul;
  ba_init(q_ul);
  const uint32_t* bm_cur = b.bm[st->par_bm];
  uint32_t* bm_next = b.bm[st->par_bm ^ 1u];
  uint32_t* ul_next = b.ul[st->par_ul ^ 1u];
  int32_t* parents = st->parents;
  uint32_t* distances = st->distances;
  const uint32_t V = b.V;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t nf = 0;
  unsigned long long edges = 0;
  for (uint32_t rbase = blockIdx.x * kRound; rbase < V; rbase += gridDim.x * kRound) {
#pragma unroll
    for (uint32_t k = 0; k < kRound / 256; k++) {
      const uint32_t base = rbase + k * 256 + warp * 32;
      const uint32_t v = base + lane;
      bool found = false, unvisited = false;
      if (v < V && parents[v] < 0) {
        found = bu_probe(b, bm_cur, v, parents, distances, edges);
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
    if (ba_size(q_ul) > kRound) ba_flush(q_ul, ul_next, &st->ctl.ul_size);
  }
  ba_flush(q_ul, ul_next, &st->ctl.ul_size);
  warp_atomic_add_total(&st->ctl.nf, nf);
  warp_atomic_add_total64(&st->ctl.edges, (uint32_t)edges);
}

// Later bottom-up levels over the unvisited list (bm_next cleared first).
__global__ void __launch_bounds__(256) bfsk_bu_list(BfsBufs b, BfsDevState* __restrict__ st) {
  constexpr uint32_t kRound = 1024;  // list entries per block round
  __shared__ BlockAppend<2 * kRound> q_ul;
  ba_init(q_ul);
  const uint32_t* bm_cur = b.bm[st->par_bm];
  uint32_t* bm_next = b.bm[st->par_bm ^ 1u];
  const uint32_t* ul_cur = b.ul[st->par_ul];
  uint32_t* ul_next = b.ul[st->par_ul ^ 1u];
  const uint32_t count = st->ul_size;
  int32_t* parents = st->parents;
  uint32_t* distances = st->distances;
  uint32_t nf = 0;
  unsigned long long edges = 0;
  for (uint32_t rbase = blockIdx.x * kRound; rbase < count; rbase += gridDim.x * kRound) {
#pragma unroll
    for (uint32_t k = 0; k < kRound / 256; k++) {
      const uint32_t t = rbase + k * 256 + threadIdx.x;
      if (t >= count) continue;
      const uint32_t v = ul_cur[t];
      if (parents[v] >= 0) continue;  // visited by a top-down step since the list was made
      if (bu_probe(b, bm_cur, v, parents, distances, edges)) {
        atomicOr(&bm_next[v >> 5], 1u << (v & 31));
        nf++;
      } else {
        ba_push(q_ul, v);
      }
    }
    if (ba_size(q_ul) > kRound) ba_flush(q_ul, ul_next, &st->ctl.ul_size);
  }
  ba_flush(q_ul, ul_next, &st->ctl.ul_size);
  warp_atomic_add_total(&st->ctl.nf, nf);
  warp_atomic_add_total64(&st->ctl.edges, (uint32_t)edges);
}

// ------------------------------------------------------------ misc ---------

// Keep the entries of a queue that have out-edges (host-state step API).
__global__ void bfsk_filter_list(const uint32_t* __restrict__ in, uint32_t n, const uint32_t* __restrict__ out_degree,
                                 uint32_t* __restrict__ out, uint32_t* __restrict__ count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = in[i];
    if (out_degree[v]) out[warp_atomic_inc(count)] = v;
  }
}

// Number of reached vertices and the sum of their out-degrees (Graph500
// traversed edges).
__global__ void __launch_bounds__(256) bfsk_reached(BfsBufs b, BfsDevState* __restrict__ st) {
  const int32_t* parents = st->parents;
  unsigned long long e = 0;
  uint32_t r = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < b.V; v += gridDim.x * blockDim.x) {
    if (parents[v] >= 0) {
      r++;
      e += b.out_degree[v];
    }
  }
  for (int o = 16; o; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    r += __shfl_down_sync(0xffffffffu, r, o);
  }
  if (lane_id() == 0) {
    if (e) atomicAdd(&st->ctl.reached_edges, e);
    if (r) atomicAdd(&st->ctl.reached, r);
  }
}

__global__ void bfsk_zero_reached(BfsDevState* __restrict__ st) {
  st->ctl.reached = 0;
  st->ctl.reached_edges = 0;
}

// ------------------------------------------------------------ drivers ------

struct Grids {
  int v, small;
};
static Grids grids(const BfsBufs& b) {
  const int sms = sm_count();
  return {sms * 8, sms * 4};
}

// Launch the kernels of one step on `s` (host-stepped driver and graph
// capture share this).  `which`: 0 top-down, 1 bottom-up first, 2 bottom-up
// list, 3 list->bitmap, 4 bitmap->list.
static void launch_part(int which, const BfsBufs& b, BfsDevState* st, cudaStream_t s) {
  const Grids gr = grids(b);
  switch (which) {
    case 0:
      bfsk_td_scan<<<gr.v, kScanT, 0, s>>>(b, st);
      bfsk_td_expand<<<gr.v, kExpT, 0, s>>>(b, st);
      break;
    case 1:
      bfsk_bu_dense<false><<<gr.v, 256, 0, s>>>(b, st);
      break;
    case 2:
      bfsk_clear_bitmap<<<gr.small, 256, 0, s>>>(b, st, 1);
      bfsk_bu_list<<<gr.v, 256, 0, s>>>(b, st);
      break;
    case 3:
      bfsk_clear_bitmap<<<gr.small, 256, 0, s>>>(b, st, 0);
      bfsk_list_to_bitmap<<<gr.small, 256, 0, s>>>(b, st);
      break;
    case 4:
      bfsk_bitmap_to_list<<<gr.small, 256, 0, s>>>(b, st);
      break;
  }
}

static int add_if(cudaGraph_t g, cudaGraphNode_t* node, cudaGraphNode_t dep, cudaGraphConditionalHandle h,
                  cudaGraph_t* body) {
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeIf;
  p.conditional.size = 1;
  OGB_CUDA(cudaGraphAddNode(node, g, dep ? &dep : nullptr, dep ? 1 : 0, &p));
  *body = p.conditional.phGraph_out[0];
  return OK;
}

static int capture_into(cudaGraph_t body, cudaStream_t cap, int which, const BfsBufs& b, BfsDevState* st) {
  OGB_CUDA(cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  launch_part(which, b, st, cap);
  cudaGraph_t out = nullptr;
  OGB_CUDA(cudaStreamEndCapture(cap, &out));
  return OK;
}

template <class... A>
static int add_kernel(cudaGraph_t g, cudaGraphNode_t* node, cudaGraphNode_t dep, void (*fn)(A...), void** args) {
  cudaKernelNodeParams p = {};
  p.func = reinterpret_cast<void*>(fn);
  p.gridDim = dim3(1);
  p.blockDim = dim3(32);
  p.sharedMemBytes = 0;
  p.kernelParams = args;
  p.extra = nullptr;
  OGB_CUDA(cudaGraphAddKernelNode(node, g, dep ? &dep : nullptr, dep ? 1 : 0, &p));
  return OK;
}

// The search loop as one executable graph (per graph buffers, mode and
// bottom-up entry rule).
static int build_search_graph(BfsWork* w, const BfsBufs& b, cudaGraphExec_t* exec) {
  BfsDevState* st = w->state.as<BfsDevState>();
  cudaGraph_t g = nullptr;
  OGB_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h_while, h_b2l, h_l2b, h_td, h_bud, h_bul;
  OGB_CUDA(cudaGraphConditionalHandleCreate(&h_while, g, 1, cudaGraphCondAssignDefault));
  OGB_CUDA(cudaGraphConditionalHandleCreate(&h_b2l, g, 0, cudaGraphCondAssignDefault));
  OGB_CUDA(cudaGraphConditionalHandleCreate(&h_l2b, g, 0, cudaGraphCondAssignDefault));
  OGB_CUDA(cudaGraphConditionalHandleCreate(&h_td, g, 0, cudaGraphCondAssignDefault));
  OGB_CUDA(cudaGraphConditionalHandleCreate(&h_bud, g, 0, cudaGraphCondAssignDefault));
  OGB_CUDA(cudaGraphConditionalHandleCreate(&h_bul, g, 0, cudaGraphCondAssignDefault));
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = h_while;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  OGB_CUDA(cudaGraphAddNode(&wnode, g, nullptr, 0, &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];

  int use = 1;
  cudaGraphNode_t n_b2l, n_dec, n_l2b, n_td, n_bud, n_bul, n_fin;
  cudaGraph_t bb;
  OGB_TRY(add_if(body, &n_b2l, nullptr, h_b2l, &bb));
  OGB_TRY(capture_into(bb, w->cap, 4, b, st));
  void* dec_args[] = {&st, &use, &h_l2b, &h_td, &h_bud, &h_bul};
  OGB_TRY(add_kernel(body, &n_dec, n_b2l, bfsk_decide, dec_args));
  OGB_TRY(add_if(body, &n_l2b, n_dec, h_l2b, &bb));
  OGB_TRY(capture_into(bb, w->cap, 3, b, st));
  OGB_TRY(add_if(body, &n_td, n_l2b, h_td, &bb));
  OGB_TRY(capture_into(bb, w->cap, 0, b, st));
  OGB_TRY(add_if(body, &n_bud, n_td, h_bud, &bb));
  OGB_TRY(capture_into(bb, w->cap, 1, b, st));
  OGB_TRY(add_if(body, &n_bul, n_bud, h_bul, &bb));
  OGB_TRY(capture_into(bb, w->cap, 2, b, st));
  void* fin_args[] = {&st, &use, &h_while, &h_b2l};
  OGB_TRY(add_kernel(body, &n_fin, n_bul, bfsk_finish, fin_args));
  cudaError_t e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(ERR_CUDA, "bfs graph instantiate: %s", cudaGetErrorString(e));
  return OK;
}

static int read_state(BfsWork* w, cudaStream_t s) {
  OGB_CUDA(cudaMemcpyAsync(w->h_state, w->state.p, offsetof(BfsDevState, trace), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

int bfs_run(DevGraph& g, uint32_t root, uint32_t mode, int32_t* parents, uint32_t* distances, BfsResult* res,
            bool time_levels, bool bu_entry_nf_frontier, cudaStream_t s) {
  const uint32_t V = g.V;
  if (root >= V) return fail(ERR_ARG, "bfs: root %u out of range (V=%u)", root, V);
  if (mode > BFS_DO) return fail(ERR_ARG, "bfs: mode %u", mode);
  BfsWork* w = nullptr;
  OGB_TRY(bfs_work_get(g, &w));
  const BfsBufs b = make_bufs(g, w, nullptr);
  BfsDevState* st = w->state.as<BfsDevState>();
  const Grids gr = grids(b);
  std::vector<float> level_ms;

  bfsk_init<<<gr.v, 256, 0, s>>>(b, st, root, parents, distances, mode, bu_entry_nf_frontier ? 1u : 0u, g.E);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaEventRecord(w->ev_start, s));
  uint32_t launches = 1;
  if (!time_levels) {
    BfsGraph& gg = w->graphs[mode][bu_entry_nf_frontier ? 1 : 0];
    if (!gg.exec) OGB_TRY(build_search_graph(w, b, &gg.exec));
    OGB_CUDA(cudaGraphLaunch(gg.exec, s));
  } else {
    // host-stepped: the same kernels, one step at a time, timed with events
    BfsDevState* h = w->h_state;
    OGB_TRY(read_state(w, s));
    while (!h->done) {
      if (h->need_b2l) {
        launch_part(4, b, st, s);
        launches++;
      }
      bfsk_decide<<<1, 32, 0, s>>>(st, 0, 0, 0, 0, 0);
      OGB_TRY(read_state(w, s));
      launches++;
      if (h->done) break;
      if (h->l2b_now) {
        launch_part(3, b, st, s);
        launches += 2;
      }
      OGB_CUDA(cudaEventRecord(w->ev_a, s));
      const int part = h->dir == kDirTD ? 0 : (h->dense_now ? 1 : 2);
      launch_part(part, b, st, s);
      launches += (part == 1) ? 1 : 2;
      OGB_CUDA(cudaEventRecord(w->ev_b, s));
      bfsk_finish<<<1, 32, 0, s>>>(st, 0, 0, 0);
      launches++;
      OGB_CUDA(cudaGetLastError());
      OGB_TRY(read_state(w, s));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, w->ev_a, w->ev_b);
      level_ms.push_back(ms);
    }
  }
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaEventRecord(w->ev_stop, s));
  bfsk_zero_reached<<<1, 1, 0, s>>>(st);
  bfsk_reached<<<gr.v, 256, 0, s>>>(b, st);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaMemcpyAsync(w->h_state, w->state.p, sizeof(BfsDevState), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  float total_ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&total_ms, w->ev_start, w->ev_stop));
  const BfsDevState* h = w->h_state;
  if (h->err) return fail((int)h->err, "bfs: a bounded device loop gave up");
  BfsResult r;
  r.iteration = h->iteration;
  r.processed_nodes = h->processed;
  r.td_steps = h->td_steps;
  r.bu_steps = h->bu_steps;
  r.edges_examined = h->edges_examined;
  r.reached = h->ctl.reached;
  r.reached_out_edges = h->ctl.reached_edges;
  r.ms = total_ms;
  r.launches = time_levels ? launches : 1 + 3 * (h->td_steps + h->bu_steps);
  r.nlevels = (int)std::min<uint32_t>(h->nlevels, kMaxTrace);
  for (int i = 0; i < r.nlevels; i++) {
    r.levels[i] = h->trace[i];
    if (i < (int)level_ms.size()) r.levels[i].ms = level_ms[i];
  }
  if (res) *res = r;
  return OK;
}

}  // namespace ogb

using namespace ogb;

// One top-down level over host state (topDownStepGraphCSR, BFS.c:639-687):
// the window's vertices with out-edges are expanded on the device and every
// vertex the level claims is returned in discovery order.
int bfs_td_step_host(DevGraph& g, const uint32_t* q, uint32_t qsize, int32_t* parents, uint32_t* distances,
                     uint32_t* next_q, uint32_t* next_size, uint32_t* mf, cudaStream_t s) {
  BfsWork* w = nullptr;
  OGB_TRY(bfs_work_get(g, &w));
  const uint32_t V = g.V;
  DevBuf d_par, d_dist, d_all, d_cnt;
  OGB_TRY(d_par.alloc((size_t)V * 4 + 4));
  OGB_TRY(d_dist.alloc((size_t)V * 4 + 4));
  OGB_TRY(d_all.alloc((size_t)V * 4 + 4));
  OGB_TRY(d_cnt.alloc(16));
  OGB_CUDA(cudaMemcpyAsync(d_par.p, parents, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(d_dist.p, distances, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->ul0.p, q, (size_t)qsize * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemsetAsync(d_cnt.p, 0, 16, s));
  if (qsize) {
    bfsk_filter_list<<<std::min<uint32_t>(sm_count() * 8, ceil_div(qsize, 256)), 256, 0, s>>>(
        w->ul0.as<uint32_t>(), qsize, g.fwd.d_out_degree(), w->q0.as<uint32_t>(), d_cnt.as<uint32_t>());
    OGB_CUDA(cudaGetLastError());
  }
  uint32_t n = 0;
  OGB_CUDA(cudaMemcpyAsync(&n, d_cnt.p, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  // a state for one step: list 0 holds the window, epoch one past the last
  BfsDevState* h = w->h_state;
  OGB_CUDA(cudaMemcpyAsync(h, w->state.p, offsetof(BfsDevState, trace), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  const uint32_t epoch = h->epoch + 1;
  memset(h, 0, offsetof(BfsDevState, trace));
  h->n = V;
  h->E = g.E;
  h->parents = d_par.as<int32_t>();
  h->distances = d_dist.as<uint32_t>();
  h->lsize = n;
  h->epoch = epoch;
  h->dir = kDirTD;
  OGB_CUDA(cudaMemcpyAsync(w->state.p, h, offsetof(BfsDevState, trace), cudaMemcpyHostToDevice, s));
  const BfsBufs b = make_bufs(g, w, d_all.as<uint32_t>());
  if (n) launch_part(0, b, w->state.as<BfsDevState>(), s);
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(read_state(w, s));
  *next_size = h->ctl.qnext;
  *mf = h->ctl.mf;
  OGB_CUDA(cudaMemcpyAsync(next_q, d_all.p, (size_t)(*next_size) * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(parents, d_par.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(distances, d_dist.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

// One bottom-up level over host state (bottomUpStepGraphCSR, BFS.c:703-754):
// bits of discovered vertices are OR-ed into the caller's next bitmap.
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
  BfsDevState* h = w->h_state;
  OGB_CUDA(cudaMemcpyAsync(h, w->state.p, offsetof(BfsDevState, trace), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  const uint32_t epoch = h->epoch;
  memset(h, 0, offsetof(BfsDevState, trace));
  h->n = V;
  h->parents = d_par.as<int32_t>();
  h->distances = d_dist.as<uint32_t>();
  h->epoch = epoch;
  h->dir = kDirBU;
  OGB_CUDA(cudaMemcpyAsync(w->state.p, h, offsetof(BfsDevState, trace), cudaMemcpyHostToDevice, s));
  const BfsBufs b = make_bufs(g, w, nullptr);
  bfsk_bu_dense<true><<<sm_count() * 8, 256, 0, s>>>(b, w->state.as<BfsDevState>());
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(read_state(w, s));
  *nf = h->ctl.nf;
  OGB_CUDA(cudaMemcpyAsync(bm_next, w->bm1.p, words * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(parents, d_par.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(distances, d_dist.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}
