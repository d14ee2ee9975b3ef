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
//  * a whole search is ONE cooperative launch (bfsk_search): the CTAs run the
//    level loop together and meet at grid barriers between phases.  Every
//    CTA keeps its own copy of the switch state in shared memory and updates
//    it from the same per-phase counters, so all copies agree without an
//    extra barrier; no host round trip and no launch per level.  Every
//    barrier wait is bounded (error word, then exit) and the loop is bounded
//    by V + 8 steps.  The learned switch (mode BFS_LEARNED) decides each step
//    from a linear prior and, near its boundary, a small network;
//  * the search is level-synchronous, so every frontier vertex has the same
//    depth: a discovered vertex gets depth + 1 without reading its parent's
//    distance (what the reference computes as distances[parent] + 1);
//  * the frontier is kept twice: its logical size (every vertex discovered
//    by the last step, which drives the loop) and an expansion list of the
//    frontier vertices WITH out-edges -- a vertex without out-edges is never
//    expanded top-down and never probed bottom-up (it is nobody's
//    in-neighbour), so it needs no slot;
//  * top-down is load-balanced by edges: a chained scan over the list's
//    out-degrees gives each vertex its edge offset and scatters, for every
//    tile of kExpTile edges, the list index where the tile starts; the expand
//    phase then gives each CTA whole edge tiles (coalesced neighbour reads,
//    independent of the degree skew).  The scan's look-back words carry the
//    scan's epoch, so they never need clearing;
//  * bottom-up: the first bottom-up level of a search walks a cached list of
//    the graph's vertices with in-edges (built once per graph: a vertex
//    without one can never be found bottom-up), later levels walk the
//    compacted list of still-unvisited vertices; each CTA takes one equal,
//    contiguous range of candidates; a candidate's first kFirst in-neighbours
//    and their frontier bits are loaded at once, longer rows go to a per-round
//    list scanned by groups of 8 lanes (the first hit in CSR order still
//    wins); the dense-probe mode walks every vertex (a warp's ballot is one
//    whole word of the next bitmap);
//  * a top-down step sets the bitmap bit of every vertex it discovers and a
//    bottom-up step lists the vertices it discovers, so a change of
//    direction needs no conversion pass (arrayQueueToBitmap /
//    bitmapToArrayQueue, arrayQueue.c:289-337); three bitmaps rotate (read,
//    write, clear), so every step clears the bitmap a later step writes while
//    it runs;
//  * a top-down step whose list has at most kExpTile entries runs as one
//    phase: every CTA scans the short list itself; up to kMidList entries it
//    is one phase too, the CTAs that own an edge tile scanning the list;
//  * queue appends are staged per CTA in shared memory (one global atomic
//    per flush); counters are summed per CTA (one atomic per CTA);
//  * bitmaps: bit v = word v>>5, bit v&31 (bitmap.h:7-9).
#include <cuda_bf16.h>

#include "graph.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace ogb {

constexpr int kScanT = 256;            // threads of the degree scan
constexpr int kScanI = 8;              // list entries per thread
constexpr int kScanTile = kScanT * kScanI;
constexpr int kExpT = 256;             // threads of the expand phase
constexpr uint32_t kExpTile = 1024;    // edges per expand tile
constexpr int kSearchT = 256;          // threads per CTA of the persistent search
constexpr int kMaxTrace = 16384;    // steps whose trace and switch inputs are kept
constexpr uint32_t kAlpha = 15, kBeta = 18;
constexpr uint32_t kBuRound = 1024;    // vertices per CTA round of a bottom-up step
constexpr uint32_t kBuSub = 2;         // list step: load/probe passes of kBuRound records per round,
                                       // before one long-row phase and one flush
constexpr uint32_t kBuCap = kBuSub * kBuRound;  // appends and long rows a round can hold

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
  uint32_t maxdeg;            // largest out-degree on the next expansion list
  unsigned long long fedges;  // out-edges of the vertices the step discovered
};

// The reference's switch state plus this search's bookkeeping.  Each CTA of
// bfsk_search holds one copy in shared memory.
struct BfsCtrl {
  uint32_t mode, bu_entry_frontier, n, max_steps;
  uint32_t mu, mf, nf, nf_prev;
  uint32_t qcount, lsize, frontier, in_bu;
  uint32_t ul_valid, ul_size, par_l, par_ul;
  uint32_t bm_r, bm_w, bm_c, depth;
  uint32_t iteration, processed, td_steps, bu_steps;
  uint32_t nlevels, epoch, overflow, qcount_prev;
  uint32_t ul_cand0;                 // 1: the unvisited list is the graph's cached in-edge list
  uint32_t ul_fresh;                 // 1: the unvisited list comes from the step just before (all unvisited)
  uint32_t lmax;                     // largest out-degree on the expansion list
  unsigned long long edges_examined;
  unsigned long long fedges;         // out-edges of the current frontier
  unsigned long long edges_visited;  // out-edges of every visited vertex
};

// Inputs of the learned direction switch, from the state before a step.
constexpr int kFeat = 8;

struct BfsDevState {
  BfsCtrl c;
  int32_t* parents;
  uint32_t* distances;
  uint32_t err;       // ERR_SPIN when a bounded wait gave up
  uint32_t bar;       // grid barrier word
  uint32_t pad[2];
  BfsCtl ctl[3];      // per-phase counters, rotating
  BfsCtl aux;         // reached counts and the host-state steps
  BfsLevel trace[kMaxTrace];
  float feat[kMaxTrace][kFeat];  // switch inputs before every step
};

// Device buffers of one graph (fixed; passed by value to every kernel).
struct BfsBufs {
  const uint2* rows_f;
  const uint32_t* nbr_f;
  const uint2* rows_i;
  const uint32_t* nbr_i;
  const uint32_t* out_degree;
  uint32_t* list[2];
  uint32_t* bm[3];
  uint32_t* ul[2];
  // Candidate records of the bottom-up steps that walk a list (two 16-byte
  // words per candidate, in two arrays): the first such step's (every vertex
  // with in-edges, in vertex order; built once per graph) and the unvisited
  // lists the steps hand on, rotating.
  const uint4* cand_a;
  const uint4* cand_b;
  uint4* ul_a[2];
  uint4* ul_b[2];
  uint32_t* offs;
  uint32_t* fstart;
  uint32_t* fdist;
  uint32_t* tile_i0;
  unsigned long long* status;
  uint32_t V, words, E, pad;
  const __nv_bfloat16* policy;  // learned switch network (8 -> 64 -> 64 -> 1, bf16), or null
  const float* policy_tail;     // its linear prior (8 coefficients, bias) and correction bound
};

const __nv_bfloat16* bfs_policy_weights();
const float* bfs_policy_tail();

struct BfsWork {
  uint32_t V = 0, E = 0;
  DevBuf q0, q1, bm0, bm1, bm2, ul0, ul1, state;
  DevBuf offs, fstart, fdist, tile_i0, scan_status;
  DevBuf cand_a, cand_b;            // records of the vertices with in-edges (built once per graph)
  DevBuf ul_a0, ul_a1, ul_b0, ul_b1;  // records of the unvisited lists (at most n_cand0 each)
  uint32_t n_cand0 = 0, cand0_build = 0;
  bool cand0_ready = false;
  BfsDevState* h_state = nullptr;   // pinned copy of the header only (up to the trace)
  uint32_t epoch = 0;               // last scan epoch used
  int search_grid = 0;          // CTAs of the search launch (co-resident)
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  ~BfsWork() {
    if (h_state) cudaFreeHost(h_state);
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_stop) cudaEventDestroy(ev_stop);
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
    OGB_TRY(w->bm2.alloc(words * 4 + 16));
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
  // the header (control state, error word, counters) is all the host reads
  // back through it; the trace arrays after it are copied on request
  if (!w->h_state) OGB_CUDA(cudaMallocHost(&w->h_state, offsetof(BfsDevState, trace)));
  if (!w->ev_start) {
    OGB_CUDA(cudaEventCreate(&w->ev_start));
    OGB_CUDA(cudaEventCreate(&w->ev_stop));
  }
  *out = w;
  return OK;
}

static BfsBufs make_bufs(DevGraph& g, BfsWork* w) {
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
  b.bm[2] = w->bm2.as<uint32_t>();
  b.ul[0] = w->ul0.as<uint32_t>();
  b.ul[1] = w->ul1.as<uint32_t>();
  b.cand_a = w->cand_a.as<uint4>();
  b.cand_b = w->cand_b.as<uint4>();
  b.ul_a[0] = w->ul_a0.as<uint4>();
  b.ul_a[1] = w->ul_a1.as<uint4>();
  b.ul_b[0] = w->ul_b0.as<uint4>();
  b.ul_b[1] = w->ul_b1.as<uint4>();
  b.offs = w->offs.as<uint32_t>();
  b.fstart = w->fstart.as<uint32_t>();
  b.fdist = w->fdist.as<uint32_t>();
  b.tile_i0 = w->tile_i0.as<uint32_t>();
  b.status = w->scan_status.as<unsigned long long>();
  b.V = g.V;
  b.words = (g.V + 31) / 32;
  b.E = g.E;
  b.pad = 0;
  b.policy = bfs_policy_weights();
  b.policy_tail = bfs_policy_tail();
  return b;
}

// ------------------------------------------------------------ learned switch

// The installed direction policy (none: null), per process: the network in
// bf16 (W2 transposed), then, 16-byte aligned, the fp32 tail (prior
// coefficients, prior bias, correction bound).
constexpr int kPolMlpN = 64 * 8 + 64 + 64 * 64 + 64 + 64 + 1;  // the library's MLP packing
constexpr int kPolTail = 8 + 1 + 1;
constexpr size_t kPolTailOff = ((size_t)kPolMlpN * 2 + 15) / 16 * 16;
static DevBuf g_policy;
static bool g_policy_set = false;
const __nv_bfloat16* bfs_policy_weights() { return g_policy_set ? g_policy.as<__nv_bfloat16>() : nullptr; }
const float* bfs_policy_tail() {
  return g_policy_set ? reinterpret_cast<const float*>(g_policy.as<char>() + kPolTailOff) : nullptr;
}

__global__ void bfsk_policy_to_bf16(const float* __restrict__ p, int n, __nv_bfloat16* __restrict__ q) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) q[i] = __float2bfloat16_rn(p[i]);
}

int bfs_set_policy(const float* params_host) {
  if (!params_host) {
    g_policy_set = false;
    return OK;
  }
  // the library's packing (W1, b1, W2[i][j], b2, w3, b3) with W2 transposed
  constexpr int in = 8, h = 64, np = kPolMlpN;
  const float* tail = params_host + np;
  for (int i = 0; i < kPolTail; i++)
    if (!std::isfinite(tail[i])) return fail(ERR_ARG, "bfs_set_policy: prior entry %d is not finite", i);
  if (tail[kPolTail - 1] < 0.f) return fail(ERR_ARG, "bfs_set_policy: negative correction bound");
  std::vector<float> p(params_host, params_host + np);
  const int w2 = h * in + h;
  for (int i = 0; i < h; i++)
    for (int j = 0; j < h; j++) p[w2 + j * h + i] = params_host[w2 + i * h + j];
  DevBuf tmp;
  OGB_TRY(tmp.alloc(np * 4));
  g_policy_set = false;
  OGB_TRY(g_policy.alloc(kPolTailOff + kPolTail * 4));
  OGB_CUDA(cudaMemcpy(tmp.p, p.data(), np * 4, cudaMemcpyHostToDevice));
  OGB_CUDA(cudaMemcpy(g_policy.as<char>() + kPolTailOff, tail, kPolTail * 4, cudaMemcpyHostToDevice));
  bfsk_policy_to_bf16<<<(np + 255) / 256, 256>>>(tmp.as<float>(), np, g_policy.as<__nv_bfloat16>());
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaDeviceSynchronize());
  g_policy_set = true;
  return OK;
}

// ------------------------------------------------------------ shared memory

struct ScanSmem {
  uint32_t w[kScanT / 32];
  uint32_t tile, prefix;
};
// Top-down: the list entries of one edge tile (or the whole list of a small
// step) and the step's appends.  The search keeps only what it uses (the
// rest of the SM's shared memory is L1, which its gathers need); the
// host-state step adds the entries' depths and a list of every discovery.
struct TdSmem {
  static constexpr bool kHost = false;
  uint32_t off[kExpTile + 2], start[kExpTile + 2], v[kExpTile + 2];
  BlockAppend<kExpTile> q_list;
  uint32_t w[kExpT / 32];
  uint32_t lo, hi;  // mid-size step: the list entries holding a tile's first and last edge
};
struct TdSmemHost : TdSmem {
  static constexpr bool kHost = true;
  uint32_t d[kExpTile + 2];
  BlockAppend<kExpTile> q_all;
};
// Bottom-up: a round's appends and its deferred long in-edge rows.  A round
// appends each of its at most kBuCap candidates to at most one list, so
// the new frontier list fills one buffer from the front and the unvisited
// list from the back.
struct BuSmem {
  uint32_t nlist, nul, base_list, base_ul;
  uint32_t buf[kBuCap];
  uint32_t nheavy;
  uint32_t hv[kBuCap];
};
__device__ __forceinline__ void bu_push_list(BuSmem& sm, uint32_t v) { sm.buf[warp_atomic_inc(&sm.nlist)] = v; }
__device__ __forceinline__ void bu_push_ul(BuSmem& sm, uint32_t v) {
  sm.buf[kBuCap - 1u - warp_atomic_inc(&sm.nul)] = v;
}
// A round's appends out, then the buffer and the long-row list are empty:
// discoveries (vertices) into list_out, and the records of the unvisited
// candidates (staged as indices into in_a / in_b) copied into out_a /
// out_b; the offsets of both are reserved together.
__device__ __forceinline__ void bu_flush(BuSmem& sm, uint32_t* list_out, uint32_t* list_count,
                                             const uint4* in_a, const uint4* in_b, uint4* out_a, uint4* out_b,
                                             uint32_t* ul_count) {
  __syncthreads();
  const uint32_t nl = sm.nlist, nu = sm.nul;
  if (threadIdx.x == 0) {
    uint32_t bl = 0, bu = 0;
    if (nl) bl = atomicAdd(list_count, nl);
    if (nu) bu = atomicAdd(ul_count, nu);
    sm.base_list = bl;
    sm.base_ul = bu;
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < nl; k += blockDim.x) list_out[sm.base_list + k] = sm.buf[k];
  for (uint32_t k = threadIdx.x; k < nu; k += blockDim.x) {
    const uint32_t s = sm.buf[kBuCap - 1u - k];
    out_a[sm.base_ul + k] = in_a[s];
    out_b[sm.base_ul + k] = in_b[s];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    sm.nlist = 0;
    sm.nul = 0;
    sm.nheavy = 0;  // the round's long rows were all read before the first barrier above
  }
  __syncthreads();
}

// A flat top-down step's appends: each of a CTA's threads expands one list
// entry of at most kFlatMaxDeg out-edges per pass.
constexpr uint32_t kFlatMaxDeg = 16;
constexpr uint32_t kFlatCap = 256 * kFlatMaxDeg;
union BfsSmem {
  ScanSmem scan;
  TdSmem td;
  BuSmem bu;
  BlockAppend<kFlatCap> flat;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void grid_clear(uint32_t* a, uint32_t* b2, uint32_t words) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) {
    if (a) a[i] = 0;
    if (b2) b2[i] = 0;
  }
}

// ------------------------------------------------------------ grid barrier -

// Barrier of all CTAs of a cooperative launch.  One counter: CTA 0 adds
// 2^31 - (grid - 1), every other CTA adds 1, so bit 31 flips exactly when the
// last CTA arrives and the low bits return to 0 (the word starts at 0).
// Thread 0 arrives with a release add at GPU scope (after the CTA's
// __syncthreads, so the CTA's writes come before it) and polls with acquire
// loads; this replaces a fence on either side (measured 2.6 us instead of
// 3.1 us per barrier of 740 CTAs).  The wait is bounded; a CTA that gives up,
// or sees the error word set by another, returns false and the caller leaves
// the search.
__device__ __forceinline__ bool grid_sync(uint32_t* bar, uint32_t* err, uint32_t* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
    uint32_t old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(bar), "r"(add) : "memory");
    uint32_t ok = 1, spins = 0;
    for (;;) {
      uint32_t cur;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(bar) : "memory");
      if ((old ^ cur) & 0x80000000u) break;
      if (ld_volatile_u32(err)) {
        ok = 0;
        break;
      }
      if (++spins > kSpinLimit) {
        atomicExch(err, (uint32_t)ERR_SPIN);
        ok = 0;
        break;
      }
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// ------------------------------------------------------------ top-down -----

// Exclusive block scan (kScanT == kExpT threads).
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

// Per-CTA sums of two 64-bit values and the maximum of a 32-bit one in one
// reduction (one pair of barriers); the results are valid in thread 0.  A
// step's 32-bit counts travel packed two to a value (low | high << 32): each
// half sums to less than 2^32 in a CTA (at most V vertices or E edges), so
// no carry crosses halves.  s_red holds kRedSlots * (warps per CTA) entries.
constexpr int kRedSlots = 3;
__device__ __forceinline__ void block_sum2_max(unsigned long long& a, unsigned long long& b, uint32_t& m,
                                               unsigned long long* s_red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  m = __reduce_max_sync(0xffffffffu, m);
  const uint32_t warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane_id() == 0) {
    s_red[warp] = a;
    s_red[nw + warp] = b;
    s_red[2 * nw + warp] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = b = 0;
    m = 0;
    for (uint32_t i = 0; i < nw; i++) {
      a += s_red[i];
      b += s_red[nw + i];
      m = max(m, (uint32_t)s_red[2 * nw + i]);
    }
  }
}

// A top-down step's counters: mf and the discoveries, packed, the
// discoveries' out-edges, and the largest out-degree it put on the list.
__device__ __forceinline__ void td_publish(BfsCtl* ctl, uint32_t mf, uint32_t found, unsigned long long fed,
                                           uint32_t mx, unsigned long long* s_red) {
  unsigned long long a = (unsigned long long)mf | ((unsigned long long)found << 32), b = fed;
  block_sum2_max(a, b, mx, s_red);
  if (threadIdx.x == 0) {
    if ((uint32_t)a) atomicAdd(&ctl->mf, (uint32_t)a);
    if (a >> 32) atomicAdd(&ctl->qnext, (uint32_t)(a >> 32));
    if (b) atomicAdd(&ctl->fedges, b);
    if (mx) atomicMax(&ctl->maxdeg, mx);
  }
}

// Look-back word: value (32 bits) | flag (bits 32-33: 1 aggregate, 2
// inclusive) | epoch (bits 34-63).  A word of an older scan never matches.
__device__ __forceinline__ unsigned long long lb_word(uint32_t epoch, uint32_t flag, uint32_t value) {
  return ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | ((unsigned long long)flag << 32) | value;
}

// Top-down, part 1: exclusive scan of the out-degrees of the expansion list
// (single pass, decoupled look-back; CTAs claim tiles in order until the
// list is done).  Writes offs[i] (first edge of entry i in the level's edge
// range), fstart[i] (its first CSR edge), fdist[i] (its depth + 1, unless
// the depth is known), the total into ctl, and for every edge tile the list
// index of the entry holding the tile's first edge.
template <bool kDepthKnown>
__device__ void td_scan_phase(const BfsBufs& b, const uint32_t* list, uint32_t n, const uint32_t* distances,
                              uint32_t epoch, BfsCtl* ctl, uint32_t* err, ScanSmem& sm) {
  if ((uint64_t)blockIdx.x * kScanTile >= n) return;  // the lower CTAs claim every tile
  for (;;) {
    if (threadIdx.x == 0) sm.tile = atomicAdd(&ctl->scan_tiles, 1u);
    __syncthreads();
    const uint32_t tile = sm.tile;
    if ((uint64_t)tile * kScanTile >= n) break;
    const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanI;
    uint32_t deg[kScanI], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanI; k++) {
      const uint64_t i = base + k;
      deg[k] = 0;
      if (i < n) {
        const uint32_t v = list[i];
        const uint2 r = __ldg(&b.rows_f[v]);
        deg[k] = r.y;
        b.fstart[i] = r.x;
        if (!kDepthKnown) b.fdist[i] = distances[v] + 1;
        sum += r.y;
      }
    }
    uint32_t tile_total = 0;
    const uint32_t excl = scan_block_excl(sum, sm.w, &tile_total);
    if (threadIdx.x < 32) {
      // decoupled look-back, one warp: lane l reads the status of tile
      // (window - l); 32 predecessors per round trip
      const uint32_t lane = threadIdx.x;
      const uint32_t want = epoch & 0x3FFFFFFFu;
      unsigned long long* sw = b.status + tile;
      if (lane == 0) st_volatile_u64(sw, lb_word(epoch, tile == 0 ? 2u : 1u, tile_total));
      uint32_t prefix = 0;
      int64_t window = (int64_t)tile - 1;
      uint32_t spins = 0;
      while (window >= 0) {
        const int64_t idx = window - (int64_t)lane;
        uint32_t flag, val;
        for (;;) {
          flag = 2;  // past tile 0: an inclusive zero
          val = 0;
          if (idx >= 0) {
            const unsigned long long v = ld_volatile_u64(b.status + idx);
            flag = ((uint32_t)(v >> 34) == want) ? ((uint32_t)(v >> 32) & 3u) : 0u;
            val = (uint32_t)v;
          }
          if (__all_sync(0xffffffffu, flag != 0)) break;
          if (++spins > kSpinLimit) {
            if (lane == 0) atomicExch(err, (uint32_t)ERR_SPIN);
            flag = 2;
            break;
          }
        }
        const uint32_t incl = __ballot_sync(0xffffffffu, flag == 2);
        const uint32_t stop = incl ? (uint32_t)(__ffs(incl) - 1) : 31u;
        uint32_t x = lane <= stop ? val : 0u;
#pragma unroll
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        prefix += x;
        if (incl) break;
        window -= 32;
      }
      if (lane == 0) {
        if (tile != 0) st_volatile_u64(sw, lb_word(epoch, 2, prefix + tile_total));
        sm.prefix = prefix;
        if ((uint64_t)(tile + 1) * kScanTile >= n) ctl->total_edges = prefix + tile_total;
      }
    }
    __syncthreads();
    uint32_t o = sm.prefix + excl;
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
// Expand the step's edges [e0, e1); staged entries [0, cnt) cover them
// (sm.off holds each entry's first edge in the step's edge range).  Each
// thread takes four edges at once: neighbour ids, then their parents, then
// the claiming CASes, each group issued back to back.  A claimed vertex gets
// its depth, its bit in bm_w (when given) and, with out-edges, a list slot.
template <bool kDepthKnown, class TS>
__device__ __forceinline__ void expand_edges(const BfsBufs& b, uint32_t e0, uint32_t e1, uint32_t cnt,
                                             int32_t* parents, uint32_t* distances, uint32_t dnext, uint32_t* bm_w,
                                             uint32_t* all_out, TS& sm, uint32_t& mf, uint32_t& found,
                                             unsigned long long& fed, uint32_t& mx) {
  static_assert(kDepthKnown || TS::kHost, "entry depths live in the host-step shared memory");
  constexpr int K = kExpTile / kExpT;
  uint32_t u[K], src[K], dd[K];
  bool ok[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    const uint32_t e = e0 + threadIdx.x + k * kExpT;
    ok[k] = e < e1;
    u[k] = 0;
    src[k] = 0;
    dd[k] = dnext;
    if (ok[k]) {
      uint32_t lo = 0, hi = cnt - 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (sm.off[mid] <= e)
          lo = mid;
        else
          hi = mid - 1;
      }
      u[k] = __ldg(&b.nbr_f[sm.start[lo] + (e - sm.off[lo])]) & 0x3FFFFFFFu;
      src[k] = sm.v[lo];
      if constexpr (!kDepthKnown) dd[k] = sm.d[lo];
    }
  }
  // parents and out-degrees together (the out-degree of a vertex this step
  // does not claim is not used, but loading it here takes it off the chain)
  int32_t p[K];
  uint32_t od[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    p[k] = ok[k] ? parents[u[k]] : 0;
    od[k] = ok[k] ? __ldg(&b.out_degree[u[k]]) : 0u;
  }
  bool won[K];
#pragma unroll
  for (int k = 0; k < K; k++) won[k] = ok[k] && p[k] < 0 && atomicCAS(&parents[u[k]], p[k], (int32_t)src[k]) == p[k];
#pragma unroll
  for (int k = 0; k < K; k++) {
    if (won[k]) {
      distances[u[k]] = dd[k];
      mf += (uint32_t)(-p[k]);
      found++;
      if (bm_w) atomicOr(&bm_w[u[k] >> 5], 1u << (u[k] & 31));
      if constexpr (TS::kHost) {
        if (all_out) ba_push(sm.q_all, u[k]);
      }
      fed += od[k];
      if (od[k]) {
        ba_push(sm.q_list, u[k]);
        mx = max(mx, od[k]);
      }
    }
  }
}

// Top-down, part 2 (lists longer than kExpTile): each CTA takes whole tiles
// of kExpTile edges of the step; the list entries overlapping a tile are
// staged in shared memory and each edge finds its entry by binary search
// there.  A vertex is claimed by CAS on its parent; the winner appends it to
// the next frontier.
template <bool kDepthKnown, class TS>
__device__ void td_expand_phase(const BfsBufs& b, const uint32_t* list, uint32_t* next_list, uint32_t n,
                                uint32_t total, int32_t* parents, uint32_t* distances, uint32_t dnext,
                                uint32_t* bm_w, uint32_t* all_out, BfsCtl* ctl, TS& sm,
                                unsigned long long* s_red) {
  const uint32_t ntiles = (total + kExpTile - 1) / kExpTile;
  if (blockIdx.x >= ntiles) return;
  ba_init(sm.q_list);
  if constexpr (TS::kHost) ba_init(sm.q_all);
  uint32_t mf = 0, found = 0, mx = 0;
  unsigned long long fed = 0;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t e0 = t * kExpTile;
    const uint32_t e1 = min(e0 + kExpTile, total);
    const uint32_t i0 = b.tile_i0[t];
    const uint32_t i1 = (t + 1 < ntiles) ? b.tile_i0[t + 1] : n - 1;
    const uint32_t cnt = i1 - i0 + 1;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
      sm.off[k] = b.offs[i0 + k];
      sm.start[k] = b.fstart[i0 + k];
      sm.v[k] = list[i0 + k];
      if constexpr (!kDepthKnown) sm.d[k] = b.fdist[i0 + k];
    }
    __syncthreads();
    expand_edges<kDepthKnown>(b, e0, e1, cnt, parents, distances, dnext, bm_w, all_out, sm, mf, found, fed, mx);
    // at most kExpTile discoveries per tile: flush every tile
    ba_flush(sm.q_list, next_list, &ctl->lnext);
    if constexpr (TS::kHost) {
      if (all_out) ba_flush(sm.q_all, all_out, &ctl->all_count);
    }
  }
  td_publish(ctl, mf, found, fed, mx, s_red);
}

// A top-down step over a list of at most kExpTile entries: every CTA loads
// the whole list and scans its out-degrees itself (no cross-CTA scan, so the
// step needs one grid barrier), then expands its share of the edge tiles.
__device__ void td_small_phase(const BfsBufs& b, const uint32_t* list, uint32_t* next_list, uint32_t n,
                               int32_t* parents, uint32_t* distances, uint32_t dnext, uint32_t* bm_w, BfsCtl* ctl,
                               TdSmem& sm, unsigned long long* s_red) {
  constexpr int K = kExpTile / kExpT;
  uint32_t deg[K], sum = 0;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const uint32_t i = threadIdx.x * K + k;
    deg[k] = 0;
    if (i < n) {
      const uint32_t v = list[i];
      const uint2 r = __ldg(&b.rows_f[v]);
      sm.v[i] = v;
      sm.start[i] = r.x;
      deg[k] = r.y;
      sum += r.y;
    }
  }
  uint32_t total = 0;
  uint32_t o = scan_block_excl(sum, sm.w, &total);
#pragma unroll
  for (int k = 0; k < K; k++) {
    const uint32_t i = threadIdx.x * K + k;
    if (i < n) {
      sm.off[i] = o;
      o += deg[k];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->total_edges = total;
  __syncthreads();
  const uint32_t ntiles = (total + kExpTile - 1) / kExpTile;
  if (blockIdx.x >= ntiles) return;
  ba_init(sm.q_list);
  uint32_t mf = 0, found = 0, mx = 0;
  unsigned long long fed = 0;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t e0 = t * kExpTile;
    const uint32_t e1 = min(e0 + kExpTile, total);
    expand_edges<true>(b, e0, e1, n, parents, distances, dnext, bm_w, nullptr, sm, mf, found, fed, mx);
    ba_flush(sm.q_list, next_list, &ctl->lnext);
  }
  td_publish(ctl, mf, found, fed, mx, s_red);
}

// A top-down step over a list of kExpTile < n <= kMidList entries, in one
// phase as well: every CTA that has an edge tile (tile count from the
// frontier's out-edge total, known from the previous step) reads the whole
// list's out-degrees (kMidList / kExpT per thread, kept in registers) and
// scans them; then, per tile, the entries overlapping the tile are staged
// (a contiguous index range: the entry holding the tile's first edge and
// the one holding its last) and expanded as in a two-phase step.  A scan
// total that disagrees with the expected one sets ERR_STATE.
constexpr uint32_t kMidList = 4096;
__device__ void td_mid_phase(const BfsBufs& b, const uint32_t* list, uint32_t* next_list, uint32_t n,
                             unsigned long long expect_total, int32_t* parents, uint32_t* distances, uint32_t dnext,
                             uint32_t* bm_w, BfsCtl* ctl, uint32_t* err, TdSmem& sm, unsigned long long* s_red) {
  constexpr int K = kMidList / kExpT;
  const uint32_t ntiles = (uint32_t)((expect_total + kExpTile - 1) / kExpTile);
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->total_edges = (uint32_t)expect_total;
  if (blockIdx.x >= ntiles) return;
  uint32_t deg[K], sum = 0;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const uint32_t i = threadIdx.x * K + k;
    deg[k] = i < n ? __ldg(&b.rows_f[list[i]]).y : 0u;
    sum += deg[k];
  }
  uint32_t total = 0;
  const uint32_t excl = scan_block_excl(sum, sm.w, &total);
  if (total != expect_total) {
    if (threadIdx.x == 0) atomicExch(err, (uint32_t)ERR_STATE);
    return;
  }
  ba_init(sm.q_list);
  uint32_t mf = 0, found = 0, mx = 0;
  unsigned long long fed = 0;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t e0 = t * kExpTile;
    const uint32_t e1 = min(e0 + kExpTile, total);
    uint32_t o = excl;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const uint32_t i = threadIdx.x * K + k;
      if (deg[k]) {
        if (o <= e0 && e0 < o + deg[k]) sm.lo = i;
        if (o <= e1 - 1 && e1 - 1 < o + deg[k]) sm.hi = i;
      }
      o += deg[k];
    }
    __syncthreads();
    const uint32_t lo = sm.lo, cnt = sm.hi - lo + 1;
    o = excl;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const uint32_t i = threadIdx.x * K + k;
      if (deg[k] && i >= lo && i < lo + cnt) {
        const uint32_t v = list[i];
        sm.v[i - lo] = v;
        sm.start[i - lo] = __ldg(&b.rows_f[v]).x;
        sm.off[i - lo] = o;
      }
      o += deg[k];
    }
    __syncthreads();
    expand_edges<true>(b, e0, e1, cnt, parents, distances, dnext, bm_w, nullptr, sm, mf, found, fed, mx);
    // at most kExpTile discoveries per tile: flush every tile (its barriers
    // also end this tile's use of the staged entries)
    ba_flush(sm.q_list, next_list, &ctl->lnext);
  }
  td_publish(ctl, mf, found, fed, mx, s_red);
}

// A top-down step over a list longer than kMidList whose entries all have at
// most kFlatMaxDeg out-edges (the largest out-degree on the list is counted
// by the step that made it): one phase, no scan.  Every thread takes one
// list entry per pass and expands its out-edges four at a time (neighbour
// ids, then parents and out-degrees, then the claiming CASes).  This is the
// usual shape of the top-down steps after a bottom-up phase: thousands of
// low-degree vertices and few edges, where a two-phase step pays a whole
// scan phase and its grid barrier for a handful of edge tiles.
__device__ void td_flat_phase(const BfsBufs& b, const uint32_t* list, uint32_t* next_list, uint32_t n,
                              unsigned long long total, int32_t* parents, uint32_t* distances, uint32_t dnext,
                              uint32_t* bm_w, BfsCtl* ctl, uint32_t* err, BlockAppend<kFlatCap>& q,
                              unsigned long long* s_red) {
  constexpr int K = 4;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->total_edges = (uint32_t)total;
  if ((uint64_t)blockIdx.x * blockDim.x >= n) return;  // CTA-uniform: no entry for this CTA
  ba_init(q);
  uint32_t mf = 0, found = 0, mx = 0;
  unsigned long long fed = 0;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const uint32_t i = base + threadIdx.x;
    uint32_t src = 0;
    uint2 r = make_uint2(0u, 0u);
    if (i < n) {
      src = list[i];
      r = __ldg(&b.rows_f[src]);
      if (r.y > kFlatMaxDeg) {  // the list's maximum said otherwise: refuse rather than overflow
        atomicExch(err, (uint32_t)ERR_STATE);
        r.y = 0;
      }
    }
    for (uint32_t j0 = 0; j0 < r.y; j0 += K) {
      uint32_t u[K], od[K];
      int32_t pp[K];
      bool ok[K];
#pragma unroll
      for (int k = 0; k < K; k++) {
        ok[k] = j0 + k < r.y;
        u[k] = ok[k] ? (__ldg(&b.nbr_f[r.x + j0 + k]) & 0x3FFFFFFFu) : 0u;
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        pp[k] = ok[k] ? parents[u[k]] : 0;
        od[k] = ok[k] ? __ldg(&b.out_degree[u[k]]) : 0u;
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (ok[k] && pp[k] < 0 && atomicCAS(&parents[u[k]], pp[k], (int32_t)src) == pp[k]) {
          distances[u[k]] = dnext;
          mf += (uint32_t)(-pp[k]);
          found++;
          atomicOr(&bm_w[u[k] >> 5], 1u << (u[k] & 31));
          fed += od[k];
          if (od[k]) {
            ba_push(q, u[k]);
            mx = max(mx, od[k]);
          }
        }
      }
    }
    // at most blockDim.x * kFlatMaxDeg claims per pass: flush every pass
    ba_flush(q, next_list, &ctl->lnext);
  }
  td_publish(ctl, mf, found, fed, mx, s_red);
}

// ------------------------------------------------------------ bottom-up ----

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kBuV = kBuRound / kSearchT;  // candidates per thread per round
constexpr uint32_t kFirst = 6;             // dense step: in-edges probed per candidate before deferral
constexpr uint32_t kRecN = 4;              // list step: in-neighbours held in a candidate record

// Long in-edge rows of a round (deferred by either kind of step): a group of
// 4 lanes per row, 8 in-edges per step (two per lane, both loads in flight,
// then all frontier probes), 64 groups per CTA; the first hit in CSR order
// wins.  Entry h is the candidate sm.hv[h]: the index of its record in rec_a
// (list step), whose vertex, in-row and out-degree are read back from the
// record, or a vertex (dense step), whose in-row is read back from rows_i;
// the row is scanned from past the in-edges the step already probed.  Rows
// without a hit go to the unvisited list (as the entry).
constexpr uint32_t kLongLanes = 4;
constexpr uint32_t kLongLoads = 2;
constexpr uint32_t kLongStep = kLongLanes * kLongLoads;
__device__ __forceinline__ void bu_long_rows(const BfsBufs& b, const uint32_t* bm_cur, uint32_t* bm_next,
                                             const uint4* rec_a, int32_t* parents, uint32_t* distances,
                                             uint32_t dnext, BuSmem& sm, uint32_t& nf, uint32_t& edges,
                                             uint32_t& mx, unsigned long long& fed) {
  const uint32_t lane = lane_id();
  const uint32_t nh = sm.nheavy;
  const uint32_t gl = threadIdx.x & (kLongLanes - 1);
  const uint32_t gshift = lane & ~(kLongLanes - 1);
  const uint32_t gmask = ((1u << kLongLanes) - 1u) << gshift;
  for (uint32_t h = threadIdx.x / kLongLanes; h < nh; h += kSearchT / kLongLanes) {
    const uint32_t hv = sm.hv[h];
    uint32_t j0, end, v, od;
    if (rec_a) {
      const uint4 r = rec_a[hv];
      v = r.x;
      od = r.w;
      j0 = r.y + kRecN;
      end = r.y + r.z;
    } else {
      const uint2 rr = __ldg(&b.rows_i[hv]);
      v = hv;
      od = 0;  // read on a hit
      j0 = rr.x + kFirst;
      end = rr.x + rr.y;
    }
    bool hit_row = false;
    for (uint32_t j = j0; j < end; j += kLongStep) {
      uint32_t x[kLongLoads];
#pragma unroll
      for (uint32_t q = 0; q < kLongLoads; q++) {
        const uint32_t jq = j + q * kLongLanes + gl;
        x[q] = jq < end ? (__ldg(&b.nbr_i[jq]) & 0x3FFFFFFFu) : kInvalid;
      }
      bool bit[kLongLoads];
#pragma unroll
      for (uint32_t q = 0; q < kLongLoads; q++) bit[q] = x[q] != kInvalid && ((bm_cur[x[q] >> 5] >> (x[q] & 31)) & 1u);
      // bit (q * kLongLanes + group lane) of m <-> in-edge j + that index
      uint32_t m = 0;
#pragma unroll
      for (uint32_t q = 0; q < kLongLoads; q++)
        m |= ((__ballot_sync(gmask, bit[q]) >> gshift) & ((1u << kLongLanes) - 1u)) << (q * kLongLanes);
      if (m) {
        const uint32_t first = (uint32_t)__ffs(m) - 1;
        if (gl == (first & (kLongLanes - 1))) {
          uint32_t u = x[0];
#pragma unroll
          for (uint32_t q = 1; q < kLongLoads; q++)
            if (first / kLongLanes == q) u = x[q];
          if (!rec_a) od = __ldg(&b.out_degree[v]);
          parents[v] = (int32_t)u;
          distances[v] = dnext;
          atomicOr(&bm_next[v >> 5], 1u << (v & 31));
          nf++;
          edges += j + first + 1 - j0;
          fed += od;
          if (od) {
            bu_push_list(sm, v);
            mx = max(mx, od);
          }
        }
        hit_row = true;
        break;
      }
    }
    if (!hit_row && gl == 0) {
      edges += end - j0;
      bu_push_ul(sm, hv);
    }
  }
}

// Step totals: nf and the edges examined, packed, the discoveries' out-edges
// and the largest out-degree put on the list.
__device__ __forceinline__ void bu_publish(BfsCtl* ctl, uint32_t nf, uint32_t edges, unsigned long long fed,
                                           uint32_t mx, unsigned long long* s_red) {
  unsigned long long a = (unsigned long long)nf | ((unsigned long long)edges << 32), c = fed;
  block_sum2_max(a, c, mx, s_red);
  if (threadIdx.x == 0) {
    if ((uint32_t)a) atomicAdd(&ctl->nf, (uint32_t)a);
    if (a >> 32) atomicAdd(&ctl->edges, a >> 32);
    if (c) atomicAdd(&ctl->fedges, c);
    if (mx) atomicMax(&ctl->maxdeg, mx);
  }
}

// One bottom-up step over every vertex (the dense-probe mode, and a graph
// without in-edges).  Each thread takes kBuV vertices at once: parents, then
// in-edge rows, then the first kFirst in-neighbours of each and their
// frontier bits, all issued together; longer rows without a hit yet go to
// the round's long-row list.  A warp's ballot stores a whole word of bm_next;
// discoveries with out-edges get a slot in list_next.  No unvisited list is
// written: the dense mode walks every vertex in every step, and in a graph
// without in-edges nothing is ever found bottom-up.  bm_clear is zeroed on
// the way.
__device__ void bu_dense_phase(const BfsBufs& b, const uint32_t* bm_cur, uint32_t* bm_next, uint32_t* bm_clear,
                               uint32_t* list_next, int32_t* parents, uint32_t* distances, uint32_t dnext,
                               BfsCtl* ctl, BuSmem& sm, unsigned long long* s_red) {
  grid_clear(bm_clear, nullptr, b.words);
  if (threadIdx.x == 0) {
    sm.nlist = 0;
    sm.nul = 0;
    sm.nheavy = 0;
  }
  __syncthreads();
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t count = b.V;
  uint32_t nf = 0, edges = 0, mx = 0;
  unsigned long long fed = 0;
  // each CTA takes one contiguous, equal range of vertices (a multiple of
  // 32, so the ballot words never straddle two CTAs)
  const uint32_t per = ((count + gridDim.x - 1) / gridDim.x + 31u) & ~31u;
  const uint32_t lo = min(count, blockIdx.x * per), hi = min(count, lo + per);
  for (uint32_t rbase = lo; rbase < hi; rbase += kBuRound) {
    uint32_t v[kBuV];
#pragma unroll
    for (int k = 0; k < kBuV; k++) {
      const uint32_t idx = rbase + k * kSearchT + threadIdx.x;
      v[k] = idx < hi ? idx : kInvalid;
    }
    // parent and in-row together (a visited candidate's row is not used)
    int32_t pv[kBuV];
    uint2 row[kBuV];
#pragma unroll
    for (int k = 0; k < kBuV; k++) {
      pv[k] = v[k] != kInvalid ? parents[v[k]] : 0;
      row[k] = v[k] != kInvalid ? __ldg(&b.rows_i[v[k]]) : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int k = 0; k < kBuV; k++)
      if (pv[k] >= 0) row[k] = make_uint2(0u, 0u);
    uint32_t u[kBuV][kFirst];
#pragma unroll
    for (int k = 0; k < kBuV; k++)
#pragma unroll
      for (uint32_t m = 0; m < kFirst; m++)
        u[k][m] = m < row[k].y ? (__ldg(&b.nbr_i[row[k].x + m]) & 0x3FFFFFFFu) : kInvalid;
    uint32_t hit[kBuV], par[kBuV];
#pragma unroll
    for (int k = 0; k < kBuV; k++) {
      hit[k] = kFirst;
      par[k] = 0;
#pragma unroll
      for (int m = (int)kFirst - 1; m >= 0; m--) {
        const uint32_t x = u[k][m];
        if (x != kInvalid && ((bm_cur[x >> 5] >> (x & 31)) & 1u)) {
          hit[k] = (uint32_t)m;
          par[k] = x;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kBuV; k++) {
      bool found = false;
      if (row[k].y) {
        if (hit[k] < kFirst) {
          parents[v[k]] = (int32_t)par[k];
          distances[v[k]] = dnext;
          found = true;
          nf++;
          edges += hit[k] + 1;
          const uint32_t od = __ldg(&b.out_degree[v[k]]);
          fed += od;
          if (od) {
            bu_push_list(sm, v[k]);
            mx = max(mx, od);
          }
        } else if (row[k].y > kFirst) {
          edges += kFirst;
          const uint32_t h = warp_atomic_inc(&sm.nheavy);
          sm.hv[h] = v[k];
        } else {
          edges += row[k].y;
        }
      }
      const uint32_t word = __ballot_sync(0xffffffffu, found);
      const uint32_t base = rbase + k * kSearchT + warp * 32;
      if (lane == 0 && base < hi) bm_next[base >> 5] = word;
    }
    __syncthreads();
    bu_long_rows(b, bm_cur, bm_next, nullptr, parents, distances, dnext, sm, nf, edges, mx, fed);
    __syncthreads();
    if (threadIdx.x == 0) {
      sm.nheavy = 0;
      sm.nul = 0;  // long rows without a hit: no unvisited list in this mode
    }
    bu_flush(sm, list_next, &ctl->lnext, nullptr, nullptr, nullptr, nullptr, &ctl->ul_size);
  }
  bu_publish(ctl, nf, edges, fed, mx, s_red);
}

// A record's k-th in-neighbour.
__device__ __forceinline__ uint32_t rec_nbr(const uint4& q, int m) {
  return m == 0 ? q.x : (m == 1 ? q.y : (m == 2 ? q.z : q.w));
}

// One bottom-up step over a list of candidate records: the first such step
// of a search walks the graph's vertices with in-edges (a vertex without one
// can never be found bottom-up), later ones the unvisited list the step
// before wrote.  A record is two 16-byte words in two arrays, A = {vertex,
// first in-edge, in-degree, out-degree} and B = the row's first kRecN
// in-neighbours (kInvalid past its end), so a warp reads 32 candidates with
// two contiguous 512-byte loads; the frontier bits of the first in-neighbours
// follow directly, instead of list entry, row, neighbour ids and bits as four
// dependent, scattered loads.  Each CTA takes one contiguous, equal range of
// records; a round is kBuSub passes of kBuV records per thread (loads, probes,
// appends), then one long-row phase and one flush for all of them.  The parents are read only
// when the list may hold visited vertices (check_parents: the first list, or
// a list that top-down steps have run after); a list written by the step just
// before holds unvisited vertices only.  Rows longer than kRecN without a hit
// go to the round's long-row list.  Unfound candidates' records are copied
// into out_a / out_b, the next step's list.  bm_clear is zeroed on the way.
__device__ void bu_rec_phase(const BfsBufs& b, const uint32_t* bm_cur, uint32_t* bm_next, uint32_t* bm_clear,
                             const uint4* in_a, const uint4* in_b, uint32_t count, bool check_parents,
                             uint4* out_a, uint4* out_b, uint32_t* list_next, int32_t* parents,
                             uint32_t* distances, uint32_t dnext, BfsCtl* ctl, BuSmem& sm,
                             unsigned long long* s_red) {
  grid_clear(bm_clear, nullptr, b.words);
  if (threadIdx.x == 0) {
    sm.nlist = 0;
    sm.nul = 0;
    sm.nheavy = 0;
  }
  __syncthreads();
  uint32_t nf = 0, edges = 0, mx = 0;
  unsigned long long fed = 0;
  const uint32_t per = ((count + gridDim.x - 1) / gridDim.x + 31u) & ~31u;
  const uint32_t lo = min(count, blockIdx.x * per), hi = min(count, lo + per);
  for (uint32_t rbase0 = lo; rbase0 < hi; rbase0 += kBuCap) {
#pragma unroll 1
    for (uint32_t sub = 0; sub < kBuSub; sub++) {
      const uint32_t rbase = rbase0 + sub * kBuRound;
      uint4 ra[kBuV], rb[kBuV];
#pragma unroll
      for (int k = 0; k < kBuV; k++) {
        const uint32_t idx = rbase + k * kSearchT + threadIdx.x;
        if (idx < hi) {
          ra[k] = in_a[idx];
          rb[k] = in_b[idx];
        } else {
          ra[k] = make_uint4(0u, 0u, 0u, 0u);  // in-degree 0: no candidate
          rb[k] = make_uint4(kInvalid, kInvalid, kInvalid, kInvalid);
        }
      }
      int32_t pv[kBuV];
#pragma unroll
      for (int k = 0; k < kBuV; k++) pv[k] = (check_parents && ra[k].z) ? parents[ra[k].x] : -1;
      uint32_t hit[kBuV], par[kBuV];
#pragma unroll
      for (int k = 0; k < kBuV; k++) {
        hit[k] = kRecN;
        par[k] = 0;
#pragma unroll
        for (int m = (int)kRecN - 1; m >= 0; m--) {
          const uint32_t x = rec_nbr(rb[k], m);
          if (x != kInvalid && ((bm_cur[x >> 5] >> (x & 31)) & 1u)) {
            hit[k] = (uint32_t)m;
            par[k] = x;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kBuV; k++) {
        const uint32_t v = ra[k].x, deg = ra[k].z, od = ra[k].w;
        if (deg == 0 || pv[k] >= 0) continue;  // no candidate, or visited
        if (hit[k] < kRecN) {
          parents[v] = (int32_t)par[k];
          distances[v] = dnext;
          nf++;
          edges += hit[k] + 1;
          atomicOr(&bm_next[v >> 5], 1u << (v & 31));
          fed += od;
          if (od) {
            bu_push_list(sm, v);
            mx = max(mx, od);
          }
        } else if (deg > kRecN) {
          edges += kRecN;
          const uint32_t h = warp_atomic_inc(&sm.nheavy);
          sm.hv[h] = rbase + k * kSearchT + threadIdx.x;
        } else {
          edges += deg;
          bu_push_ul(sm, rbase + k * kSearchT + threadIdx.x);
        }
      }
    }
    __syncthreads();
    bu_long_rows(b, bm_cur, bm_next, in_a, parents, distances, dnext, sm, nf, edges, mx, fed);
    // the flush's first barrier ends the long rows (it also clears their count)
    bu_flush(sm, list_next, &ctl->lnext, in_a, in_b, out_a, out_b, &ctl->ul_size);
  }
  bu_publish(ctl, nf, edges, fed, mx, s_red);
}

// ---- bottom-up of the host-state step (depth read from the parent) --------

struct BuHostSmem {
  BlockAppend<2 * kBuRound> q;
};

// Scan v's in-edges in CSR order for the first in-neighbour in the frontier.
__device__ __forceinline__ bool bu_probe_host(const BfsBufs& b, const uint32_t* bm_cur, uint32_t v, int32_t* parents,
                                              uint32_t* distances, uint32_t& edges) {
  const uint2 row = __ldg(&b.rows_i[v]);
  for (uint32_t j = row.x; j < row.x + row.y; j++) {
    const uint32_t u = __ldg(&b.nbr_i[j]) & 0x3FFFFFFFu;
    if ((bm_cur[u >> 5] >> (u & 31)) & 1u) {
      parents[v] = (int32_t)u;
      distances[v] = distances[u] + 1;
      edges += j + 1 - row.x;
      return true;
    }
  }
  edges += row.y;
  return false;
}

// Every vertex; a warp's ballot is OR-ed into one word of bm_next.
__device__ void bu_host_phase(const BfsBufs& b, const uint32_t* bm_cur, uint32_t* bm_next, uint32_t* ul_next,
                              int32_t* parents, uint32_t* distances, BfsCtl* ctl, BuHostSmem& sm,
                              unsigned long long* s_red) {
  ba_init(sm.q);
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t nf = 0, edges = 0;
  for (uint32_t rbase = blockIdx.x * kBuRound; rbase < b.V; rbase += gridDim.x * kBuRound) {
#pragma unroll
    for (uint32_t k = 0; k < kBuRound / kSearchT; k++) {
      const uint32_t base = rbase + k * kSearchT + warp * 32;
      const uint32_t v = base + lane;
      bool found = false, unvisited = false;
      if (v < b.V && parents[v] < 0) {
        found = bu_probe_host(b, bm_cur, v, parents, distances, edges);
        unvisited = !found;
      }
      const uint32_t word = __ballot_sync(0xffffffffu, found);
      if (lane == 0 && base < b.V) bm_next[base >> 5] |= word;
      nf += found;
      if (unvisited) ba_push(sm.q, v);
    }
    if (ba_size(sm.q) > kBuRound) ba_flush(sm.q, ul_next, &ctl->ul_size);
  }
  ba_flush(sm.q, ul_next, &ctl->ul_size);
  block_add_total<uint32_t>(&ctl->nf, nf, reinterpret_cast<uint32_t*>(s_red));
  block_add_total<unsigned long long>(&ctl->edges, (unsigned long long)edges, s_red);
}

// ------------------------------------------------------------ control ------

constexpr uint32_t kActDone = 0, kActTD = 1, kActBU = 2;

// Counters of a finished phase, read past any cached copy.
__device__ __forceinline__ void load_ctl(const BfsCtl* p, BfsCtl& out) {
  const volatile BfsCtl* v = p;
  out.qnext = v->qnext;
  out.lnext = v->lnext;
  out.mf = v->mf;
  out.nf = v->nf;
  out.ul_size = v->ul_size;
  out.total_edges = v->total_edges;
  out.edges = v->edges;
  out.fedges = v->fedges;
  out.maxdeg = v->maxdeg;
}

__device__ __forceinline__ void zero_ctl(BfsCtl* p) {
  BfsCtl z = {};
  *p = z;
}

// Before a step: stop on an empty queue, else pick the direction with the
// reference's rule (BFS.c:520-560).
__device__ uint32_t ctrl_decide(BfsCtrl& c, bool policy_bu) {
  if (c.overflow) return kActDone;
  if (c.mode == BFS_LEARNED) {
    // the learned switch: every step's direction from the policy (any order
    // of directions is valid: both kinds of step keep the frontier as a list
    // and as a bitmap); the loop ends on an empty frontier
    if (c.qcount == 0) return kActDone;
    c.frontier = c.qcount;
    if (policy_bu) {
      c.in_bu = 1;
      c.nf = c.qcount;
      c.nf_prev = c.nf;
      return kActBU;
    }
    c.in_bu = 0;
    c.mu -= min(c.mf, c.mu);
    c.epoch++;
    return kActTD;
  }
  if (!c.in_bu && c.qcount == 0) return kActDone;
  if (c.in_bu) {
    c.frontier = c.nf;
    c.nf_prev = c.nf;
    return kActBU;
  }
  const bool bu = (c.mode == BFS_PULL) || (c.mode == BFS_PULL_DENSE) || (c.mode == BFS_DO && c.mf > c.mu / kAlpha);
  c.frontier = c.qcount;
  if (bu) {
    c.in_bu = 1;
    c.nf = c.bu_entry_frontier ? c.qcount : 0u;
    c.nf_prev = c.nf;
    return kActBU;
  }
  c.mu -= c.mf;
  c.epoch++;
  return kActTD;
}

__device__ void ctrl_level(BfsCtrl& c, BfsDevState* st, bool leader, uint32_t dir, uint32_t disc,
                           unsigned long long edges, unsigned long long t0) {
  if (leader && c.nlevels < (uint32_t)kMaxTrace) {
    BfsLevel L;
    L.direction = dir;
    L.discovered = disc;
    L.frontier = c.frontier;
    L.mf = c.mf;
    L.mu = c.mu;
    L.edges = edges;
    L.ms = (float)((double)(global_ns() - t0) * 1e-6);
    st->trace[c.nlevels] = L;
  }
  c.nlevels++;
  c.iteration++;
  c.depth++;
  c.processed += disc;
  c.edges_examined += edges;
  c.qcount_prev = c.frontier;
  if (c.iteration > c.max_steps) c.overflow = 1;
}

// The learned switch's inputs, from the reference's switch state before a
// step (nf, nf_prev, mf, mu, n: BFS.c:510-516) plus the bottom-up step's
// candidate count; counts enter as L(x) = log2(1 + x).
__device__ __forceinline__ void bfs_features(const BfsCtrl& c, uint32_t E, float* f) {
  const unsigned long long left = (unsigned long long)E > c.edges_visited ? (unsigned long long)E - c.edges_visited : 0ull;
  const uint32_t cand = c.ul_valid ? c.ul_size : c.n;
  const float lq = log2f(1.0f + (float)c.qcount);
  f[0] = lq;                                                         // frontier vertices
  f[1] = log2f(1.0f + (float)c.fedges);                              // frontier out-edges
  f[2] = log2f(1.0f + (float)left);                                  // unexplored out-edges
  f[3] = log2f(1.0f + (float)cand);                                  // bottom-up candidates (list or all)
  f[4] = log2f(1.0f + (float)c.n);                                   // vertices
  f[5] = lq - log2f(1.0f + (float)c.qcount_prev);                    // frontier growth
  f[6] = (float)c.processed / (float)max(c.n, 1u);                   // visited fraction
  f[7] = c.ul_valid ? 1.0f : 0.0f;                                   // a bottom-up step would walk the unvisited list
}

// Policy network layout on the device (bf16): W1[64][8], b1[64], W2T[64][64]
// (transposed: W2T[j][i] = W2[i][j]), b2[64], w3[64], b3.
constexpr int kPolIn = kFeat, kPolH = 64;
constexpr int kPolW1 = 0, kPolB1 = kPolH * kPolIn, kPolW2T = kPolB1 + kPolH, kPolB2 = kPolW2T + kPolH * kPolH,
              kPolW3 = kPolB2 + kPolH, kPolB3 = kPolW3 + kPolH, kPolN = kPolB3 + 1;
static_assert(kPolN == kPolMlpN, "policy packing");
constexpr size_t kPolSmem = ((size_t)kPolN * 2 + 15) / 16 * 16;  // bytes staged (the tail starts there)
static_assert(kPolSmem == kPolTailOff, "the staged network ends where the tail begins");
static_assert(sizeof(BfsSmem) >= kPolSmem, "the phase scratch holds the policy network");

// Policy output of a warp (bf16 weights in shared memory, fp32 sums): lane
// l owns hidden units l and l + 32; every lane returns the output.
__device__ __forceinline__ float policy_logit(const __nv_bfloat16* P, const float* f, uint32_t lane) {
  float ha = __bfloat162float(P[kPolB1 + lane]), hb = __bfloat162float(P[kPolB1 + lane + 32]);
#pragma unroll
  for (int j = 0; j < kPolIn; j++) {
    ha = fmaf(__bfloat162float(P[kPolW1 + lane * kPolIn + j]), f[j], ha);
    hb = fmaf(__bfloat162float(P[kPolW1 + (lane + 32) * kPolIn + j]), f[j], hb);
  }
  ha = fmaxf(ha, 0.f);
  hb = fmaxf(hb, 0.f);
  float sa = __bfloat162float(P[kPolB2 + lane]), sb = __bfloat162float(P[kPolB2 + lane + 32]);
#pragma unroll 8
  for (int j = 0; j < kPolH; j++) {
    const float hj = __shfl_sync(0xffffffffu, j < 32 ? ha : hb, j & 31);
    sa = fmaf(__bfloat162float(P[kPolW2T + j * kPolH + lane]), hj, sa);
    sb = fmaf(__bfloat162float(P[kPolW2T + j * kPolH + lane + 32]), hj, sb);
  }
  float y = __bfloat162float(P[kPolW3 + lane]) * fmaxf(sa, 0.f) +
            __bfloat162float(P[kPolW3 + lane + 32]) * fmaxf(sb, 0.f);
#pragma unroll
  for (int o = 16; o; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
  return y + __bfloat162float(P[kPolB3]);
}

__device__ void ctrl_finish_td(BfsCtrl& c, uint32_t total_edges, const BfsCtl& k, BfsDevState* st, bool leader,
                               unsigned long long t0) {
  c.mf = k.mf;
  c.qcount = k.qnext;
  c.lsize = k.lnext;
  c.lmax = k.maxdeg;
  c.fedges = k.fedges;
  c.edges_visited += k.fedges;
  c.par_l ^= 1u;
  const uint32_t r = c.bm_r;
  c.bm_r = c.bm_w;
  c.bm_w = r;
  c.td_steps++;
  c.ul_fresh = 0;  // the unvisited list may now hold vertices this step visited
  ctrl_level(c, st, leader, 0, c.qcount, total_edges, t0);
}

// After a bottom-up step (read bm_r, wrote bm_w, cleared bm_c): rotate, and
// decide whether the bottom-up phase continues (BFS.c:583-585).  The step
// also listed its discoveries, so the queue is ready when the phase ends
// (mf = 1 then, BFS.c:588).
__device__ void ctrl_finish_bu(BfsCtrl& c, const BfsCtl& k, BfsDevState* st, bool leader, unsigned long long t0) {
  c.nf = k.nf;
  c.ul_size = k.ul_size;
  c.ul_valid = c.mode == BFS_PULL_DENSE ? 0u : 1u;  // that mode walks every vertex in every step
  c.ul_cand0 = 0;
  c.ul_fresh = 1;
  c.par_ul ^= 1u;
  c.qcount = k.nf;
  c.lsize = k.lnext;
  c.lmax = k.maxdeg;
  c.fedges = k.fedges;
  c.edges_visited += k.fedges;
  c.par_l ^= 1u;
  const uint32_t r = c.bm_r;
  c.bm_r = c.bm_w;
  c.bm_w = c.bm_c;
  c.bm_c = r;
  c.bu_steps++;
  ctrl_level(c, st, leader, 1, c.nf, k.edges, t0);
  if (c.mode == BFS_LEARNED) return;  // the policy picks every step
  const bool cont = (c.mode == BFS_PULL || c.mode == BFS_PULL_DENSE) ? (c.nf > 0)
                                                                    : ((c.nf > c.nf_prev) || (c.nf > c.n / kBeta));
  if (!cont) {
    c.in_bu = 0;
    c.mf = 1;
  }
}

// ------------------------------------------------------------ kernels ------

// parents[v] = -out_degree[v] (or -1), distances[v] = 0 (BFS.c:58-74); the
// root gets itself as parent; bitmap 0 holds the root, the others are clear;
// the state starts as the reference's loop does (mu = E, mf =
// out_degree(root), queue = {root}).
__global__ void __launch_bounds__(256) bfsk_init(BfsBufs b, BfsDevState* st, uint32_t root, int32_t* parents,
                                                 uint32_t* distances, uint32_t mode, uint32_t bu_entry_frontier,
                                                 uint32_t E, uint32_t epoch, uint32_t n_cand0) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < b.V; v += stride) {
    const uint32_t d = b.out_degree[v];
    parents[v] = (v == root) ? (int32_t)root : (d ? -(int32_t)d : -1);
    distances[v] = 0;
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.words; i += stride) {
    b.bm[0][i] = (i == (root >> 5)) ? (1u << (root & 31)) : 0u;
    b.bm[1][i] = 0;
    b.bm[2][i] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t d = b.out_degree[root];
    BfsCtrl c = {};
    c.mode = mode;
    c.bu_entry_frontier = bu_entry_frontier;
    c.n = b.V;
    c.max_steps = b.V + 8;
    c.mu = E;
    c.mf = d;
    c.qcount = 1;
    c.lsize = d ? 1u : 0u;
    c.bm_r = 0;
    c.bm_w = 1;
    c.bm_c = 2;
    c.iteration = 1;
    c.processed = 1;
    c.epoch = epoch;
    c.fedges = d;
    c.edges_visited = d;
    c.lmax = d;
    // the first bottom-up step walks the cached list of vertices with
    // in-edges (a vertex without any can never be found bottom-up); the
    // dense-probe mode walks every vertex in every step
    if (n_cand0 && mode != BFS_PULL_DENSE) {
      c.ul_valid = 1;
      c.ul_size = n_cand0;
      c.ul_cand0 = 1;
    }
    st->c = c;
    st->parents = parents;
    st->distances = distances;
    st->err = 0;
    st->bar = 0;
    zero_ctl(&st->ctl[0]);
    zero_ctl(&st->ctl[1]);
    zero_ctl(&st->ctl[2]);
    b.list[0][0] = root;
  }
}

// More roots after bfsk_init's first one (a search over a disjoint union of
// graphs, one root each): each gets itself as parent and its frontier bit,
// joins the queue (and the expansion list when it has out-edges); mf sums
// their out-degrees.  Duplicates are skipped.  One thread, after bfsk_init.
__global__ void bfsk_set_roots(BfsBufs b, BfsDevState* st, const uint32_t* __restrict__ roots, uint32_t n) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int32_t* parents = st->parents;
  BfsCtrl c = st->c;
  for (uint32_t i = 1; i < n; i++) {
    const uint32_t r = roots[i];
    if (parents[r] == (int32_t)r) continue;
    parents[r] = (int32_t)r;
    b.bm[0][r >> 5] |= 1u << (r & 31);
    const uint32_t d = b.out_degree[r];
    c.lmax = max(c.lmax, d);
    c.qcount++;
    c.processed++;
    c.mf += d;
    c.fedges += d;
    c.edges_visited += d;
    if (d) b.list[0][c.lsize++] = r;
  }
  st->c = c;
}

// The whole search: all CTAs co-resident (cooperative launch), one grid
// barrier after every phase.  Phase p counts into ctl[p % 3]; CTA 0 clears
// ctl[(p + 1) % 3] when phase p starts (its last reader finished two
// barriers earlier).  A top-down step is one phase when its list has at most
// kExpTile entries, else two (scan, expand); a bottom-up step is one phase.
__global__ void __launch_bounds__(kSearchT, 4) bfsk_search(BfsBufs b, BfsDevState* st) {
  __shared__ __align__(16) BfsSmem sm;
  __shared__ BfsCtrl S;
  __shared__ unsigned long long s_red[kRedSlots * kSearchT / 32];
  __shared__ uint32_t s_act, s_ok;
  __shared__ unsigned long long s_t0;
  __shared__ float s_tail[kPolTail];
  __shared__ float s_z;
  __shared__ uint32_t s_need;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
  if (threadIdx.x == 0) S = st->c;
  if (b.policy && threadIdx.x < kPolTail) s_tail[threadIdx.x] = b.policy_tail[threadIdx.x];
  __syncthreads();
  int32_t* parents = st->parents;
  uint32_t* distances = st->distances;
  BfsCtl* ctl = st->ctl;
  uint32_t p = 0;
  for (;;) {
    const bool learned = S.mode == BFS_LEARNED;
    if (threadIdx.x < 32) {
      float f[kFeat];
      bfs_features(S, b.E, f);
      if (leader && S.nlevels < (uint32_t)kMaxTrace && !S.overflow)
        for (int i = 0; i < kFeat; i++) st->feat[S.nlevels][i] = f[i];
      bool bu = false, need = false;
      if (learned) {
        // z = prior . f + bias; the network adds at most +-bound, so it is
        // needed only when that can change the sign
        float z = s_tail[kFeat];
#pragma unroll
        for (int i = 0; i < kFeat; i++) z = fmaf(s_tail[i], f[i], z);
        need = fabsf(z) <= s_tail[kFeat + 1];
        bu = z > 0.0f;
        if (threadIdx.x == 0) s_z = z;
      }
      if (threadIdx.x == 0) {
        s_need = need ? 1u : 0u;
        if (!need) {  // decided here: no second barrier
          s_act = ctrl_decide(S, bu);
          s_t0 = global_ns();
        }
      }
    }
    __syncthreads();
    if (s_need) {
      // learned switch near its boundary: stage the network in the phase
      // scratch (no phase is running between steps), warp 0 evaluates it
      const uint4* src = reinterpret_cast<const uint4*>(b.policy);
      uint4* dst = reinterpret_cast<uint4*>(&sm);
      for (uint32_t i = threadIdx.x; i < kPolSmem / 16; i += blockDim.x) dst[i] = __ldg(&src[i]);
      __syncthreads();
      if (threadIdx.x < 32) {
        float f[kFeat];
        bfs_features(S, b.E, f);
        const float bound = s_tail[kFeat + 1];
        const float y = policy_logit(reinterpret_cast<const __nv_bfloat16*>(&sm), f, threadIdx.x);
        if (threadIdx.x == 0) s_z += fminf(fmaxf(y, -bound), bound);
      }
      if (threadIdx.x == 0) {
        s_act = ctrl_decide(S, s_z > 0.0f);
        s_t0 = global_ns();
      }
      __syncthreads();
    }
    const uint32_t act = s_act;
    if (act == kActDone) break;
    const uint32_t dnext = S.depth + 1;
    if (act == kActTD) {
      const uint32_t* list = b.list[S.par_l];
      uint32_t* next = b.list[S.par_l ^ 1u];
      uint32_t* bm_w = b.bm[S.bm_w];
      const uint32_t n = S.lsize;
      grid_clear(b.bm[S.bm_r], b.bm[S.bm_c], b.words);  // a top-down step reads no bitmap
      if (leader) zero_ctl(&ctl[(p + 1) % 3]);
      uint32_t total;
      if (n <= kExpTile) {
        td_small_phase(b, list, next, n, parents, distances, dnext, bm_w, &ctl[p % 3], sm.td, s_red);
        if (!grid_sync(&st->bar, &st->err, &s_ok)) break;
        total = ld_volatile_u32(&ctl[p % 3].total_edges);
      } else if (n <= kMidList) {
        td_mid_phase(b, list, next, n, S.fedges, parents, distances, dnext, bm_w, &ctl[p % 3], &st->err, sm.td,
                     s_red);
        if (!grid_sync(&st->bar, &st->err, &s_ok)) break;
        total = ld_volatile_u32(&ctl[p % 3].total_edges);
      } else if (S.lmax <= kFlatMaxDeg) {
        td_flat_phase(b, list, next, n, S.fedges, parents, distances, dnext, bm_w, &ctl[p % 3], &st->err, sm.flat,
                      s_red);
        if (!grid_sync(&st->bar, &st->err, &s_ok)) break;
        total = ld_volatile_u32(&ctl[p % 3].total_edges);
      } else {
        td_scan_phase<true>(b, list, n, distances, S.epoch, &ctl[p % 3], &st->err, sm.scan);
        if (!grid_sync(&st->bar, &st->err, &s_ok)) break;
        total = ld_volatile_u32(&ctl[p % 3].total_edges);
        p++;
        if (leader) zero_ctl(&ctl[(p + 1) % 3]);
        td_expand_phase<true, TdSmem>(b, list, next, n, total, parents, distances, dnext, bm_w, nullptr, &ctl[p % 3], sm.td,
                              s_red);
        if (!grid_sync(&st->bar, &st->err, &s_ok)) break;
      }
      if (threadIdx.x == 0) {
        BfsCtl k;
        load_ctl(&ctl[p % 3], k);
        ctrl_finish_td(S, total, k, st, blockIdx.x == 0, s_t0);
      }
      p++;
    } else {
      if (leader) zero_ctl(&ctl[(p + 1) % 3]);
      if (!S.ul_valid) {
        bu_dense_phase(b, b.bm[S.bm_r], b.bm[S.bm_w], b.bm[S.bm_c], b.list[S.par_l ^ 1u], parents, distances, dnext,
                       &ctl[p % 3], sm.bu, s_red);
      } else {
        const bool c0 = S.ul_cand0 != 0;
        bu_rec_phase(b, b.bm[S.bm_r], b.bm[S.bm_w], b.bm[S.bm_c], c0 ? b.cand_a : b.ul_a[S.par_ul],
                     c0 ? b.cand_b : b.ul_b[S.par_ul], S.ul_size, c0 || !S.ul_fresh, b.ul_a[S.par_ul ^ 1u],
                     b.ul_b[S.par_ul ^ 1u], b.list[S.par_l ^ 1u], parents, distances, dnext, &ctl[p % 3], sm.bu,
                     s_red);
      }
      if (!grid_sync(&st->bar, &st->err, &s_ok)) break;
      if (threadIdx.x == 0) {
        BfsCtl k;
        load_ctl(&ctl[p % 3], k);
        ctrl_finish_bu(S, k, st, blockIdx.x == 0, s_t0);
      }
      p++;
    }
  }
  if (leader) st->c = S;
}

// ---- kernels of the host-state steps (depth read from the parent) --------

__global__ void __launch_bounds__(kScanT) bfsk_td_scan_host(BfsBufs b, BfsDevState* st, uint32_t n,
                                                           const uint32_t* distances, uint32_t epoch) {
  __shared__ ScanSmem sm;
  td_scan_phase<false>(b, b.list[0], n, distances, epoch, &st->aux, &st->err, sm);
}

__global__ void __launch_bounds__(kExpT) bfsk_td_expand_host(BfsBufs b, BfsDevState* st, uint32_t n,
                                                             int32_t* parents, uint32_t* distances,
                                                             uint32_t* all_out) {
  __shared__ TdSmemHost sm;
  __shared__ unsigned long long s_red[kRedSlots * kExpT / 32];
  td_expand_phase<false, TdSmemHost>(b, b.list[0], b.list[1], n, st->aux.total_edges, parents, distances, 0, nullptr, all_out,
                         &st->aux, sm, s_red);
}

__global__ void __launch_bounds__(kSearchT) bfsk_bu_host(BfsBufs b, BfsDevState* st, int32_t* parents,
                                                        uint32_t* distances) {
  __shared__ BuHostSmem sm;
  __shared__ unsigned long long s_red[2 * kSearchT / 32];
  bu_host_phase(b, b.bm[0], b.bm[1], b.ul[1], parents, distances, &st->aux, sm, s_red);
}

// Keep the entries of a queue that have out-edges.
__global__ void bfsk_filter_list(const uint32_t* __restrict__ in, uint32_t n, const uint32_t* __restrict__ out_degree,
                                 uint32_t* __restrict__ out, uint32_t* __restrict__ count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = in[i];
    if (out_degree[v]) out[warp_atomic_inc(count)] = v;
  }
}

// Number of reached vertices and the sum of their out-degrees (Graph500
// traversed edges), into st->aux.
__global__ void __launch_bounds__(256) bfsk_reached(BfsBufs b, BfsDevState* st) {
  __shared__ unsigned long long s_red[8];
  const int32_t* parents = st->parents;
  unsigned long long e = 0;
  uint32_t r = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < b.V; v += gridDim.x * blockDim.x) {
    if (parents[v] >= 0) {
      r++;
      e += b.out_degree[v];
    }
  }
  block_add_total<unsigned long long>(&st->aux.reached_edges, e, s_red);
  block_add_total<uint32_t>(&st->aux.reached, r, reinterpret_cast<uint32_t*>(s_red));
}

// ------------------------------------------------------------ host copy ----

// One byte of depth per vertex (a search of fewer than 255 levels): the host
// copy moves V bytes of depths instead of 4V and widens them.
__global__ void __launch_bounds__(256) bfsk_depth_bytes(uint32_t V, const uint32_t* __restrict__ distances,
                                                        uchar4* __restrict__ out) {
  const uint32_t n4 = (V + 3) / 4;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x) {
    const uint32_t v = 4 * i;
    uchar4 q;
    q.x = (unsigned char)distances[v];
    q.y = v + 1 < V ? (unsigned char)distances[v + 1] : 0;
    q.z = v + 2 < V ? (unsigned char)distances[v + 2] : 0;
    q.w = v + 3 < V ? (unsigned char)distances[v + 3] : 0;
    out[i] = q;
  }
}

int bfs_depth_bytes(uint32_t V, const uint32_t* distances, uint8_t* out, cudaStream_t s) {
  const uint32_t n4 = (V + 3) / 4;
  const int grid = (int)std::min<uint32_t>(sm_count() * 8, std::max<uint32_t>(1, (n4 + 255) / 256));
  bfsk_depth_bytes<<<grid, 256, 0, s>>>(V, distances, reinterpret_cast<uchar4*>(out));
  OGB_CUDA(cudaGetLastError());
  return OK;
}

// ------------------------------------------------------------ drivers ------

__global__ void bfsk_cand_flags(const uint2* __restrict__ rows_i, uint32_t V, uint32_t* __restrict__ flags) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    flags[v] = rows_i[v].y ? 1u : 0u;
}

// The record of every vertex with in-edges at its place in vertex order
// (pos: exclusive scan of the flags): A = {vertex, first in-edge, in-degree,
// out-degree}, B = its first kRecN in-neighbours (ids without the mask bits;
// kInvalid past the row's end).
__global__ void bfsk_cand_records(const uint2* __restrict__ rows_i, const uint32_t* __restrict__ nbr_i,
                                  const uint32_t* __restrict__ out_degree, uint32_t V,
                                  const uint32_t* __restrict__ pos, uint4* __restrict__ rec_a,
                                  uint4* __restrict__ rec_b) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint2 row = rows_i[v];
    if (!row.y) continue;
    uint32_t n[kRecN];
#pragma unroll
    for (uint32_t m = 0; m < kRecN; m++) n[m] = m < row.y ? (nbr_i[row.x + m] & 0x3FFFFFFFu) : kInvalid;
    const uint32_t p = pos[v];
    rec_a[p] = make_uint4(v, row.x, row.y, out_degree[v]);
    rec_b[p] = make_uint4(n[0], n[1], n[2], n[3]);
  }
}

// The records of the graph's vertices with in-edges, in vertex order, once
// per build: the first list bottom-up step's candidates (about half the
// vertices of an RMAT graph have no in-edge).  The unvisited lists the steps
// hand on hold at most as many records.
static int bfs_cand0(DevGraph& g, BfsWork* w, cudaStream_t s) {
  if (w->cand0_ready && w->cand0_build == g.build_id) return OK;
  const uint32_t V = g.V;
  // scratch from the search's own V-sized buffers (free outside a search)
  uint32_t* flags = w->fstart.as<uint32_t>();
  uint32_t* pos = w->offs.as<uint32_t>();      // V + 1 words
  uint32_t* tmp = w->fdist.as<uint32_t>();     // scan_tmp_words(V) <= V + 4 words
  const int grid = sm_count() * 8;
  bfsk_cand_flags<<<grid, 256, 0, s>>>(g.inv.d_rows(), V, flags);
  OGB_TRY(scan_exclusive_u32(flags, pos, V, tmp, s));
  uint32_t n = 0;
  OGB_CUDA(cudaMemcpyAsync(&n, pos + V, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  const size_t bytes = (size_t)n * 16 + 16;
  OGB_TRY(w->cand_a.alloc(bytes));
  OGB_TRY(w->cand_b.alloc(bytes));
  OGB_TRY(w->ul_a0.alloc(bytes));
  OGB_TRY(w->ul_a1.alloc(bytes));
  OGB_TRY(w->ul_b0.alloc(bytes));
  OGB_TRY(w->ul_b1.alloc(bytes));
  bfsk_cand_records<<<grid, 256, 0, s>>>(g.inv.d_rows(), g.inv.d_dst(), g.fwd.d_out_degree(), V, pos,
                                         w->cand_a.as<uint4>(), w->cand_b.as<uint4>());
  OGB_CUDA(cudaGetLastError());
  w->n_cand0 = n;
  w->cand0_build = g.build_id;
  w->cand0_ready = true;
  return OK;
}

int bfs_run(DevGraph& g, uint32_t root, uint32_t mode, int32_t* parents, uint32_t* distances, BfsResult* res,
            bool want_trace, bool bu_entry_nf_frontier, cudaStream_t s, bool want_reached) {
  return bfs_run_roots(g, &root, 1, mode, parents, distances, res, want_trace, bu_entry_nf_frontier, s,
                       want_reached);
}

int bfs_run_roots(DevGraph& g, const uint32_t* roots, uint32_t nroots, uint32_t mode, int32_t* parents,
                  uint32_t* distances, BfsResult* res, bool want_trace, bool bu_entry_nf_frontier, cudaStream_t s,
                  bool want_reached) {
  const uint32_t V = g.V;
  if (nroots == 0) return fail(ERR_ARG, "bfs: no root");
  for (uint32_t i = 0; i < nroots; i++)
    if (roots[i] >= V) return fail(ERR_ARG, "bfs: root %u out of range (V=%u)", roots[i], V);
  const uint32_t root = roots[0];
  if (mode > BFS_PULL_DENSE) return fail(ERR_ARG, "bfs: mode %u", mode);
  if (mode == BFS_LEARNED && !bfs_policy_weights()) return fail(ERR_ARG, "bfs: no learned switch installed");
  BfsWork* w = nullptr;
  OGB_TRY(bfs_work_get(g, &w));
  BfsDevState* st = w->state.as<BfsDevState>();
  if (!w->search_grid) {
    int nb = 0;
    OGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, bfsk_search, kSearchT, 0));
    if (nb < 1) return fail(ERR_CUDA, "bfs: search kernel does not fit on an SM");
    w->search_grid = nb * sm_count();
  }
  OGB_TRY(bfs_cand0(g, w, s));
  BfsBufs b = make_bufs(g, w);  // after bfs_cand0: it (re)allocates the record buffers
  if (mode != BFS_LEARNED) {  // the network is read only by the learned switch
    b.policy = nullptr;
    b.policy_tail = nullptr;
  }
  bfsk_init<<<sm_count() * 8, 256, 0, s>>>(b, st, root, parents, distances, mode, bu_entry_nf_frontier ? 1u : 0u,
                                            g.E, w->epoch, w->n_cand0);
  DevBuf d_roots;
  if (nroots > 1) {
    OGB_TRY(d_roots.alloc((size_t)nroots * 4));
    OGB_CUDA(cudaMemcpyAsync(d_roots.p, roots, (size_t)nroots * 4, cudaMemcpyHostToDevice, s));
    bfsk_set_roots<<<1, 32, 0, s>>>(b, st, d_roots.as<uint32_t>(), nroots);
  }
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaEventRecord(w->ev_start, s));
  void* args[] = {(void*)&b, (void*)&st};
  OGB_CUDA(cudaLaunchCooperativeKernel((void*)bfsk_search, dim3(w->search_grid), dim3(kSearchT), args, 0, s));
  OGB_CUDA(cudaEventRecord(w->ev_stop, s));
  OGB_CUDA(cudaMemsetAsync(&st->aux, 0, sizeof(BfsCtl), s));
  if (want_reached) {
    bfsk_reached<<<sm_count() * 8, 256, 0, s>>>(b, st);
    OGB_CUDA(cudaGetLastError());
  }
  OGB_CUDA(cudaMemcpyAsync(w->h_state, w->state.p, offsetof(BfsDevState, trace), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  float total_ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&total_ms, w->ev_start, w->ev_stop));
  const BfsDevState* h = w->h_state;
  w->epoch = h->c.epoch;
  if (h->err)
    return fail((int)h->err, h->err == ERR_STATE ? "bfs: a device-side consistency check failed"
                                                 : "bfs: a bounded device wait gave up");
  if (h->c.overflow) return fail(ERR_SPIN, "bfs: more than V + 8 steps");
  BfsResult r;
  r.iteration = h->c.iteration;
  r.processed_nodes = h->c.processed;
  r.td_steps = h->c.td_steps;
  r.bu_steps = h->c.bu_steps;
  r.edges_examined = h->c.edges_examined;
  r.reached = h->aux.reached;
  r.reached_out_edges = h->aux.reached_edges;
  r.ms = total_ms;
  r.launches = 1;  // kernels in the timed region: the search (init runs before it)
  r.nlevels = (int)h->c.nlevels;
  const uint32_t ntrace = std::min<uint32_t>(h->c.nlevels, kMaxTrace);
  if (want_trace && ntrace) {
    r.levels.resize(ntrace);
    r.feat.resize((size_t)ntrace * kFeat);
    OGB_CUDA(cudaMemcpyAsync(r.levels.data(), st->trace, sizeof(BfsLevel) * ntrace, cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaMemcpyAsync(r.feat.data(), st->feat, sizeof(float) * kFeat * ntrace, cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaStreamSynchronize(s));
  }
  if (res) *res = std::move(r);
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
  BfsDevState* st = w->state.as<BfsDevState>();
  const BfsBufs b = make_bufs(g, w);
  OGB_CUDA(cudaMemcpyAsync(d_par.p, parents, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(d_dist.p, distances, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->ul0.p, q, (size_t)qsize * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemsetAsync(d_cnt.p, 0, 16, s));
  OGB_CUDA(cudaMemsetAsync(&st->aux, 0, sizeof(BfsCtl), s));
  OGB_CUDA(cudaMemsetAsync(&st->err, 0, 4, s));
  if (qsize) {
    bfsk_filter_list<<<std::min<uint32_t>(sm_count() * 8, ceil_div(qsize, 256)), 256, 0, s>>>(
        w->ul0.as<uint32_t>(), qsize, g.fwd.d_out_degree(), b.list[0], d_cnt.as<uint32_t>());
    OGB_CUDA(cudaGetLastError());
  }
  uint32_t n = 0;
  OGB_CUDA(cudaMemcpyAsync(&n, d_cnt.p, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  if (n) {
    const uint32_t epoch = ++w->epoch;
    bfsk_td_scan_host<<<sm_count() * 8, kScanT, 0, s>>>(b, st, n, d_dist.as<uint32_t>(), epoch);
    bfsk_td_expand_host<<<sm_count() * 8, kExpT, 0, s>>>(b, st, n, d_par.as<int32_t>(), d_dist.as<uint32_t>(),
                                                         d_all.as<uint32_t>());
    OGB_CUDA(cudaGetLastError());
  }
  OGB_CUDA(cudaMemcpyAsync(w->h_state, w->state.p, offsetof(BfsDevState, trace), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  if (w->h_state->err) return fail((int)w->h_state->err, "bfs step: a bounded device wait gave up");
  *next_size = w->h_state->aux.qnext;
  *mf = w->h_state->aux.mf;
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
  BfsDevState* st = w->state.as<BfsDevState>();
  const BfsBufs b = make_bufs(g, w);
  OGB_CUDA(cudaMemcpyAsync(d_par.p, parents, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(d_dist.p, distances, (size_t)V * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->bm0.p, bm_cur, words * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->bm1.p, bm_next, words * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemsetAsync(&st->aux, 0, sizeof(BfsCtl), s));
  bfsk_bu_host<<<sm_count() * 8, kSearchT, 0, s>>>(b, st, d_par.as<int32_t>(), d_dist.as<uint32_t>());
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaMemcpyAsync(w->h_state, w->state.p, offsetof(BfsDevState, trace), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  *nf = w->h_state->aux.nf;
  OGB_CUDA(cudaMemcpyAsync(bm_next, w->bm1.p, words * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(parents, d_par.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(distances, d_dist.p, (size_t)V * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}
