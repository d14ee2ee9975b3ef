// pagerank.cu -- PageRank pull and push over the device CSR.
//
// Reference: pageRankPullGraphCSR (00_graph_bench/src/algorithms/openmp/
// pageRank.c:939-1062) and pageRankPushGraphCSR (:1064-1186):
//   start       pr[v] = base_pr = 1 - 0.85f (unnormalized, :47-75)
//   contrib     c[u] = pr[u] / (float)out_degree[u], 0 if out_degree is 0
//   pull        s[v] = sum of c[u] over in-edges (inverse CSR)
//   push        s[u] += c[v] over out-edges (float atomics)
//   update      pr'[v] = base_pr + damp * s[v]  (two roundings, no FMA)
//   error       |pr' - pr| in float, accumulated / V in double; active
//               counts |pr' - pr| >= epsilon; stop after an iteration with
//               no active vertex (iterations then holds that iteration's
//               index) or after `iterations`
//   finish      pr /= (float)V
//
// Device design: the contrib of the next iteration is written by the update
// of this one (double-buffered), so an iteration of pull is ONE kernel that
// gathers, updates, writes the next contrib and reduces error/active.
// Work split by row length (in-degree for pull, out-degree for push):
//   light rows (<= warp_thr edges): a thread per vertex, vertices in
//     ascending order so a warp's 32 rows are adjacent in memory; pull sums
//     sequentially in CSR order -- the reference's exact order;
//   heavy rows (<= cta_thr): a warp per vertex, lanes strided over the row,
//     butterfly-folded;
//   very heavy rows (> cta_thr): cut into chunks of kPrChunk edges, one CTA
//     per chunk (256 threads strided, butterfly per warp, warps in order);
//     the CTA that finishes a vertex's last chunk adds the chunk sums in chunk
//     order and updates the vertex.  A hub therefore never serializes an
//     iteration, and every sum has one fixed order (deterministic).
// Every strided loop issues four independent gathers before it adds them, in
// the same order as the plain loop, so the order is unchanged.
// Pull gathers one contrib value per edge, at random, so it is bound by
// memory latency more than by HBM bandwidth.  Pull therefore runs on a
// re-laid copy of the inverse neighbour array (built once per graph): source
// ids renumbered by descending out-degree, so the contribs of the sources of
// most edges share few cache lines (contrib is kept in that numbering; a
// pull CTA can also stage the leading renumbered sources in shared memory,
// off by default), and the rows of in-degree <= warp_thr stored first and
// contiguous, so a warp loads the edges of 128 light rows with coalesced
// loads and gathers them 256 at a time (light rows were the latency tail of
// the iteration: a lane walked its row one dependent gather per step).  The
// rows, their order and every summation order are unchanged, so the results
// are bit-identical.  Pull runs one 1024-thread CTA per SM; it takes chunks
// first (four 256-thread groups per CTA), then warp rows, then light rows.  Iterations are launched back to back
// without host round trips: each iteration's last CTA records error/active
// and, when active == 0, sets a stop flag that later launches read first.
#include "graph.cuh"

#include <algorithm>
#include <vector>

namespace ogb {

constexpr uint32_t kPrMaxIters = 1024;
constexpr int kPrThreads = 256;      // push kernels
constexpr int kPullThreads = 1024;   // pull: one CTA per SM
constexpr int kPullGroup = 256;      // threads per chunk group (the oracle's cta_threads)
constexpr int kPullGroups = kPullThreads / kPullGroup;
constexpr uint32_t kStage = 256;     // staged edges per warp and window
constexpr int kLightR = 4;           // light rows per lane (128 per warp unit)
constexpr uint32_t kUnit = 4096;     // medium-row edges per warp unit
constexpr uint32_t kTab = 64;        // medium rows per table batch
constexpr uint32_t kWarpSmemWords = kStage + 3 * kTab + 1;  // stage + table of one warp
constexpr size_t kPullDynSmem = (size_t)(kPullThreads / 32) * kWarpSmemWords * 4;
constexpr uint32_t kHotLimit = 0;    // renumbered sources whose contrib a pull CTA stages in shared memory
constexpr uint32_t kPrChunk = 8192;  // edges per chunk of a very heavy row
constexpr uint32_t kPushHubDeg = 256;  // push: destinations with more in-edges are hubs
constexpr uint32_t kHubChunk = 1024;   // push: in-edges of a hub summed by one warp

// Row-length thresholds of the work split (settable; the GPU-order mode of
// the oracle takes the same values).
static uint32_t g_warp_thr = 32;
static uint32_t g_cta_thr = 2048;

void pagerank_set_bins(uint32_t warp_thr, uint32_t cta_thr) {
  g_warp_thr = warp_thr;
  g_cta_thr = std::max(cta_thr, warp_thr);
}
void pagerank_get_bins(uint32_t* warp_thr, uint32_t* cta_thr, uint32_t* cta_threads, uint32_t* chunk) {
  *warp_thr = g_warp_thr;
  *cta_thr = g_cta_thr;
  *cta_threads = kPullGroup;
  *chunk = kPrChunk;
}

struct PrCtl {
  double err[kPrMaxIters];
  uint32_t active[kPrMaxIters];
  uint32_t blocks_done[kPrMaxIters];
  uint32_t claim_med[kPrMaxIters];    // pull: medium units handed out
  uint32_t claim_light[kPrMaxIters];  // pull: light units handed out
  uint32_t stop;       // 1 once an iteration ended with no active vertex
  uint32_t stop_iter;  // index of that iteration
};

struct PrChunkItem {
  uint32_t v, j0, j1, k;  // vertex, edge range, index of the vertex in the chunked list
};

struct PrWork {
  uint32_t V = 0;
  int listed_pull = -1;                // direction the lists describe
  uint32_t listed_warp = 0, listed_cta = 0, listed_build = 0;
  // pull: source ids renumbered by descending out-degree
  uint32_t rl_build = 0, rl_warp = 0, rl_cta = 0;
  bool rl_ready = false;
  DevBuf perm, nbr_rl, rows_rl, off_light, med_v, med_off, unit_first, rl_tmp;
  uint32_t n_med = 0, n_units = 0, med_base = 0;
  uint32_t hot = 0;  // staged renumbered sources
  DevBuf contrib0, contrib1, next, ctl;
  DevBuf heavy;                        // vertex ids of the warp rows (n_warp), then the chunked rows
  DevBuf chunks;                       // PrChunkItem per chunk
  DevBuf vfirst, vcount, done;         // per chunked vertex: first chunk, chunk count, finished chunks
  DevBuf partials;                     // float per chunk
  uint32_t n_warp = 0, n_cta = 0, n_chunks = 0;
  // push: the pushes into each hub (in-degree > kPushHubDeg) are summed over
  // the hub's in-row and applied once per chunk; the other out-edges scatter
  // from a filtered copy of the forward CSR
  uint32_t push_build = 0;
  bool push_ready = false;
  DevBuf rows_fp, nbr_fp, hub_items;   // filtered rows {start, count}, their neighbours; hub chunks {v, j0, j1, 0}
  uint32_t n_hub_items = 0;
  PrCtl* h_ctl = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~PrWork() {
    if (h_ctl) cudaFreeHost(h_ctl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

void pr_work_free(PrWork* w) { delete w; }

// ------------------------------------------------------------ heavy lists ---

__global__ void pr_heavy_count_kernel(uint32_t V, const uint2* __restrict__ rows, uint32_t warp_thr,
                                      uint32_t cta_thr, uint32_t* __restrict__ counts) {
  uint32_t cw = 0, cc = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    cw += (d > warp_thr && d <= cta_thr);
    cc += (d > cta_thr);
  }
  warp_atomic_add_total(&counts[0], cw);
  warp_atomic_add_total(&counts[1], cc);
}

// Order inside a list does not change results: each row is reduced by one
// warp, or by its chunks in a fixed order.
__global__ void pr_heavy_fill_kernel(uint32_t V, const uint2* __restrict__ rows, uint32_t warp_thr,
                                     uint32_t cta_thr, uint32_t* __restrict__ cursor, uint32_t* __restrict__ list,
                                     uint32_t off_cta, uint4* __restrict__ cta_rows) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint2 r = rows[v];
    if (r.y > cta_thr) {
      const uint32_t k = atomicAdd(&cursor[1], 1u);
      list[off_cta + k] = v;
      cta_rows[k] = make_uint4(v, r.x, r.y, 0);
    } else if (r.y > warp_thr) {
      list[atomicAdd(&cursor[0], 1u)] = v;
    }
  }
}

// ---------------------------------------------------------------- update ----

struct PrParams {
  float base_pr, damp;
  double epsilon;
  uint32_t V;
  uint32_t warp_thr;
  // many graphs in one (a disjoint union): graph of each vertex, graphs that
  // stopped (their vertices keep their rank), and each vertex's change for
  // the per-graph error / stop rule; null for a single graph
  const uint32_t* gid;
  const uint32_t* frozen;
  float* delta;
};

// contrib_next is indexed by renumbered id when perm is given.
__device__ __forceinline__ void pr_update(uint32_t v, float s, float* __restrict__ pr,
                                          const uint32_t* __restrict__ out_degree,
                                          float* __restrict__ contrib_next, const PrParams& p, double& err,
                                          uint32_t& active, const uint32_t* __restrict__ perm = nullptr) {
  const float prev = pr[v];
  float nv = __fadd_rn(p.base_pr, __fmul_rn(p.damp, s));
  if (p.frozen && p.frozen[p.gid[v]]) nv = prev;
  pr[v] = nv;
  const uint32_t d = out_degree[v];
  contrib_next[perm ? perm[v] : v] = d ? __fdiv_rn(nv, (float)d) : 0.0f;
  if (p.delta) p.delta[v] = __fsub_rn(nv, prev);
  const double e = fabs((double)__fsub_rn(nv, prev));
  err += e / (double)p.V;
  active += (e >= p.epsilon) ? 1u : 0u;
}

template <int NT = kPrThreads>
__device__ __forceinline__ void pr_block_finish(double err, uint32_t active, PrCtl* ctl, uint32_t it) {
  __shared__ double s_err[NT / 32];
  __shared__ uint32_t s_act[NT / 32];
  for (int o = 16; o; o >>= 1) {
    err += __shfl_down_sync(0xffffffffu, err, o);
    active += __shfl_down_sync(0xffffffffu, active, o);
  }
  const int warp = threadIdx.x >> 5;
  if (lane_id() == 0) {
    s_err[warp] = err;
    s_act[warp] = active;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0;
    uint32_t a = 0;
    for (int w = 0; w < NT / 32; w++) {
      e += s_err[w];
      a += s_act[w];
    }
    if (e != 0.0) atomicAdd(&ctl->err[it], e);
    if (a) atomicAdd(&ctl->active[it], a);
    __threadfence();
    const uint32_t done = atomicAdd(&ctl->blocks_done[it], 1u);
    if (done == gridDim.x - 1) {
      __threadfence();
      if (atomicAdd(&ctl->active[it], 0u) == 0u) {
        ctl->stop_iter = it;
        ctl->stop = 1;
      }
    }
  }
}

// s += c[nbr[j]] for j = j0, j0+STRIDE, ... < j1, in that order; each step
// issues four predicated neighbour loads, then their four gathers.
template <uint32_t STRIDE>
__device__ __forceinline__ float strided_sum(const float* __restrict__ c, const uint32_t* __restrict__ nbr,
                                             uint32_t j0, uint32_t j1) {
  float s = 0.0f;
  for (uint32_t j = j0; j < j1; j += 4 * STRIDE) {
    uint32_t x[4];
#pragma unroll
    for (int k = 0; k < 4; k++) x[k] = (j + k * STRIDE < j1) ? __ldg(&nbr[j + k * STRIDE]) : 0u;
    float cx[4];
#pragma unroll
    for (int k = 0; k < 4; k++) cx[k] = (j + k * STRIDE < j1) ? __ldg(&c[x[k]]) : 0.0f;
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (j + k * STRIDE < j1) s = __fadd_rn(s, cx[k]);
  }
  return s;
}

__device__ __forceinline__ float warp_fold(float s) {
#pragma unroll
  for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
}

__device__ __forceinline__ uint32_t ceil_div_dev(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// Update inputs of vertex v, loaded before its sum is ready.
struct PrVtx {
  float prev;
  uint32_t deg, pm;
};
__device__ __forceinline__ PrVtx pr_vtx(uint32_t v, const float* __restrict__ pr, const uint32_t* __restrict__ out_degree,
                                        const uint32_t* __restrict__ perm) {
  PrVtx x;
  x.prev = pr[v];
  x.deg = __ldg(&out_degree[v]);
  x.pm = __ldg(&perm[v]);
  return x;
}
// pr_update with preloaded inputs (contrib_next at the renumbered id).
__device__ __forceinline__ void pr_update_pre(uint32_t v, float s, const PrVtx& x, float* __restrict__ pr,
                                              float* __restrict__ contrib_next, const PrParams& p, double& err,
                                              uint32_t& active) {
  float nv = __fadd_rn(p.base_pr, __fmul_rn(p.damp, s));
  if (p.frozen && p.frozen[p.gid[v]]) nv = x.prev;
  pr[v] = nv;
  contrib_next[x.pm] = x.deg ? __fdiv_rn(nv, (float)x.deg) : 0.0f;
  if (p.delta) p.delta[v] = __fsub_rn(nv, x.prev);
  const double e = fabs((double)__fsub_rn(nv, x.prev));
  err += e / (double)p.V;
  active += (e >= p.epsilon) ? 1u : 0u;
}

__device__ __forceinline__ void cp_async4(float* dst_smem, const float* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// A warp walks an edge range [e0, e1) in windows of kStage edges: the
// contribs of a window are copied straight into the warp's stage by
// asynchronous 4-byte copies (kStage / 32 per lane in flight, no registers
// held for them), and the neighbour ids of the next window load meanwhile.
struct StagePipe {
  uint32_t u[kStage / 32];
  __device__ __forceinline__ void load(const uint32_t* __restrict__ nbr, uint32_t w0, uint32_t e1, uint32_t lane) {
#pragma unroll
    for (uint32_t m = 0; m < kStage / 32; m++) {
      const uint32_t j = w0 + m * 32 + lane;
      u[m] = j < e1 ? __ldg(&nbr[j]) : 0u;
    }
  }
  // Gather window [w0, min(w0 + kStage, e1)) into stage; the next window's
  // ids are loaded into u meanwhile.  The caller syncs the warp afterwards.
  __device__ __forceinline__ void gather(float* stage, const uint32_t* __restrict__ nbr, const float* __restrict__ c,
                                         const float* s_hot, uint32_t hot, uint32_t w0, uint32_t e1, uint32_t lane) {
#pragma unroll
    for (uint32_t m = 0; m < kStage / 32; m++) {
      const uint32_t j = w0 + m * 32 + lane;
      if (j < e1) {
        if (u[m] < hot)
          stage[m * 32 + lane] = s_hot[u[m]];
        else
          cp_async4(&stage[m * 32 + lane], c + u[m]);
      }
    }
    load(nbr, w0 + kStage, e1, lane);
    cp_async_wait_all();
  }
};

// Pull iteration, one CTA per SM (1024 threads).  The inverse neighbour
// array is in the re-laid form: light rows (in-degree <= warp_thr) first,
// then medium rows (<= cta_thr), then the rest, each class contiguous in
// vertex order, with renumbered source ids.  Work, each kind strided over
// the grid:
//  (1) chunks of very heavy rows, one 256-thread group per chunk (four in
//      flight per CTA): lanes strided, warps folded, the group's warps summed
//      in order, the chunk sums in chunk order by the group that finishes a
//      row's last chunk;
//  (2) medium rows, a warp per unit of kUnit edges (the rows starting in
//      it): the unit's edges are gathered kStage at a time into the warp's
//      stage with coalesced loads; lane l adds the elements l, l+32, ... of
//      each row in order, and the row is butterfly-folded when it ends;
//  (3) light rows, a warp per 128 consecutive vertices: their edges are
//      contiguous, gathered into the stage the same way, and each lane adds
//      its four rows' values in CSR order.
// rows_rl, pr and out_degree are in original vertex order; contrib and
// contrib_next are indexed by renumbered id (perm).
__global__ void __launch_bounds__(kPullThreads, 1) pr_pull_kernel(
    uint32_t hot, const PrChunkItem* __restrict__ chunks, uint32_t n_chunks, const uint32_t* __restrict__ vfirst,
    const uint32_t* __restrict__ vcount, uint32_t* __restrict__ done, float* __restrict__ partials,
    const uint2* __restrict__ rows, const uint32_t* __restrict__ off_light, const uint32_t* __restrict__ unit_first,
    uint32_t n_units, const uint32_t* __restrict__ med_off, const uint32_t* __restrict__ med_v, uint32_t med_base,
    const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ out_degree, const uint32_t* __restrict__ perm,
    const float* __restrict__ contrib, float* __restrict__ contrib_next, float* __restrict__ pr, PrParams p,
    PrCtl* __restrict__ ctl, uint32_t it) {
  extern __shared__ uint32_t s_dyn[];  // per warp: stage and medium-row table; then the hot contribs
  __shared__ float s_part[kPullGroups][kPullGroup / 32];
  __shared__ uint32_t s_last[kPullGroups];
  if (ctl->stop) return;
  float* s_hot = reinterpret_cast<float*>(s_dyn + (kPullThreads / 32) * kWarpSmemWords);
  for (uint32_t i = threadIdx.x; i < hot / 4; i += kPullThreads)
    reinterpret_cast<float4*>(s_hot)[i] = __ldg(reinterpret_cast<const float4*>(contrib) + i);
  __syncthreads();
  double err = 0.0;
  uint32_t active = 0;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;

  // (1) chunks of very heavy rows, one group per chunk
  {
    const uint32_t grp = threadIdx.x / kPullGroup, gt = threadIdx.x % kPullGroup;
    for (uint32_t g = blockIdx.x * kPullGroups + grp; g < n_chunks; g += gridDim.x * kPullGroups) {
      const PrChunkItem ci = chunks[g];
      float sum = strided_sum<kPullGroup>(contrib, nbr, ci.j0 + gt, ci.j1);
      sum = warp_fold(sum);
      if (lane == 0) s_part[grp][gt >> 5] = sum;
      asm volatile("bar.sync %0, %1;" ::"r"(grp + 1), "r"(kPullGroup) : "memory");
      if (gt == 0) {
        float tot = 0.0f;
        for (int w = 0; w < kPullGroup / 32; w++) tot = __fadd_rn(tot, s_part[grp][w]);
        partials[g] = tot;
        __threadfence();
        const uint32_t cnt = vcount[ci.k];
        s_last[grp] = (atomicAdd(&done[ci.k], 1u) == cnt - 1) ? 1u : 0u;
        if (s_last[grp]) {
          __threadfence();
          const uint32_t f = vfirst[ci.k];
          float rs = 0.0f;
          for (uint32_t c = 0; c < cnt; c++) rs = __fadd_rn(rs, __ldcg(&partials[f + c]));
          done[ci.k] = 0;
          pr_update(ci.v, rs, pr, out_degree, contrib_next, p, err, active, perm);
        }
      }
      asm volatile("bar.sync %0, %1;" ::"r"(grp + 1), "r"(kPullGroup) : "memory");
    }
  }

  uint32_t* mine = s_dyn + warp * kWarpSmemWords;
  float* stage = reinterpret_cast<float*>(mine);

  // (2) medium rows, a warp per unit, rows taken in batches of kTab
  uint32_t* toff = mine + kStage;
  uint32_t* tv = toff + kTab + 1;
  float* tsum = reinterpret_cast<float*>(tv + kTab);
  uint32_t* claim = &ctl->claim_med[it];
  uint32_t t = __shfl_sync(0xffffffffu, lane == 0 ? atomicAdd(claim, 1u) : 0u, 0);
  while (t < n_units) {
    const uint32_t t_next = lane == 0 ? atomicAdd(claim, 1u) : 0u;  // next claim, in flight meanwhile
    const uint32_t i0 = unit_first[t], i1 = unit_first[t + 1];
    for (uint32_t ib = i0; ib < i1; ib += kTab) {
      const uint32_t nr = min(ib + kTab, i1) - ib;
      for (uint32_t k = lane; k <= nr; k += 32) toff[k] = med_base + med_off[ib + k];
      for (uint32_t k = lane; k < nr; k += 32) tv[k] = med_v[ib + k];
      __syncwarp();
      const uint32_t e0 = toff[0], e1 = toff[nr];
      uint32_t r = 0;
      float s = 0.0f;
      StagePipe pipe;
      pipe.load(nbr, e0, e1, lane);
      for (uint32_t w0 = e0; w0 < e1; w0 += kStage) {
        const uint32_t w1 = min(w0 + kStage, e1);
        pipe.gather(stage, nbr, contrib, s_hot, hot, w0, e1, lane);
        __syncwarp();
        while (r < nr) {
          const uint32_t rs = toff[r], re = toff[r + 1];
          const uint32_t lo = max(rs, w0), hi = min(re, w1);
          // lane l takes the row's elements rs + l + 32 m
          for (uint32_t j = lo + ((rs + lane - lo) & 31u); j < hi; j += 32) s = __fadd_rn(s, stage[j - w0]);
          if (re > w1) break;  // the row goes on in the next window
          s = warp_fold(s);
          if (lane == 0) tsum[r] = s;
          s = 0.0f;
          r++;
        }
        __syncwarp();
      }
      for (uint32_t k = lane; k < nr; k += 32) {
        const uint32_t v = tv[k];
        const PrVtx x = pr_vtx(v, pr, out_degree, perm);
        pr_update_pre(v, tsum[k], x, pr, contrib_next, p, err, active);
      }
      __syncwarp();
    }
    t = __shfl_sync(0xffffffffu, t_next, 0);
  }

  // (3) light rows, a warp per 128 consecutive vertices
  const uint32_t n_light = ceil_div_dev(p.V, 32 * kLightR);
  claim = &ctl->claim_light[it];
  t = __shfl_sync(0xffffffffu, lane == 0 ? atomicAdd(claim, 1u) : 0u, 0);
  while (t < n_light) {
    const uint32_t t_next = lane == 0 ? atomicAdd(claim, 1u) : 0u;
    const uint32_t base = t * (32 * kLightR);
    const uint32_t vend = min(base + 32 * kLightR, p.V);
    uint32_t st[kLightR], en[kLightR];
    bool light[kLightR];
    PrVtx x[kLightR];
    float s[kLightR];
#pragma unroll
    for (int k = 0; k < kLightR; k++) {
      const uint32_t v = base + k * 32 + lane;
      st[k] = en[k] = 0;
      light[k] = false;
      s[k] = 0.0f;
      if (v < p.V) {
        light[k] = rows[v].y <= p.warp_thr;
        st[k] = off_light[v];
        en[k] = off_light[v + 1];
        if (light[k]) x[k] = pr_vtx(v, pr, out_degree, perm);
      }
    }
    const uint32_t seg0 = off_light[base], seg1 = off_light[vend];
    StagePipe pipe;
    pipe.load(nbr, seg0, seg1, lane);
    for (uint32_t w0 = seg0; w0 < seg1; w0 += kStage) {
      const uint32_t w1 = min(w0 + kStage, seg1);
      pipe.gather(stage, nbr, contrib, s_hot, hot, w0, seg1, lane);
      __syncwarp();
      uint32_t lo[kLightR], n[kLightR], nmax = 0;
#pragma unroll
      for (int k = 0; k < kLightR; k++) {
        lo[k] = max(st[k], w0);
        const uint32_t hi = min(en[k], w1);
        n[k] = hi > lo[k] ? hi - lo[k] : 0u;
        nmax = max(nmax, n[k]);
      }
      for (uint32_t i = 0; i < nmax; i++) {
#pragma unroll
        for (int k = 0; k < kLightR; k++)
          if (i < n[k]) s[k] = __fadd_rn(s[k], stage[lo[k] - w0 + i]);
      }
      __syncwarp();
    }
#pragma unroll
    for (int k = 0; k < kLightR; k++)
      if (light[k]) pr_update_pre(base + k * 32 + lane, s[k], x[k], pr, contrib_next, p, err, active);
    t = __shfl_sync(0xffffffffu, t_next, 0);
  }
  pr_block_finish<kPullThreads>(err, active, ctl, it);
}

// ---------------------------------------------------------------- renumbering

// key = ~out_degree (ascending sort = descending degree), payload = id.
__global__ void pr_rl_keys_kernel(uint32_t V, const uint32_t* __restrict__ out_degree, uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ ids) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    keys[v] = ~out_degree[v];
    ids[v] = v;
  }
}

// perm[old id] = new id, from the sorted ids (new id -> old id).
__global__ void pr_rl_perm_kernel(uint32_t V, const uint32_t* __restrict__ order, uint32_t* __restrict__ perm) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) perm[order[i]] = i;
}

// Row lengths by class (light <= warp_thr < medium <= cta_thr < chunked),
// and the medium flag.
__global__ void pr_rl_split_kernel(uint32_t V, const uint2* __restrict__ rows, uint32_t warp_thr, uint32_t cta_thr,
                                   uint32_t* __restrict__ dl, uint32_t* __restrict__ dm, uint32_t* __restrict__ dc,
                                   uint32_t* __restrict__ fm) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    const uint32_t cls = d <= warp_thr ? 0u : (d <= cta_thr ? 1u : 2u);
    dl[v] = cls == 0 ? d : 0u;
    dm[v] = cls == 1 ? d : 0u;
    dc[v] = cls == 2 ? d : 0u;
    fm[v] = cls == 1 ? 1u : 0u;
  }
}

// New row offsets (light | medium | chunked), and the medium row list:
// med_v[i] = vertex, med_off[i] = its offset inside the medium class.
__global__ void pr_rl_rows_kernel(uint32_t V, const uint2* __restrict__ rows, uint32_t warp_thr, uint32_t cta_thr,
                                  const uint32_t* __restrict__ off_l, const uint32_t* __restrict__ off_m,
                                  const uint32_t* __restrict__ off_c, const uint32_t* __restrict__ idx_m,
                                  uint2* __restrict__ rows_rl, uint32_t* __restrict__ med_v,
                                  uint32_t* __restrict__ med_off) {
  const uint32_t L = off_l[V], M = off_m[V];
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    uint32_t o;
    if (d <= warp_thr) {
      o = off_l[v];
    } else if (d <= cta_thr) {
      o = L + off_m[v];
      med_v[idx_m[v]] = v;
      med_off[idx_m[v]] = off_m[v];
    } else {
      o = L + M + off_c[v];
    }
    rows_rl[v] = make_uint2(o, d);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) med_off[idx_m[V]] = M;
}

// unit_first[t] = first medium row starting at or after t * kUnit.
__global__ void pr_rl_units_kernel(uint32_t n_units, const uint32_t* __restrict__ med_off, uint32_t n_med,
                                   uint32_t* __restrict__ unit_first) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= n_units; t += gridDim.x * blockDim.x) {
    const uint64_t key = (uint64_t)t * kUnit;
    uint32_t lo = 0, hi = n_med;  // answer in [0, n_med]
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if ((uint64_t)med_off[mid] < key)
        lo = mid + 1;
      else
        hi = mid;
    }
    unit_first[t] = lo;
  }
}

// Copy every row into the new layout with renumbered source ids (a warp
// per row).
__global__ void pr_rl_copy_kernel(uint32_t V, const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr,
                                  const uint2* __restrict__ rows_rl, const uint32_t* __restrict__ perm,
                                  uint32_t* __restrict__ out) {
  const uint32_t lane = lane_id();
  const uint32_t nwarps = gridDim.x * (blockDim.x / 32);
  for (uint32_t v = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); v < V; v += nwarps) {
    const uint2 r = rows[v];
    const uint32_t o = rows_rl[v].x;
    for (uint32_t i = lane; i < r.y; i += 32) out[o + i] = perm[nbr[r.x + i] & 0x3FFFFFFFu];
  }
}


// ---------------------------------------------------------------- push ------
//
// Push adds c[v] into next[u] for every out-edge v -> u (pageRank.c:1117-1134:
// one float atomic per edge).  On RMAT graphs a few destinations take most of
// those adds (RMAT-22: the 35,443 with more than 256 in-edges take 56 % of
// them, the largest 161 K), and float atomics on one address serialize at its
// L2 slice.
// So the adds into every hub -- a destination with more than kPushHubDeg
// in-edges -- are combined first: a warp sums, for a chunk of kHubChunk of the
// hub's pushers (its in-row lists exactly the sources that push into it), the
// values they push, and applies the sum with one atomic.  Every other out-edge
// is scattered with its own atomic from a filtered copy of the forward CSR
// (built once per graph).  The set of additions is the reference's; only their
// order differs, which the reference's own atomics leave open as well.

// The filtered forward CSR is a stable compaction of the forward edge array:
// a flag per edge (its destination is not a hub), an exclusive scan of the
// flags, then each kept edge moves to its scanned position and each row's
// start is the scan at the row's first edge.  Edge-parallel, so the rows of
// the sources with most out-edges cost no more than any others.
__global__ void pr_push_flag_kernel(uint32_t E, const uint32_t* __restrict__ nbr_f, const uint2* __restrict__ rows_i,
                                    uint32_t hub_deg, uint32_t* __restrict__ flag) {
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
    flag[e] = rows_i[nbr_f[e] & 0x3FFFFFFFu].y <= hub_deg ? 1u : 0u;
}

__global__ void pr_push_compact_kernel(uint32_t E, const uint32_t* __restrict__ nbr_f, const uint32_t* __restrict__ flag,
                                       const uint32_t* __restrict__ pos, uint32_t* __restrict__ nbr_fp) {
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
    if (flag[e]) nbr_fp[pos[e]] = nbr_f[e];
}

__global__ void pr_push_rows_kernel(uint32_t V, const uint2* __restrict__ rows_f, const uint32_t* __restrict__ pos,
                                    uint2* __restrict__ rows_fp) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint2 r = rows_f[v];
    // a row without edges may sit anywhere (its edges_idx is 0): it keeps none
    const uint32_t a = r.y ? pos[r.x] : 0u;
    rows_fp[v] = make_uint2(a, r.y ? pos[r.x + r.y] - a : 0u);
  }
}

// Hub chunks per vertex, then their table {hub, first in-edge, end, 0}.
__global__ void pr_hub_count_kernel(uint32_t V, const uint2* __restrict__ rows_i, uint32_t hub_deg,
                                    uint32_t* __restrict__ cnt) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows_i[v].y;
    cnt[v] = d > hub_deg ? (d + kHubChunk - 1) / kHubChunk : 0u;
  }
}
__global__ void pr_hub_fill_kernel(uint32_t V, const uint2* __restrict__ rows_i, uint32_t hub_deg,
                                   const uint32_t* __restrict__ pos, uint4* __restrict__ items) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint2 r = rows_i[v];
    if (r.y <= hub_deg) continue;
    uint32_t k = pos[v];
    for (uint32_t c = 0; c < r.y; c += kHubChunk, k++) items[k] = make_uint4(v, r.x + c, r.x + min(r.y, c + kHubChunk), 0u);
  }
}

// Push scatter, four kinds of blocks: hub chunks (a warp per chunk: the
// chunk's pushers' contribs summed, four gathers in flight per lane, one
// atomic), then the filtered rows split by out-degree like the pull gather
// (chunks of very long rows, a warp per long row, a thread per short row),
// one atomic per edge.
__global__ void __launch_bounds__(kPrThreads) pr_push_scatter_kernel(
    uint32_t nb_hub, const uint4* __restrict__ hub_items, uint32_t n_hub_items, const uint32_t* __restrict__ nbr_i,
    uint32_t nb_chunk, uint32_t nb_warp, const uint32_t* __restrict__ heavy, uint32_t n_warp,
    const PrChunkItem* __restrict__ chunks, uint32_t n_chunks, uint32_t V, uint32_t warp_thr,
    const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr, const float* __restrict__ contrib,
    float* __restrict__ next, const PrCtl* __restrict__ ctl) {
  if (ctl->stop) return;
  uint32_t b = blockIdx.x;
  if (b < nb_hub) {
    const uint32_t lane = lane_id();
    const uint32_t wstride = nb_hub * (kPrThreads / 32);
    for (uint32_t t = b * (kPrThreads / 32) + (threadIdx.x >> 5); t < n_hub_items; t += wstride) {
      const uint4 it = hub_items[t];
      float sum = 0.0f;
      for (uint32_t j = it.y + lane; j < it.z; j += 4 * 32) {
        uint32_t x[4];
#pragma unroll
        for (int k = 0; k < 4; k++) x[k] = (j + k * 32 < it.z) ? (__ldg(&nbr_i[j + k * 32]) & 0x3FFFFFFFu) : 0u;
        float cx[4];
#pragma unroll
        for (int k = 0; k < 4; k++) cx[k] = (j + k * 32 < it.z) ? __ldg(&contrib[x[k]]) : 0.0f;
#pragma unroll
        for (int k = 0; k < 4; k++) sum += cx[k];
      }
      sum = warp_fold(sum);
      if (lane == 0) atomicAdd(&next[it.x], sum);
    }
    return;
  }
  b -= nb_hub;
  if (b < nb_chunk) {
    for (uint32_t g = b; g < n_chunks; g += nb_chunk) {
      const PrChunkItem ci = chunks[g];
      const float c = contrib[ci.v];
      for (uint32_t j = ci.j0 + threadIdx.x; j < ci.j1; j += kPrThreads) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  } else if (b < nb_chunk + nb_warp) {
    const uint32_t w0 = (b - nb_chunk) * (kPrThreads / 32) + (threadIdx.x >> 5);
    const uint32_t wstride = nb_warp * (kPrThreads / 32);
    for (uint32_t t = w0; t < n_warp; t += wstride) {
      const uint32_t v = heavy[t];
      const uint2 row = rows[v];
      const float c = contrib[v];
      for (uint32_t j = row.x + lane_id(); j < row.x + row.y; j += 32) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  } else {
    const uint32_t lb = b - nb_chunk - nb_warp;
    const uint32_t nlb = gridDim.x - nb_hub - nb_chunk - nb_warp;
    for (uint32_t v = lb * kPrThreads + threadIdx.x; v < V; v += nlb * kPrThreads) {
      const uint2 row = rows[v];
      if (row.y > warp_thr) continue;
      const float c = contrib[v];
      for (uint32_t j = row.x; j < row.x + row.y; j++) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  }
}

// One vertex of the push update: the reference's rank update, its contrib for
// the next iteration, and its |change| / V (as a product with 1 / V: one more
// rounding per term than a division, far inside the sum's own order effects).
__device__ __forceinline__ float pr_push_vtx(float s, float prev, uint32_t d, float& c, const PrParams& p,
                                             double inv_v, double& err, uint32_t& active) {
  const float nv = __fadd_rn(p.base_pr, __fmul_rn(p.damp, s));
  c = d ? __fdiv_rn(nv, (float)d) : 0.0f;
  const double e = fabs((double)__fsub_rn(nv, prev));
  err += e * inv_v;
  active += (e >= p.epsilon) ? 1u : 0u;
  return nv;
}

// Push update: next -> ranks and next contribs, next cleared.  Four vertices
// per thread and step with 16-byte loads and stores (the arrays are 16-byte
// aligned), so each thread keeps several loads in flight; a scalar tail.
__global__ void __launch_bounds__(kPrThreads) pr_push_update_kernel(uint32_t V, const uint32_t* __restrict__ out_degree,
                                                                    float* __restrict__ next,
                                                                    float* __restrict__ contrib_next,
                                                                    float* __restrict__ pr, PrParams p,
                                                                    PrCtl* __restrict__ ctl, uint32_t it) {
  if (ctl->stop) return;
  double err = 0.0;
  uint32_t active = 0;
  const double inv_v = 1.0 / (double)p.V;
  const uint32_t stride = gridDim.x * kPrThreads;
  const bool vec = !p.frozen && !p.delta &&
                   ((reinterpret_cast<uintptr_t>(next) | reinterpret_cast<uintptr_t>(contrib_next) |
                     reinterpret_cast<uintptr_t>(pr) | reinterpret_cast<uintptr_t>(out_degree)) & 15) == 0;
  uint32_t v0 = 0;
  if (vec) {
    const uint32_t nq = V / 4;
    for (uint32_t q = blockIdx.x * kPrThreads + threadIdx.x; q < nq; q += stride) {
      const float4 sv = reinterpret_cast<const float4*>(next)[q];
      const float4 pv = reinterpret_cast<const float4*>(pr)[q];
      const uint4 dv = reinterpret_cast<const uint4*>(out_degree)[q];
      reinterpret_cast<float4*>(next)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      float4 nv, cv;
      nv.x = pr_push_vtx(sv.x, pv.x, dv.x, cv.x, p, inv_v, err, active);
      nv.y = pr_push_vtx(sv.y, pv.y, dv.y, cv.y, p, inv_v, err, active);
      nv.z = pr_push_vtx(sv.z, pv.z, dv.z, cv.z, p, inv_v, err, active);
      nv.w = pr_push_vtx(sv.w, pv.w, dv.w, cv.w, p, inv_v, err, active);
      reinterpret_cast<float4*>(pr)[q] = nv;
      reinterpret_cast<float4*>(contrib_next)[q] = cv;
    }
    v0 = nq * 4;
  }
  for (uint32_t v = v0 + blockIdx.x * kPrThreads + threadIdx.x; v < V; v += stride) {
    const float sv = next[v];
    next[v] = 0.0f;
    if (vec) {
      float c;
      pr[v] = pr_push_vtx(sv, pr[v], out_degree[v], c, p, inv_v, err, active);
      contrib_next[v] = c;
    } else {
      pr_update(v, sv, pr, out_degree, contrib_next, p, err, active);
    }
  }
  pr_block_finish(err, active, ctl, it);
}

__global__ void pr_init_kernel(uint32_t V, const uint32_t* __restrict__ out_degree, const float* __restrict__ init,
                               float base_pr, float* __restrict__ pr, float* __restrict__ contrib,
                               float* __restrict__ next, const uint32_t* __restrict__ perm) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const float x = init ? init[v] : base_pr;
    pr[v] = x;
    const uint32_t d = out_degree[v];
    contrib[perm ? perm[v] : v] = d ? __fdiv_rn(x, (float)d) : 0.0f;
    if (next) next[v] = 0.0f;
  }
}

__global__ void pr_normalize_kernel(uint32_t V, float* __restrict__ pr) {
  const float fv = (float)V;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    pr[v] = __fdiv_rn(pr[v], fv);
}

// Heavy lists and the chunk table of one direction (built once per graph,
// direction and thresholds; the only host round trips of PageRank).
// Pull lists refer to the renumbered layout (rows_rl), push lists to the
// filtered forward CSR (rows_fp).
static int pr_build_lists(DevGraph& g, PrWork* w, bool pull, cudaStream_t s) {
  const uint32_t V = g.V;
  const uint2* rows = pull ? w->rows_rl.as<uint2>() : w->rows_fp.as<uint2>();
  uint32_t* cnt = w->ctl.as<uint32_t>() + sizeof(PrCtl) / 4;  // scratch words after the control block
  OGB_CUDA(cudaMemsetAsync(cnt, 0, 16, s));
  const int grid = sm_count() * 8;
  pr_heavy_count_kernel<<<grid, 256, 0, s>>>(V, rows, g_warp_thr, g_cta_thr, cnt);
  OGB_CUDA(cudaGetLastError());
  uint32_t h[2];
  OGB_CUDA(cudaMemcpyAsync(h, cnt, 8, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  w->n_warp = h[0];
  w->n_cta = h[1];
  DevBuf cta_rows;
  OGB_TRY(cta_rows.alloc((size_t)w->n_cta * 16 + 16));
  OGB_CUDA(cudaMemsetAsync(cnt, 0, 16, s));
  pr_heavy_fill_kernel<<<grid, 256, 0, s>>>(V, rows, g_warp_thr, g_cta_thr, cnt, w->heavy.as<uint32_t>(), w->n_warp,
                                            cta_rows.as<uint4>());
  OGB_CUDA(cudaGetLastError());
  std::vector<uint4> cr(w->n_cta);
  if (w->n_cta) OGB_CUDA(cudaMemcpyAsync(cr.data(), cta_rows.p, (size_t)w->n_cta * 16, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  std::vector<PrChunkItem> items;
  std::vector<uint32_t> first(w->n_cta), count(w->n_cta);
  for (uint32_t k = 0; k < w->n_cta; k++) {
    const uint32_t v = cr[k].x, a = cr[k].y, d = cr[k].z;
    first[k] = (uint32_t)items.size();
    for (uint32_t c = 0; c < d; c += kPrChunk) items.push_back({v, a + c, a + std::min(d, c + kPrChunk), k});
    count[k] = (uint32_t)items.size() - first[k];
  }
  w->n_chunks = (uint32_t)items.size();
  OGB_TRY(w->chunks.alloc(items.size() * sizeof(PrChunkItem) + 16));
  OGB_TRY(w->partials.alloc(items.size() * 4 + 16));
  OGB_TRY(w->vfirst.alloc((size_t)w->n_cta * 4 + 16));
  OGB_TRY(w->vcount.alloc((size_t)w->n_cta * 4 + 16));
  OGB_TRY(w->done.alloc((size_t)w->n_cta * 4 + 16));
  if (!items.empty()) {
    OGB_CUDA(cudaMemcpyAsync(w->chunks.p, items.data(), items.size() * sizeof(PrChunkItem), cudaMemcpyHostToDevice, s));
    OGB_CUDA(cudaMemcpyAsync(w->vfirst.p, first.data(), first.size() * 4, cudaMemcpyHostToDevice, s));
    OGB_CUDA(cudaMemcpyAsync(w->vcount.p, count.data(), count.size() * 4, cudaMemcpyHostToDevice, s));
  }
  OGB_CUDA(cudaMemsetAsync(w->done.p, 0, (size_t)w->n_cta * 4 + 16, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

// Re-laid pull graph (once per graph, warp_thr and cta_thr): ids sorted by
// descending out-degree (stable: ties by id), perm = old -> new; the inverse
// neighbour array copied with renumbered ids into light | medium | chunked
// classes, each contiguous in vertex order; rows_rl = {new offset,
// in-degree}; off_light = offsets of the light rows (V + 1 entries, other
// rows empty); the medium row list (med_v, med_off) and its units.
static int pr_build_relabel(DevGraph& g, PrWork* w, cudaStream_t s) {
  const uint32_t V = g.V, E = g.E;
  const size_t Vp = ((size_t)V + 8) & ~(size_t)3;  // words per V + 1 array, padded
  OGB_TRY(w->perm.alloc((size_t)V * 4 + 16));
  OGB_TRY(w->nbr_rl.alloc((size_t)E * 4 + 16));
  OGB_TRY(w->rows_rl.alloc((size_t)V * 8 + 16));
  OGB_TRY(w->off_light.alloc(Vp * 4));
  OGB_TRY(w->rl_tmp.alloc((Vp * 8 + scan_tmp_words(V)) * 4));
  const int grid = sm_count() * 8;
  uint32_t* t0 = w->rl_tmp.as<uint32_t>();
  uint32_t* a[8];
  for (int i = 0; i < 8; i++) a[i] = t0 + i * Vp;
  uint32_t* scan_tmp = t0 + 8 * Vp;
  // sort ids by ~out_degree: a0 keys, a1 ids -> a2 sorted keys, a3 order
  pr_rl_keys_kernel<<<grid, 256, 0, s>>>(V, g.fwd.d_out_degree(), a[0], a[1]);
  OGB_CUDA(cudaGetLastError());
  KV in{a[0], a[1], nullptr};
  KV out{a[2], a[3], nullptr};
  OGB_TRY(sort_pairs(in, out, V, g.sort_ws, s));
  pr_rl_perm_kernel<<<grid, 256, 0, s>>>(V, a[3], w->perm.as<uint32_t>());
  // classes: a0 light, a1 medium, a2 chunked lengths, a3 medium flags; scans
  // into off_light, a4, a5, a6
  pr_rl_split_kernel<<<grid, 256, 0, s>>>(V, g.inv.d_rows(), g_warp_thr, g_cta_thr, a[0], a[1], a[2], a[3]);
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(scan_exclusive_u32(a[0], w->off_light.as<uint32_t>(), V, scan_tmp, s));
  OGB_TRY(scan_exclusive_u32(a[1], a[4], V, scan_tmp, s));
  OGB_TRY(scan_exclusive_u32(a[2], a[5], V, scan_tmp, s));
  OGB_TRY(scan_exclusive_u32(a[3], a[6], V, scan_tmp, s));
  uint32_t tot[3];
  OGB_CUDA(cudaMemcpyAsync(&tot[0], w->off_light.as<uint32_t>() + V, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(&tot[1], a[4] + V, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(&tot[2], a[6] + V, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  w->med_base = tot[0];
  w->n_med = tot[2];
  w->n_units = ceil_div(tot[1], kUnit);
  OGB_TRY(w->med_v.alloc((size_t)w->n_med * 4 + 16));
  OGB_TRY(w->med_off.alloc((size_t)w->n_med * 4 + 16));
  OGB_TRY(w->unit_first.alloc((size_t)w->n_units * 4 + 16));
  pr_rl_rows_kernel<<<grid, 256, 0, s>>>(V, g.inv.d_rows(), g_warp_thr, g_cta_thr, w->off_light.as<uint32_t>(), a[4],
                                         a[5], a[6], w->rows_rl.as<uint2>(), w->med_v.as<uint32_t>(),
                                         w->med_off.as<uint32_t>());
  pr_rl_units_kernel<<<grid, 256, 0, s>>>(w->n_units, w->med_off.as<uint32_t>(), w->n_med,
                                          w->unit_first.as<uint32_t>());
  pr_rl_copy_kernel<<<grid, 256, 0, s>>>(V, g.inv.d_rows(), g.inv.d_dst(), w->rows_rl.as<uint2>(),
                                         w->perm.as<uint32_t>(), w->nbr_rl.as<uint32_t>());
  OGB_CUDA(cudaGetLastError());
  int dev = 0, optin = 0;
  OGB_CUDA(cudaGetDevice(&dev));
  OGB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  OGB_CUDA(cudaFuncGetAttributes(&fa, pr_pull_kernel));
  const size_t room = (size_t)optin - fa.sharedSizeBytes - kPullDynSmem - 1024;  // and a margin
  const uint32_t vcap = (V + 3) & ~3u;  // contrib buffers hold V + 4 floats
  w->hot = std::min<uint32_t>(kHotLimit & ~3u, (uint32_t)std::min<size_t>(vcap, (room / 16) * 4));
  const size_t smem = kPullDynSmem + (size_t)w->hot * 4;
  OGB_CUDA(cudaFuncSetAttribute(pr_pull_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // the rest of the SM's unified L1 / shared memory stays L1: the gathers of
  // the highest-degree sources hit there
  int smem_per_sm = 0;
  OGB_CUDA(cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  const int pct = (int)std::min<size_t>(100, ((smem + fa.sharedSizeBytes + 2048) * 100 + smem_per_sm - 1) / smem_per_sm);
  OGB_CUDA(cudaFuncSetAttribute(pr_pull_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

// Push preparation (once per graph): the filtered forward CSR without the
// out-edges into hubs, and the hub chunk table.
static int pr_build_push(DevGraph& g, PrWork* w, cudaStream_t s) {
  const uint32_t V = g.V, E = g.E;
  const size_t Ep = ((size_t)E + 8) & ~(size_t)3;  // words per E + 1 array, padded
  const size_t Vp = ((size_t)V + 8) & ~(size_t)3;
  DevBuf tmp;
  OGB_TRY(tmp.alloc((2 * std::max(Ep, Vp) + scan_tmp_words(std::max(E, V))) * 4));
  uint32_t* flag = tmp.as<uint32_t>();
  uint32_t* pos = flag + std::max(Ep, Vp);
  uint32_t* scan_tmp = pos + std::max(Ep, Vp);
  const int grid = sm_count() * 8;
  pr_push_flag_kernel<<<grid, 256, 0, s>>>(E, g.fwd.d_dst(), g.inv.d_rows(), kPushHubDeg, flag);
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(scan_exclusive_u32(flag, pos, E, scan_tmp, s));
  uint32_t n_fp = 0;
  OGB_CUDA(cudaMemcpyAsync(&n_fp, pos + E, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  OGB_TRY(w->rows_fp.alloc((size_t)V * 8 + 16));
  OGB_TRY(w->nbr_fp.alloc((size_t)n_fp * 4 + 16));
  pr_push_compact_kernel<<<grid, 256, 0, s>>>(E, g.fwd.d_dst(), flag, pos, w->nbr_fp.as<uint32_t>());
  pr_push_rows_kernel<<<grid, 256, 0, s>>>(V, g.fwd.d_rows(), pos, w->rows_fp.as<uint2>());
  // hub chunks (flag / pos reused as V + 1 arrays)
  pr_hub_count_kernel<<<grid, 256, 0, s>>>(V, g.inv.d_rows(), kPushHubDeg, flag);
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(scan_exclusive_u32(flag, pos, V, scan_tmp, s));
  uint32_t n_items = 0;
  OGB_CUDA(cudaMemcpyAsync(&n_items, pos + V, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  OGB_TRY(w->hub_items.alloc((size_t)n_items * 16 + 16));
  pr_hub_fill_kernel<<<grid, 256, 0, s>>>(V, g.inv.d_rows(), kPushHubDeg, pos, w->hub_items.as<uint4>());
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaStreamSynchronize(s));  // before the scratch is released
  w->n_hub_items = n_items;
  return OK;
}

static int pr_work_get(DevGraph& g, bool pull, PrWork** out, cudaStream_t s) {
  if (!g.pr) g.pr = new PrWork();
  PrWork* w = g.pr;
  const uint32_t V = g.V;
  if (w->V != V || !w->contrib0.p) {
    OGB_TRY(w->contrib0.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->contrib1.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->next.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->heavy.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->ctl.alloc(sizeof(PrCtl) + 64));
    w->V = V;
    w->listed_pull = -1;
  }
  if (!w->h_ctl) OGB_CUDA(cudaMallocHost(&w->h_ctl, sizeof(PrCtl)));
  if (!w->ev0) {
    OGB_CUDA(cudaEventCreate(&w->ev0));
    OGB_CUDA(cudaEventCreate(&w->ev1));
  }
  const int want = pull ? 1 : 0;
  if (pull && (!w->rl_ready || w->rl_build != g.build_id || w->rl_warp != g_warp_thr || w->rl_cta != g_cta_thr)) {
    OGB_TRY(pr_build_relabel(g, w, s));
    w->rl_ready = true;
    w->rl_build = g.build_id;
    w->rl_warp = g_warp_thr;
    w->rl_cta = g_cta_thr;
    w->listed_pull = -1;
  }
  if (!pull && (!w->push_ready || w->push_build != g.build_id)) {
    OGB_TRY(pr_build_push(g, w, s));
    w->push_ready = true;
    w->push_build = g.build_id;
    w->listed_pull = -1;
  }
  if (w->listed_pull != want || w->listed_warp != g_warp_thr || w->listed_cta != g_cta_thr ||
      w->listed_build != g.build_id) {
    OGB_TRY(pr_build_lists(g, w, pull, s));
    w->listed_pull = want;
    w->listed_warp = g_warp_thr;
    w->listed_cta = g_cta_thr;
    w->listed_build = g.build_id;
  }
  *out = w;
  return OK;
}

int pagerank_run(DevGraph& g, uint32_t mode, uint32_t max_iters, double epsilon, float* ranks, const float* init,
                 PrResult* res, cudaStream_t s) {
  if (max_iters > kPrMaxIters) return fail(ERR_ARG, "pagerank: at most %u iterations", kPrMaxIters);
  const uint32_t V = g.V;
  if (V == 0) return fail(ERR_ARG, "pagerank: empty graph");
  const bool pull = mode == PR_PULL;
  PrWork* w = nullptr;
  OGB_TRY(pr_work_get(g, pull, &w, s));
  constexpr int T = kPrThreads;
  const int sms = sm_count();
  PrParams p;
  p.damp = 0.85f;
  p.base_pr = 1.0f - p.damp;
  p.epsilon = epsilon;
  p.V = V;
  p.warp_thr = g_warp_thr;
  p.gid = nullptr;
  p.frozen = nullptr;
  p.delta = nullptr;
  PrCtl* d_ctl = w->ctl.as<PrCtl>();
  OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(PrCtl), s));
  float* c_cur = w->contrib0.as<float>();
  float* c_nxt = w->contrib1.as<float>();
  float* nxt = w->next.as<float>();
  const uint32_t* perm = pull ? w->perm.as<uint32_t>() : nullptr;
  pr_init_kernel<<<sms * 8, 256, 0, s>>>(V, g.fwd.d_out_degree(), init, p.base_pr, ranks, c_cur, pull ? nullptr : nxt,
                                         perm);
  OGB_CUDA(cudaGetLastError());

  const uint32_t nb_chunk = w->n_chunks ? std::min<uint32_t>(sms * 4, w->n_chunks) : 0;
  const uint32_t nb_warp = w->n_warp ? std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(w->n_warp, T / 32))) : 0;
  const uint32_t nb_light = std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(V, T)));
  const uint32_t nb_hub = (!pull && w->n_hub_items)
                              ? std::min<uint32_t>(sms * 4, ceil_div(w->n_hub_items, T / 32)) : 0;
  const uint32_t grid = nb_hub + nb_chunk + nb_warp + nb_light;
  const uint2* rows = pull ? g.inv.d_rows() : w->rows_fp.as<uint2>();
  const uint32_t* nbr = pull ? g.inv.d_dst() : w->nbr_fp.as<uint32_t>();
  const uint32_t* heavy = w->heavy.as<uint32_t>();
  const PrChunkItem* chunks = w->chunks.as<PrChunkItem>();

  OGB_CUDA(cudaEventRecord(w->ev0, s));
  for (uint32_t it = 0; it < max_iters; it++) {
    if (pull) {
      pr_pull_kernel<<<sms, kPullThreads, kPullDynSmem + (size_t)w->hot * 4, s>>>(
          w->hot, chunks, w->n_chunks, w->vfirst.as<uint32_t>(), w->vcount.as<uint32_t>(), w->done.as<uint32_t>(),
          w->partials.as<float>(), w->rows_rl.as<uint2>(), w->off_light.as<uint32_t>(), w->unit_first.as<uint32_t>(),
          w->n_units, w->med_off.as<uint32_t>(), w->med_v.as<uint32_t>(), w->med_base, w->nbr_rl.as<uint32_t>(),
          g.fwd.d_out_degree(), perm, c_cur, c_nxt, ranks, p, d_ctl, it);
    } else {
      pr_push_scatter_kernel<<<grid, T, 0, s>>>(nb_hub, w->hub_items.as<uint4>(), w->n_hub_items, g.inv.d_dst(),
                                                 nb_chunk, nb_warp, heavy, w->n_warp, chunks, w->n_chunks, V,
                                                 g_warp_thr, rows, nbr, c_cur, nxt, d_ctl);
      pr_push_update_kernel<<<sms * 8, T, 0, s>>>(V, g.fwd.d_out_degree(), nxt, c_nxt, ranks, p, d_ctl, it);
    }
    OGB_CUDA(cudaGetLastError());
    std::swap(c_cur, c_nxt);
  }
  pr_normalize_kernel<<<sms * 8, 256, 0, s>>>(V, ranks);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaEventRecord(w->ev1, s));
  OGB_CUDA(cudaMemcpyAsync(w->h_ctl, d_ctl, sizeof(PrCtl), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&ms, w->ev0, w->ev1));
  PrResult r;
  r.ms = ms;
  r.launches = 2 + max_iters * (pull ? 1 : 2);
  if (w->h_ctl->stop) {
    r.converged = 1;
    r.iterations = w->h_ctl->stop_iter;
    r.executed = w->h_ctl->stop_iter + 1;
  } else {
    r.iterations = max_iters;
    r.executed = max_iters;
  }
  for (uint32_t i = 0; i < r.executed && i < 1024; i++) {
    r.err_hist[i] = w->h_ctl->err[i];
    r.active_hist[i] = w->h_ctl->active[i];
  }
  if (r.executed) {
    r.error_total = w->h_ctl->err[r.executed - 1];
    r.activeVertices = w->h_ctl->active[r.executed - 1];
  }
  if (res) *res = r;
  return OK;
}

// ------------------------------------------------------------ many graphs ---

// Per-graph error and stop rule of one iteration over a disjoint union: a
// CTA per graph sums |change| / V_g (fp64) and counts the vertices that
// changed by >= epsilon; a graph with none stops (its vertices keep their
// rank from then on), as the reference's loop breaks (pageRank.c:1024-1033).
__global__ void __launch_bounds__(256) prk_batch_reduce(PrBatchDev b, double eps, uint32_t it) {
  __shared__ double s_e[8];
  __shared__ uint32_t s_a[8];
  const uint32_t gph = blockIdx.x;
  if (b.frozen[gph]) return;
  const uint32_t lo = b.voff[gph], hi = b.voff[gph + 1];
  const double n = (double)(hi - lo);
  double e = 0.0;
  uint32_t a = 0;
  for (uint32_t v = lo + threadIdx.x; v < hi; v += blockDim.x) {
    const double d = fabs((double)b.delta[v]);
    e += d / n;
    a += (d >= eps) ? 1u : 0u;
  }
  for (int o = 16; o; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    a += __shfl_down_sync(0xffffffffu, a, o);
  }
  if (lane_id() == 0) {
    s_e[threadIdx.x >> 5] = e;
    s_a[threadIdx.x >> 5] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double te = 0.0;
    uint32_t ta = 0;
    for (int w = 0; w < 8; w++) {
      te += s_e[w];
      ta += s_a[w];
    }
    b.err_last[gph] = te;
    b.active_last[gph] = ta;
    b.executed[gph] = it + 1;
    if (ta == 0) {
      b.frozen[gph] = 1;
      b.stop_iter[gph] = it;
    }
  }
}

// pr /= V of the vertex's own graph (pageRank.c:1049-1052)
__global__ void prk_batch_normalize(uint32_t V, PrBatchDev b, float* __restrict__ pr) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t gph = b.gid[v];
    pr[v] = __fdiv_rn(pr[v], (float)(b.voff[gph + 1] - b.voff[gph]));
  }
}

// PageRank pull over a disjoint union of graphs, every graph with its own
// stop rule and normalization; the results equal single-graph runs (same
// rows, same summation orders).  The whole run -- init, the iterations,
// the per-graph reductions and the normalization -- is captured once into a
// CUDA graph (cached in *exec for the same arguments) and launched as one.
int pagerank_batch_run(DevGraph& g, const PrBatchDev& b, uint32_t ngraphs, uint32_t max_iters, double epsilon,
                       float* ranks, cudaGraphExec_t* exec, bool* rebuilt, cudaStream_t s) {
  if (max_iters > kPrMaxIters) return fail(ERR_ARG, "pagerank: at most %u iterations", kPrMaxIters);
  const uint32_t V = g.V;
  if (V == 0) return fail(ERR_ARG, "pagerank: empty graph");
  PrWork* w = nullptr;
  OGB_TRY(pr_work_get(g, true, &w, s));
  if (rebuilt) *rebuilt = false;
  if (!*exec) {
    const int sms = sm_count();
    PrParams p;
    p.damp = 0.85f;
    p.base_pr = 1.0f - p.damp;
    p.epsilon = epsilon;
    p.V = V;
    p.warp_thr = g_warp_thr;
    p.gid = b.gid;
    p.frozen = b.frozen;
    p.delta = b.delta;
    PrCtl* d_ctl = w->ctl.as<PrCtl>();
    float* c_cur = w->contrib0.as<float>();
    float* c_nxt = w->contrib1.as<float>();
    const uint32_t* perm = w->perm.as<uint32_t>();
    cudaStream_t cs = nullptr;
    OGB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaMemsetAsync(d_ctl, 0, sizeof(PrCtl), cs);
      cudaMemsetAsync(b.frozen, 0, (size_t)ngraphs * 4, cs);
      cudaMemsetAsync(b.stop_iter, 0xFF, (size_t)ngraphs * 4, cs);
      cudaMemsetAsync(b.executed, 0, (size_t)ngraphs * 4, cs);
      pr_init_kernel<<<sms * 8, 256, 0, cs>>>(V, g.fwd.d_out_degree(), nullptr, p.base_pr, ranks, c_cur, nullptr, perm);
      for (uint32_t it = 0; it < max_iters; it++) {
        pr_pull_kernel<<<sms, kPullThreads, kPullDynSmem + (size_t)w->hot * 4, cs>>>(
            w->hot, w->chunks.as<PrChunkItem>(), w->n_chunks, w->vfirst.as<uint32_t>(), w->vcount.as<uint32_t>(),
            w->done.as<uint32_t>(), w->partials.as<float>(), w->rows_rl.as<uint2>(), w->off_light.as<uint32_t>(),
            w->unit_first.as<uint32_t>(), w->n_units, w->med_off.as<uint32_t>(), w->med_v.as<uint32_t>(),
            w->med_base, w->nbr_rl.as<uint32_t>(), g.fwd.d_out_degree(), perm, c_cur, c_nxt, ranks, p, d_ctl, it);
        prk_batch_reduce<<<ngraphs, 256, 0, cs>>>(b, epsilon, it);
        std::swap(c_cur, c_nxt);
      }
      prk_batch_normalize<<<sms * 8, 256, 0, cs>>>(V, b, ranks);
      e = cudaStreamEndCapture(cs, &graph);
    }
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return fail(ERR_CUDA, "pagerank batch capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ERR_CUDA, "pagerank batch instantiate: %s", cudaGetErrorString(e));
    if (rebuilt) *rebuilt = true;
  }
  OGB_CUDA(cudaGraphLaunch(*exec, s));
  return OK;
}

}  // namespace ogb
