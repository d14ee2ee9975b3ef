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
// Chunk CTAs come first in the grid, then warp rows, then light rows, so the
// long-latency work starts first.  Iterations are launched back to back
// without host round trips: each iteration's last CTA records error/active
// and, when active == 0, sets a stop flag that later launches read first.
#include "graph.cuh"

#include <algorithm>
#include <vector>

namespace ogb {

constexpr uint32_t kPrMaxIters = 1024;
constexpr int kPrThreads = 256;
constexpr uint32_t kPrChunk = 8192;  // edges per chunk of a very heavy row

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
  *cta_threads = kPrThreads;
  *chunk = kPrChunk;
}

struct PrCtl {
  double err[kPrMaxIters];
  uint32_t active[kPrMaxIters];
  uint32_t blocks_done[kPrMaxIters];
  uint32_t stop;       // 1 once an iteration ended with no active vertex
  uint32_t stop_iter;  // index of that iteration
};

struct PrChunkItem {
  uint32_t v, j0, j1, k;  // vertex, edge range, index of the vertex in the chunked list
};

struct PrWork {
  uint32_t V = 0;
  int listed_pull = -1;                // direction the lists describe
  uint32_t listed_warp = 0, listed_cta = 0;
  DevBuf contrib0, contrib1, next, ctl;
  DevBuf heavy;                        // vertex ids of the warp rows (n_warp), then the chunked rows
  DevBuf chunks;                       // PrChunkItem per chunk
  DevBuf vfirst, vcount, done;         // per chunked vertex: first chunk, chunk count, finished chunks
  DevBuf partials;                     // float per chunk
  uint32_t n_warp = 0, n_cta = 0, n_chunks = 0;
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
};

__device__ __forceinline__ void pr_update(uint32_t v, float s, float* __restrict__ pr,
                                          const uint32_t* __restrict__ out_degree,
                                          float* __restrict__ contrib_next, const PrParams& p, double& err,
                                          uint32_t& active) {
  const float nv = __fadd_rn(p.base_pr, __fmul_rn(p.damp, s));
  const float prev = pr[v];
  pr[v] = nv;
  const uint32_t d = out_degree[v];
  contrib_next[v] = d ? __fdiv_rn(nv, (float)d) : 0.0f;
  const double e = fabs((double)__fsub_rn(nv, prev));
  err += e / (double)p.V;
  active += (e >= p.epsilon) ? 1u : 0u;
}

__device__ __forceinline__ void pr_block_finish(double err, uint32_t active, PrCtl* ctl, uint32_t it) {
  __shared__ double s_err[kPrThreads / 32];
  __shared__ uint32_t s_act[kPrThreads / 32];
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
    for (int w = 0; w < kPrThreads / 32; w++) {
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

// s += c[nbr[j]] for j = j0, j0+STRIDE, ... < j1, in that order, with four
// gathers in flight.
template <uint32_t STRIDE>
__device__ __forceinline__ float strided_sum(const float* __restrict__ c, const uint32_t* __restrict__ nbr,
                                             uint32_t j0, uint32_t j1) {
  float s = 0.0f;
  uint32_t j = j0;
  for (; j + 3 * STRIDE < j1; j += 4 * STRIDE) {
    const uint32_t a = nbr[j] & 0x3FFFFFFFu, b = nbr[j + STRIDE] & 0x3FFFFFFFu;
    const uint32_t d = nbr[j + 2 * STRIDE] & 0x3FFFFFFFu, e = nbr[j + 3 * STRIDE] & 0x3FFFFFFFu;
    const float ca = c[a], cb = c[b], cd = c[d], ce = c[e];
    s = __fadd_rn(s, ca);
    s = __fadd_rn(s, cb);
    s = __fadd_rn(s, cd);
    s = __fadd_rn(s, ce);
  }
  for (; j < j1; j += STRIDE) s = __fadd_rn(s, c[nbr[j] & 0x3FFFFFFFu]);
  return s;
}

__device__ __forceinline__ float warp_fold(float s) {
#pragma unroll
  for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
}

// Two strided sums at once (rows A and B of one warp), each in the order of
// strided_sum<32>: eight gathers in flight per lane instead of four.
__device__ __forceinline__ void strided_sum2(const float* __restrict__ c, const uint32_t* __restrict__ nbr,
                                             uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1, float& sa,
                                             float& sb) {
  constexpr uint32_t S = 32;
  sa = 0.0f;
  sb = 0.0f;
  uint32_t ja = a0, jb = b0;
  while (ja + 3 * S < a1 && jb + 3 * S < b1) {
    const uint32_t x0 = nbr[ja] & 0x3FFFFFFFu, x1 = nbr[ja + S] & 0x3FFFFFFFu;
    const uint32_t x2 = nbr[ja + 2 * S] & 0x3FFFFFFFu, x3 = nbr[ja + 3 * S] & 0x3FFFFFFFu;
    const uint32_t y0 = nbr[jb] & 0x3FFFFFFFu, y1 = nbr[jb + S] & 0x3FFFFFFFu;
    const uint32_t y2 = nbr[jb + 2 * S] & 0x3FFFFFFFu, y3 = nbr[jb + 3 * S] & 0x3FFFFFFFu;
    const float cx0 = c[x0], cx1 = c[x1], cx2 = c[x2], cx3 = c[x3];
    const float cy0 = c[y0], cy1 = c[y1], cy2 = c[y2], cy3 = c[y3];
    sa = __fadd_rn(sa, cx0);
    sa = __fadd_rn(sa, cx1);
    sa = __fadd_rn(sa, cx2);
    sa = __fadd_rn(sa, cx3);
    sb = __fadd_rn(sb, cy0);
    sb = __fadd_rn(sb, cy1);
    sb = __fadd_rn(sb, cy2);
    sb = __fadd_rn(sb, cy3);
    ja += 4 * S;
    jb += 4 * S;
  }
  // tails, each in its own order (identical to continuing strided_sum<32>)
  for (; ja + 3 * S < a1; ja += 4 * S) {
    const uint32_t x0 = nbr[ja] & 0x3FFFFFFFu, x1 = nbr[ja + S] & 0x3FFFFFFFu;
    const uint32_t x2 = nbr[ja + 2 * S] & 0x3FFFFFFFu, x3 = nbr[ja + 3 * S] & 0x3FFFFFFFu;
    const float cx0 = c[x0], cx1 = c[x1], cx2 = c[x2], cx3 = c[x3];
    sa = __fadd_rn(sa, cx0);
    sa = __fadd_rn(sa, cx1);
    sa = __fadd_rn(sa, cx2);
    sa = __fadd_rn(sa, cx3);
  }
  for (; jb + 3 * S < b1; jb += 4 * S) {
    const uint32_t y0 = nbr[jb] & 0x3FFFFFFFu, y1 = nbr[jb + S] & 0x3FFFFFFFu;
    const uint32_t y2 = nbr[jb + 2 * S] & 0x3FFFFFFFu, y3 = nbr[jb + 3 * S] & 0x3FFFFFFFu;
    const float cy0 = c[y0], cy1 = c[y1], cy2 = c[y2], cy3 = c[y3];
    sb = __fadd_rn(sb, cy0);
    sb = __fadd_rn(sb, cy1);
    sb = __fadd_rn(sb, cy2);
    sb = __fadd_rn(sb, cy3);
  }
  for (; ja < a1; ja += S) sa = __fadd_rn(sa, c[nbr[ja] & 0x3FFFFFFFu]);
  for (; jb < b1; jb += S) sb = __fadd_rn(sb, c[nbr[jb] & 0x3FFFFFFFu]);
}

// Pull iteration, one grid: blocks [0, nb_chunk) reduce chunks of very heavy
// rows, the next nb_warp blocks the warp rows, the rest walk all vertices in
// order and take the light rows.
__global__ void __launch_bounds__(kPrThreads) pr_pull_kernel(
    uint32_t nb_chunk, uint32_t nb_warp, const uint32_t* __restrict__ heavy, uint32_t n_warp,
    const PrChunkItem* __restrict__ chunks, uint32_t n_chunks, const uint32_t* __restrict__ vfirst,
    const uint32_t* __restrict__ vcount, uint32_t* __restrict__ done, float* __restrict__ partials,
    const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ out_degree,
    const float* __restrict__ contrib, float* __restrict__ contrib_next, float* __restrict__ pr, PrParams p,
    PrCtl* __restrict__ ctl, uint32_t it) {
  __shared__ float s_part[kPrThreads / 32];
  __shared__ uint32_t s_last;
  if (ctl->stop) return;
  double err = 0.0;
  uint32_t active = 0;
  const uint32_t b = blockIdx.x;
  if (b < nb_chunk) {
    for (uint32_t g = b; g < n_chunks; g += nb_chunk) {
      const PrChunkItem ci = chunks[g];
      float s = strided_sum<kPrThreads>(contrib, nbr, ci.j0 + threadIdx.x, ci.j1);
      s = warp_fold(s);
      if (lane_id() == 0) s_part[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int w = 0; w < kPrThreads / 32; w++) tot = __fadd_rn(tot, s_part[w]);
        partials[g] = tot;
        __threadfence();
        const uint32_t cnt = vcount[ci.k];
        s_last = (atomicAdd(&done[ci.k], 1u) == cnt - 1) ? 1u : 0u;
        if (s_last) {
          __threadfence();
          const uint32_t f = vfirst[ci.k];
          float sum = 0.0f;
          for (uint32_t c = 0; c < cnt; c++) sum = __fadd_rn(sum, __ldcg(&partials[f + c]));
          done[ci.k] = 0;
          pr_update(ci.v, sum, pr, out_degree, contrib_next, p, err, active);
        }
      }
      __syncthreads();
    }
  } else if (b < nb_chunk + nb_warp) {
    // a warp reduces two rows at a time (t and t + wstride)
    const uint32_t lane = lane_id();
    const uint32_t w0 = (b - nb_chunk) * (kPrThreads / 32) + (threadIdx.x >> 5);
    const uint32_t wstride = nb_warp * (kPrThreads / 32);
    for (uint32_t t = w0; t < n_warp; t += 2 * wstride) {
      const uint32_t va = heavy[t];
      const bool has_b = t + wstride < n_warp;
      const uint32_t vb = has_b ? heavy[t + wstride] : va;
      const uint2 ra = rows[va];
      const uint2 rb = has_b ? rows[vb] : make_uint2(0, 0);
      float sa, sb;
      strided_sum2(contrib, nbr, ra.x + lane, ra.x + ra.y, rb.x + lane, rb.x + rb.y, sa, sb);
      sa = warp_fold(sa);
      sb = warp_fold(sb);
      if (lane == 0) {
        pr_update(va, sa, pr, out_degree, contrib_next, p, err, active);
        if (has_b) pr_update(vb, sb, pr, out_degree, contrib_next, p, err, active);
      }
    }
  } else {
    // light rows: a warp takes 128 consecutive vertices, each lane four rows
    // (lane, lane+32, lane+64, lane+96) reduced side by side, every row
    // sequentially in CSR order from 0.0f
    constexpr int R = 4;
    const uint32_t lane = lane_id();
    const uint32_t lw = (b - nb_chunk - nb_warp) * (kPrThreads / 32) + (threadIdx.x >> 5);
    const uint32_t nlw = (gridDim.x - nb_chunk - nb_warp) * (kPrThreads / 32);
    for (uint32_t base = lw * (32 * R); base < p.V; base += nlw * (32 * R)) {
      uint32_t a[R], d[R], dmax = 0;
      float s[R];
#pragma unroll
      for (int k = 0; k < R; k++) {
        const uint32_t v = base + k * 32 + lane;
        const uint2 r = (v < p.V) ? rows[v] : make_uint2(0, 0);
        a[k] = r.x;
        d[k] = (v < p.V && r.y <= p.warp_thr) ? r.y : 0u;
        s[k] = 0.0f;
        dmax = max(dmax, d[k]);
      }
      for (uint32_t i = 0; i < dmax; i++) {
        uint32_t u[R];
#pragma unroll
        for (int k = 0; k < R; k++) u[k] = (i < d[k]) ? (nbr[a[k] + i] & 0x3FFFFFFFu) : 0u;
        float c[R];
#pragma unroll
        for (int k = 0; k < R; k++) c[k] = (i < d[k]) ? contrib[u[k]] : 0.0f;
#pragma unroll
        for (int k = 0; k < R; k++)
          if (i < d[k]) s[k] = __fadd_rn(s[k], c[k]);
      }
#pragma unroll
      for (int k = 0; k < R; k++) {
        const uint32_t v = base + k * 32 + lane;
        if (v < p.V && rows[v].y <= p.warp_thr) pr_update(v, s[k], pr, out_degree, contrib_next, p, err, active);
      }
    }
  }
  pr_block_finish(err, active, ctl, it);
}

// Push scatter: contrib of each source added to its out-neighbours, split by
// out-degree like the pull gather (chunks scatter their edge range).
__global__ void __launch_bounds__(kPrThreads) pr_push_scatter_kernel(
    uint32_t nb_chunk, uint32_t nb_warp, const uint32_t* __restrict__ heavy, uint32_t n_warp,
    const PrChunkItem* __restrict__ chunks, uint32_t n_chunks, uint32_t V, uint32_t warp_thr,
    const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr, const float* __restrict__ contrib,
    float* __restrict__ next, const PrCtl* __restrict__ ctl) {
  if (ctl->stop) return;
  const uint32_t b = blockIdx.x;
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
    const uint32_t nlb = gridDim.x - nb_chunk - nb_warp;
    for (uint32_t v = lb * kPrThreads + threadIdx.x; v < V; v += nlb * kPrThreads) {
      const uint2 row = rows[v];
      if (row.y > warp_thr) continue;
      const float c = contrib[v];
      for (uint32_t j = row.x; j < row.x + row.y; j++) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  }
}

__global__ void __launch_bounds__(kPrThreads) pr_push_update_kernel(uint32_t V, const uint32_t* __restrict__ out_degree,
                                                                    float* __restrict__ next,
                                                                    float* __restrict__ contrib_next,
                                                                    float* __restrict__ pr, PrParams p,
                                                                    PrCtl* __restrict__ ctl, uint32_t it) {
  if (ctl->stop) return;
  double err = 0.0;
  uint32_t active = 0;
  for (uint32_t v = blockIdx.x * kPrThreads + threadIdx.x; v < V; v += gridDim.x * kPrThreads) {
    const float s = next[v];
    next[v] = 0.0f;
    pr_update(v, s, pr, out_degree, contrib_next, p, err, active);
  }
  pr_block_finish(err, active, ctl, it);
}

__global__ void pr_init_kernel(uint32_t V, const uint32_t* __restrict__ out_degree, const float* __restrict__ init,
                               float base_pr, float* __restrict__ pr, float* __restrict__ contrib,
                               float* __restrict__ next) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const float x = init ? init[v] : base_pr;
    pr[v] = x;
    const uint32_t d = out_degree[v];
    contrib[v] = d ? __fdiv_rn(x, (float)d) : 0.0f;
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
static int pr_build_lists(DevGraph& g, PrWork* w, bool pull, cudaStream_t s) {
  const uint32_t V = g.V;
  const uint2* rows = pull ? g.inv.d_rows() : g.fwd.d_rows();
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
  if (w->listed_pull != want || w->listed_warp != g_warp_thr || w->listed_cta != g_cta_thr) {
    OGB_TRY(pr_build_lists(g, w, pull, s));
    w->listed_pull = want;
    w->listed_warp = g_warp_thr;
    w->listed_cta = g_cta_thr;
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
  PrCtl* d_ctl = w->ctl.as<PrCtl>();
  OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(PrCtl), s));
  float* c_cur = w->contrib0.as<float>();
  float* c_nxt = w->contrib1.as<float>();
  float* nxt = w->next.as<float>();
  pr_init_kernel<<<sms * 8, 256, 0, s>>>(V, g.fwd.d_out_degree(), init, p.base_pr, ranks, c_cur, pull ? nullptr : nxt);
  OGB_CUDA(cudaGetLastError());

  const uint32_t nb_chunk = w->n_chunks ? std::min<uint32_t>(sms * 4, w->n_chunks) : 0;
  const uint32_t nb_warp = w->n_warp ? std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(w->n_warp, T / 32))) : 0;
  const uint32_t nb_light = std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(V, T)));
  const uint32_t grid = nb_chunk + nb_warp + nb_light;
  const uint2* rows = pull ? g.inv.d_rows() : g.fwd.d_rows();
  const uint32_t* nbr = pull ? g.inv.d_dst() : g.fwd.d_dst();
  const uint32_t* heavy = w->heavy.as<uint32_t>();
  const PrChunkItem* chunks = w->chunks.as<PrChunkItem>();

  OGB_CUDA(cudaEventRecord(w->ev0, s));
  for (uint32_t it = 0; it < max_iters; it++) {
    if (pull) {
      pr_pull_kernel<<<grid, T, 0, s>>>(nb_chunk, nb_warp, heavy, w->n_warp, chunks, w->n_chunks,
                                         w->vfirst.as<uint32_t>(), w->vcount.as<uint32_t>(), w->done.as<uint32_t>(),
                                         w->partials.as<float>(), rows, nbr, g.fwd.d_out_degree(), c_cur, c_nxt,
                                         ranks, p, d_ctl, it);
    } else {
      pr_push_scatter_kernel<<<grid, T, 0, s>>>(nb_chunk, nb_warp, heavy, w->n_warp, chunks, w->n_chunks, V,
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

}  // namespace ogb
