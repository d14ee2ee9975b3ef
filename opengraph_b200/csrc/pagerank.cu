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
//   heavy rows (> warp_thr): a warp per vertex, lanes strided over the row,
//     butterfly-folded; rows > cta_thr: a 256-thread CTA per vertex.
// The heavy lists are built once per graph and direction.  Iterations are
// launched back to back without host round trips: each iteration's last CTA
// records error/active and, when active == 0, sets a stop flag that later
// launches read first.
#include "graph.cuh"

#include <algorithm>
#include <vector>

namespace ogb {

constexpr uint32_t kPrMaxIters = 1024;
constexpr int kPrThreads = 256;

// Row-length thresholds of the work split (settable; the GPU-order mode of
// the oracle takes the same values).
static uint32_t g_warp_thr = 32;
static uint32_t g_cta_thr = 2048;

void pagerank_set_bins(uint32_t warp_thr, uint32_t cta_thr) {
  g_warp_thr = warp_thr;
  g_cta_thr = std::max(cta_thr, warp_thr);
}
void pagerank_get_bins(uint32_t* warp_thr, uint32_t* cta_thr, uint32_t* cta_threads) {
  *warp_thr = g_warp_thr;
  *cta_thr = g_cta_thr;
  *cta_threads = kPrThreads;
}

struct PrCtl {
  double err[kPrMaxIters];
  uint32_t active[kPrMaxIters];
  uint32_t blocks_done[kPrMaxIters];
  uint32_t stop;       // 1 once an iteration ended with no active vertex
  uint32_t stop_iter;  // index of that iteration
};

struct PrWork {
  uint32_t V = 0;
  int listed_pull = -1;                // direction the heavy lists describe
  uint32_t listed_warp = 0, listed_cta = 0;
  DevBuf contrib0, contrib1, next, ctl;
  DevBuf heavy;                        // vertex ids: [warp list | cta list]
  uint32_t n_warp = 0, n_cta = 0;
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

// Order inside a list does not change results: each heavy vertex is reduced
// by exactly one warp or CTA in a fixed order.
__global__ void pr_heavy_fill_kernel(uint32_t V, const uint2* __restrict__ rows, uint32_t warp_thr,
                                     uint32_t cta_thr, uint32_t* __restrict__ cursor, uint32_t* __restrict__ list,
                                     uint32_t off_cta) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    if (d > cta_thr)
      list[off_cta + atomicAdd(&cursor[1], 1u)] = v;
    else if (d > warp_thr)
      list[atomicAdd(&cursor[0], 1u)] = v;
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

// Sum of c[nbr[j]] over a row by the calling warp (lanes strided, butterfly).
__device__ __forceinline__ float warp_row_sum(const float* __restrict__ c, const uint32_t* __restrict__ nbr,
                                              uint2 row) {
  float s = 0.0f;
  for (uint32_t j = row.x + lane_id(); j < row.x + row.y; j += 32) s = __fadd_rn(s, c[nbr[j] & 0x3FFFFFFFu]);
#pragma unroll
  for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
}

// Pull iteration, one grid: blocks [0, nb_light) walk all vertices in order
// and take the light rows, the next nb_warp blocks the warp list, the rest
// the CTA list.
__global__ void __launch_bounds__(kPrThreads) pr_pull_kernel(
    uint32_t nb_light, uint32_t nb_warp, const uint32_t* __restrict__ heavy, uint32_t n_warp, uint32_t n_cta,
    const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr, const uint32_t* __restrict__ out_degree,
    const float* __restrict__ contrib, float* __restrict__ contrib_next, float* __restrict__ pr, PrParams p,
    PrCtl* __restrict__ ctl, uint32_t it) {
  if (ctl->stop) return;
  double err = 0.0;
  uint32_t active = 0;
  const uint32_t b = blockIdx.x;
  if (b < nb_light) {
    for (uint32_t v = b * kPrThreads + threadIdx.x; v < p.V; v += nb_light * kPrThreads) {
      const uint2 row = rows[v];
      if (row.y > p.warp_thr) continue;
      float s = 0.0f;
      for (uint32_t j = row.x; j < row.x + row.y; j++) s = __fadd_rn(s, contrib[nbr[j] & 0x3FFFFFFFu]);
      pr_update(v, s, pr, out_degree, contrib_next, p, err, active);
    }
  } else if (b < nb_light + nb_warp) {
    const uint32_t w0 = (b - nb_light) * (kPrThreads / 32) + (threadIdx.x >> 5);
    const uint32_t wstride = nb_warp * (kPrThreads / 32);
    for (uint32_t t = w0; t < n_warp; t += wstride) {
      const uint32_t v = heavy[t];
      const float s = warp_row_sum(contrib, nbr, rows[v]);
      if (lane_id() == 0) pr_update(v, s, pr, out_degree, contrib_next, p, err, active);
    }
  } else {
    __shared__ float s_part[kPrThreads / 32];
    const uint32_t cb = b - nb_light - nb_warp;
    const uint32_t ncb = gridDim.x - nb_light - nb_warp;
    for (uint32_t t = cb; t < n_cta; t += ncb) {
      const uint32_t v = heavy[n_warp + t];
      const uint2 row = rows[v];
      float s = 0.0f;
      for (uint32_t j = row.x + threadIdx.x; j < row.x + row.y; j += kPrThreads)
        s = __fadd_rn(s, contrib[nbr[j] & 0x3FFFFFFFu]);
#pragma unroll
      for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
      if (lane_id() == 0) s_part[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int w = 0; w < kPrThreads / 32; w++) tot = __fadd_rn(tot, s_part[w]);
        pr_update(v, tot, pr, out_degree, contrib_next, p, err, active);
      }
      __syncthreads();
    }
  }
  pr_block_finish(err, active, ctl, it);
}

// Push scatter: contrib of each source added to its out-neighbours, split by
// out-degree like the pull gather.
__global__ void __launch_bounds__(kPrThreads) pr_push_scatter_kernel(
    uint32_t nb_light, uint32_t nb_warp, const uint32_t* __restrict__ heavy, uint32_t n_warp, uint32_t n_cta,
    uint32_t V, uint32_t warp_thr, const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr,
    const float* __restrict__ contrib, float* __restrict__ next, const PrCtl* __restrict__ ctl) {
  if (ctl->stop) return;
  const uint32_t b = blockIdx.x;
  if (b < nb_light) {
    for (uint32_t v = b * kPrThreads + threadIdx.x; v < V; v += nb_light * kPrThreads) {
      const uint2 row = rows[v];
      if (row.y > warp_thr) continue;
      const float c = contrib[v];
      for (uint32_t j = row.x; j < row.x + row.y; j++) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  } else if (b < nb_light + nb_warp) {
    const uint32_t w0 = (b - nb_light) * (kPrThreads / 32) + (threadIdx.x >> 5);
    const uint32_t wstride = nb_warp * (kPrThreads / 32);
    for (uint32_t t = w0; t < n_warp; t += wstride) {
      const uint32_t v = heavy[t];
      const uint2 row = rows[v];
      const float c = contrib[v];
      for (uint32_t j = row.x + lane_id(); j < row.x + row.y; j += 32) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  } else {
    const uint32_t cb = b - nb_light - nb_warp;
    const uint32_t ncb = gridDim.x - nb_light - nb_warp;
    for (uint32_t t = cb; t < n_cta; t += ncb) {
      const uint32_t v = heavy[n_warp + t];
      const uint2 row = rows[v];
      const float c = contrib[v];
      for (uint32_t j = row.x + threadIdx.x; j < row.x + row.y; j += kPrThreads)
        atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
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
    const uint2* rows = pull ? g.inv.d_rows() : g.fwd.d_rows();
    uint32_t* cnt = w->ctl.as<uint32_t>() + sizeof(PrCtl) / 4;  // 16 scratch words after the control block
    OGB_CUDA(cudaMemsetAsync(cnt, 0, 16, s));
    const int grid = sm_count() * 8;
    pr_heavy_count_kernel<<<grid, 256, 0, s>>>(V, rows, g_warp_thr, g_cta_thr, cnt);
    OGB_CUDA(cudaGetLastError());
    OGB_CUDA(cudaMemcpyAsync(w->h_ctl, cnt, 8, cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaStreamSynchronize(s));
    w->n_warp = reinterpret_cast<uint32_t*>(w->h_ctl)[0];
    w->n_cta = reinterpret_cast<uint32_t*>(w->h_ctl)[1];
    OGB_CUDA(cudaMemsetAsync(cnt, 0, 16, s));
    pr_heavy_fill_kernel<<<grid, 256, 0, s>>>(V, rows, g_warp_thr, g_cta_thr, cnt, w->heavy.as<uint32_t>(),
                                              w->n_warp);
    OGB_CUDA(cudaGetLastError());
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

  const uint32_t nb_light = std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(V, T)));
  const uint32_t nb_warp = w->n_warp ? std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(w->n_warp, T / 32))) : 0;
  const uint32_t nb_cta = w->n_cta ? std::min<uint32_t>(sms * 2, w->n_cta) : 0;
  const uint32_t grid = nb_light + nb_warp + nb_cta;
  const uint2* rows = pull ? g.inv.d_rows() : g.fwd.d_rows();
  const uint32_t* nbr = pull ? g.inv.d_dst() : g.fwd.d_dst();
  const uint32_t* heavy = w->heavy.as<uint32_t>();

  OGB_CUDA(cudaEventRecord(w->ev0, s));
  for (uint32_t it = 0; it < max_iters; it++) {
    if (pull) {
      pr_pull_kernel<<<grid, T, 0, s>>>(nb_light, nb_warp, heavy, w->n_warp, w->n_cta, rows, nbr,
                                         g.fwd.d_out_degree(), c_cur, c_nxt, ranks, p, d_ctl, it);
    } else {
      pr_push_scatter_kernel<<<grid, T, 0, s>>>(nb_light, nb_warp, heavy, w->n_warp, w->n_cta, V, g_warp_thr, rows,
                                                 nbr, c_cur, nxt, d_ctl);
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
