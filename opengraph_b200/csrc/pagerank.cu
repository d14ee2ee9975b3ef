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
// Vertices are split once per graph into degree bins: a thread per vertex
// (sequential fp32 sum in CSR order, the reference's exact order), a warp
// per vertex, and a CTA per vertex (fixed-order tree sums; deterministic run
// to run).  Iterations are launched back to back without host round trips:
// each iteration's last CTA records error/active and, when active == 0, sets
// a stop flag that later launches read first.
#include "graph.cuh"

#include <algorithm>
#include <vector>

namespace ogb {

constexpr uint32_t kPrMaxIters = 1024;
constexpr uint32_t kBinWarp = 32;    // in-degree above this: warp per vertex
constexpr uint32_t kBinCta = 2048;   // in-degree above this: CTA per vertex

struct PrCtl {
  double err[kPrMaxIters];
  uint32_t active[kPrMaxIters];
  uint32_t blocks_done[kPrMaxIters];
  uint32_t stop;       // 1 once an iteration ended with no active vertex
  uint32_t stop_iter;  // index of that iteration
};

struct PrWork {
  uint32_t V = 0;
  int binned_for_pull = -1;  // which direction the bins describe
  DevBuf contrib0, contrib1, next, ctl;
  DevBuf bins;               // vertex ids: [thread bin | warp bin | cta bin]
  uint32_t n_thread = 0, n_warp = 0, n_cta = 0;
  PrCtl* h_ctl = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~PrWork() {
    if (h_ctl) cudaFreeHost(h_ctl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

void pr_work_free(PrWork* w) { delete w; }

// ------------------------------------------------------------------ bins ----

__global__ void pr_bin_count_kernel(uint32_t V, const uint2* __restrict__ rows, uint32_t* __restrict__ counts) {
  uint32_t c[3] = {0, 0, 0};
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    c[d > kBinCta ? 2 : (d > kBinWarp ? 1 : 0)]++;
  }
  for (int b = 0; b < 3; b++) warp_atomic_add_total(&counts[b], c[b]);
}

// Order inside a bin does not matter for the results (each vertex is
// reduced by exactly one thread, warp or CTA).
__global__ void pr_bin_fill_kernel(uint32_t V, const uint2* __restrict__ rows, uint32_t* __restrict__ cursor,
                                   uint32_t* __restrict__ bins, uint32_t off_warp, uint32_t off_cta) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    const int b = d > kBinCta ? 2 : (d > kBinWarp ? 1 : 0);
    uint32_t base = b == 0 ? 0 : (b == 1 ? off_warp : off_cta);
    bins[base + atomicAdd(&cursor[b], 1u)] = v;
  }
}

// ---------------------------------------------------------------- update ----

struct PrParams {
  float base_pr, damp;
  double epsilon;
  double inv_v;  // 1.0 / V is NOT used: the reference divides each error by V
  uint32_t V;
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

template <int THREADS>
__device__ __forceinline__ void pr_block_finish(double err, uint32_t active, PrCtl* ctl, uint32_t it) {
  __shared__ double s_err[THREADS / 32];
  __shared__ uint32_t s_act[THREADS / 32];
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
    for (int w = 0; w < THREADS / 32; w++) {
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

// Pull iteration: all three bins in one grid.  Blocks [0, nb_thread) run the
// thread bin, the next nb_warp blocks the warp bin, the rest the CTA bin.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) pr_pull_kernel(
    const uint32_t* __restrict__ bins, uint32_t n_thread, uint32_t n_warp, uint32_t n_cta, uint32_t nb_thread,
    uint32_t nb_warp, const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr,
    const uint32_t* __restrict__ out_degree, const float* __restrict__ contrib, float* __restrict__ contrib_next,
    float* __restrict__ pr, PrParams p, PrCtl* __restrict__ ctl, uint32_t it) {
  if (ctl->stop) return;
  double err = 0.0;
  uint32_t active = 0;
  const uint32_t b = blockIdx.x;
  if (b < nb_thread) {
    for (uint32_t t = b * THREADS + threadIdx.x; t < n_thread; t += nb_thread * THREADS) {
      const uint32_t v = bins[t];
      const uint2 row = rows[v];
      float s = 0.0f;
      for (uint32_t j = row.x; j < row.x + row.y; j++) s = __fadd_rn(s, contrib[nbr[j] & 0x3FFFFFFFu]);
      pr_update(v, s, pr, out_degree, contrib_next, p, err, active);
    }
  } else if (b < nb_thread + nb_warp) {
    const uint32_t lane = lane_id();
    const uint32_t w0 = (b - nb_thread) * (THREADS / 32) + (threadIdx.x >> 5);
    const uint32_t wstride = nb_warp * (THREADS / 32);
    for (uint32_t t = w0; t < n_warp; t += wstride) {
      const uint32_t v = bins[n_thread + t];
      const uint2 row = rows[v];
      float s = 0.0f;
      for (uint32_t j = row.x + lane; j < row.x + row.y; j += 32) s = __fadd_rn(s, contrib[nbr[j] & 0x3FFFFFFFu]);
      for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
      if (lane == 0) pr_update(v, s, pr, out_degree, contrib_next, p, err, active);
    }
  } else {
    __shared__ float s_part[THREADS / 32];
    const uint32_t cb = b - nb_thread - nb_warp;
    const uint32_t ncb = gridDim.x - nb_thread - nb_warp;
    for (uint32_t t = cb; t < n_cta; t += ncb) {
      const uint32_t v = bins[n_thread + n_warp + t];
      const uint2 row = rows[v];
      float s = 0.0f;
      for (uint32_t j = row.x + threadIdx.x; j < row.x + row.y; j += THREADS)
        s = __fadd_rn(s, contrib[nbr[j] & 0x3FFFFFFFu]);
      for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
      if (lane_id() == 0) s_part[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int w = 0; w < THREADS / 32; w++) tot = __fadd_rn(tot, s_part[w]);
        pr_update(v, tot, pr, out_degree, contrib_next, p, err, active);
      }
      __syncthreads();
    }
  }
  pr_block_finish<THREADS>(err, active, ctl, it);
}

// Push scatter: contrib of each source added to its out-neighbours.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) pr_push_scatter_kernel(
    const uint32_t* __restrict__ bins, uint32_t n_thread, uint32_t n_warp, uint32_t n_cta, uint32_t nb_thread,
    uint32_t nb_warp, const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr,
    const float* __restrict__ contrib, float* __restrict__ next, const PrCtl* __restrict__ ctl) {
  if (ctl->stop) return;
  const uint32_t b = blockIdx.x;
  if (b < nb_thread) {
    for (uint32_t t = b * THREADS + threadIdx.x; t < n_thread; t += nb_thread * THREADS) {
      const uint32_t v = bins[t];
      const uint2 row = rows[v];
      const float c = contrib[v];
      for (uint32_t j = row.x; j < row.x + row.y; j++) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  } else if (b < nb_thread + nb_warp) {
    const uint32_t lane = lane_id();
    const uint32_t w0 = (b - nb_thread) * (THREADS / 32) + (threadIdx.x >> 5);
    const uint32_t wstride = nb_warp * (THREADS / 32);
    for (uint32_t t = w0; t < n_warp; t += wstride) {
      const uint32_t v = bins[n_thread + t];
      const uint2 row = rows[v];
      const float c = contrib[v];
      for (uint32_t j = row.x + lane; j < row.x + row.y; j += 32) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  } else {
    const uint32_t cb = b - nb_thread - nb_warp;
    const uint32_t ncb = gridDim.x - nb_thread - nb_warp;
    for (uint32_t t = cb; t < n_cta; t += ncb) {
      const uint32_t v = bins[n_thread + n_warp + t];
      const uint2 row = rows[v];
      const float c = contrib[v];
      for (uint32_t j = row.x + threadIdx.x; j < row.x + row.y; j += THREADS) atomicAdd(&next[nbr[j] & 0x3FFFFFFFu], c);
    }
  }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) pr_push_update_kernel(uint32_t V, const uint32_t* __restrict__ out_degree,
                                                                 float* __restrict__ next,
                                                                 float* __restrict__ contrib_next,
                                                                 float* __restrict__ pr, PrParams p,
                                                                 PrCtl* __restrict__ ctl, uint32_t it) {
  if (ctl->stop) return;
  double err = 0.0;
  uint32_t active = 0;
  for (uint32_t v = blockIdx.x * THREADS + threadIdx.x; v < V; v += gridDim.x * THREADS) {
    const float s = next[v];
    next[v] = 0.0f;
    pr_update(v, s, pr, out_degree, contrib_next, p, err, active);
  }
  pr_block_finish<THREADS>(err, active, ctl, it);
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
    OGB_TRY(w->bins.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->ctl.alloc(sizeof(PrCtl)));
    w->V = V;
    w->binned_for_pull = -1;
  }
  if (!w->h_ctl) OGB_CUDA(cudaMallocHost(&w->h_ctl, sizeof(PrCtl)));
  if (!w->ev0) {
    OGB_CUDA(cudaEventCreate(&w->ev0));
    OGB_CUDA(cudaEventCreate(&w->ev1));
  }
  const int want = pull ? 1 : 0;
  if (w->binned_for_pull != want) {
    const uint2* rows = pull ? g.inv.d_rows() : g.fwd.d_rows();
    uint32_t* d_cnt = reinterpret_cast<uint32_t*>(w->h_ctl);  // reuse pinned memory as scratch
    DevBuf cnt;
    OGB_TRY(cnt.alloc(32));
    OGB_CUDA(cudaMemsetAsync(cnt.p, 0, 32, s));
    const int grid = sm_count() * 8;
    pr_bin_count_kernel<<<grid, 256, 0, s>>>(V, rows, cnt.as<uint32_t>());
    OGB_CUDA(cudaGetLastError());
    OGB_CUDA(cudaMemcpyAsync(d_cnt, cnt.p, 12, cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaStreamSynchronize(s));
    w->n_thread = d_cnt[0];
    w->n_warp = d_cnt[1];
    w->n_cta = d_cnt[2];
    OGB_CUDA(cudaMemsetAsync(cnt.p, 0, 32, s));
    pr_bin_fill_kernel<<<grid, 256, 0, s>>>(V, rows, cnt.as<uint32_t>(), w->bins.as<uint32_t>(), w->n_thread,
                                            w->n_thread + w->n_warp);
    OGB_CUDA(cudaGetLastError());
    OGB_CUDA(cudaStreamSynchronize(s));
    w->binned_for_pull = want;
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
  constexpr int T = 256;
  const int sms = sm_count();
  PrParams p;
  p.damp = 0.85f;
  p.base_pr = 1.0f - p.damp;
  p.epsilon = epsilon;
  p.inv_v = 0.0;
  p.V = V;
  PrCtl* d_ctl = w->ctl.as<PrCtl>();
  OGB_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(PrCtl), s));
  float* c_cur = w->contrib0.as<float>();
  float* c_nxt = w->contrib1.as<float>();
  float* nxt = w->next.as<float>();
  pr_init_kernel<<<sms * 8, 256, 0, s>>>(V, g.fwd.d_out_degree(), init, p.base_pr, ranks, c_cur, pull ? nullptr : nxt);
  OGB_CUDA(cudaGetLastError());

  // grid split between the bins (roughly by work)
  const uint32_t nb_thread = std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(w->n_thread, T)));
  const uint32_t nb_warp = w->n_warp ? std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(w->n_warp, T / 32))) : 0;
  const uint32_t nb_cta = w->n_cta ? std::min<uint32_t>(sms * 2, w->n_cta) : 0;
  const uint32_t grid = nb_thread + nb_warp + nb_cta;
  const uint2* rows = pull ? g.inv.d_rows() : g.fwd.d_rows();
  const uint32_t* nbr = pull ? g.inv.d_dst() : g.fwd.d_dst();
  const uint32_t* bins = w->bins.as<uint32_t>();

  OGB_CUDA(cudaEventRecord(w->ev0, s));
  for (uint32_t it = 0; it < max_iters; it++) {
    if (pull) {
      pr_pull_kernel<T><<<grid, T, 0, s>>>(bins, w->n_thread, w->n_warp, w->n_cta, nb_thread, nb_warp, rows, nbr,
                                           g.fwd.d_out_degree(), c_cur, c_nxt, ranks, p, d_ctl, it);
    } else {
      pr_push_scatter_kernel<T><<<grid, T, 0, s>>>(bins, w->n_thread, w->n_warp, w->n_cta, nb_thread, nb_warp, rows,
                                                   nbr, c_cur, nxt, d_ctl);
      pr_push_update_kernel<T><<<sms * 8, T, 0, s>>>(V, g.fwd.d_out_degree(), nxt, c_nxt, ranks, p, d_ctl, it);
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
