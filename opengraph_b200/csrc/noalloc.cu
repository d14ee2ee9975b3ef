// noalloc.cu -- PageRank pull that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they want a
// PageRank: code that runs while its process's memory is owned by another
// allocator or pool that must not be bypassed, services that forbid
// allocation on their request path (cudaMalloc synchronizes the device and
// can fail under fragmentation), and embeddings where the library may not
// hold allocations of its own between calls.  ogb_pagerank_pull_noalloc
// serves them: the caller passes the graph (inverse CSR) and the output, and
// every scratch buffer the iteration needs lives in one file-scope
// __device__ array of fixed size, defined below.  The array is part of the
// library's device image: every GPU that loads the library holds it
// (kScratchBytes below, about 12.6 MB) until the process exits.
//
// The computation is the library's pull PageRank (pageRank.c:939-1062
// semantics) with the row split of pagerank_run's pull kernel at its default
// thresholds (rows <= 32 edges summed by one thread in CSR order, rows <= 2048
// by a warp, both in the same order as that kernel; longer rows by one
// 256-thread CTA, where that kernel cuts them into chunks), reading the row
// start and length arrays directly instead of the packed rows of a DevGraph.
//
// Calls share the one array and each call overwrites what the previous one
// left there; two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on it.
#include <stdio.h>

#include <algorithm>
#include <mutex>

#include "../../include/ogb200_device.h"
#include "common.cuh"

namespace {

constexpr uint32_t kMaxV = OGB_NOALLOC_MAX_VERTICES;
constexpr uint32_t kMaxIters = 1024;
constexpr int kT = 256;
constexpr uint32_t kWarpThr = 32;
constexpr uint32_t kCtaThr = 2048;

struct NaCtl {
  double err[kMaxIters];
  uint32_t active[kMaxIters];
  uint32_t blocks_done[kMaxIters];
  uint32_t stop, stop_iter;
  uint32_t n_warp, n_cta;      // heavy-list sizes
  uint32_t cur_warp, cur_cta;  // fill cursors
};

// Scratch layout: contrib[2][kMaxV] floats, heavy[kMaxV] u32, then NaCtl.
constexpr size_t kOffContrib0 = 0;
constexpr size_t kOffContrib1 = (size_t)kMaxV * 4;
constexpr size_t kOffHeavy = (size_t)kMaxV * 8;
constexpr size_t kOffCtl = (size_t)kMaxV * 12;
constexpr size_t kScratchBytes = kOffCtl + ((sizeof(NaCtl) + 255) / 256) * 256;
static_assert(kScratchBytes <= (13u << 20), "scratch grew past the size the header states");

// The scratch.  Host code never dereferences or launches with this name: it
// is a host-side stand-in for the device symbol; the device address comes
// from cudaGetSymbolAddress in noalloc_setup().
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DevInfo {
  unsigned char* scratch;  // device address of g_noalloc_scratch on this device
  int sms;
};
constexpr int kMaxDevices = 64;
static DevInfo g_dev[kMaxDevices];  // filled by the first call on each device
static std::mutex g_dev_mu;         // guards g_dev: two host threads may make a first call at once

struct NaParams {
  float base_pr, damp;
  double epsilon;
  uint32_t V;
};

__global__ void na_init_kernel(uint32_t V, const uint32_t* __restrict__ out_degree, float base_pr,
                               float* __restrict__ pr, float* __restrict__ contrib) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    pr[v] = base_pr;
    const uint32_t d = out_degree[v];
    contrib[v] = d ? __fdiv_rn(base_pr, (float)d) : 0.0f;
  }
}

__global__ void na_heavy_count_kernel(uint32_t V, const uint32_t* __restrict__ deg, NaCtl* __restrict__ ctl) {
  uint32_t cw = 0, cc = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = deg[v];
    cw += (d > kWarpThr && d <= kCtaThr);
    cc += (d > kCtaThr);
  }
  ogb::warp_atomic_add_total(&ctl->n_warp, cw);
  ogb::warp_atomic_add_total(&ctl->n_cta, cc);
}

__global__ void na_heavy_fill_kernel(uint32_t V, const uint32_t* __restrict__ deg, uint32_t* __restrict__ heavy,
                                     NaCtl* __restrict__ ctl) {
  const uint32_t off_cta = ctl->n_warp;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = deg[v];
    if (d > kCtaThr)
      heavy[off_cta + atomicAdd(&ctl->cur_cta, 1u)] = v;
    else if (d > kWarpThr)
      heavy[atomicAdd(&ctl->cur_warp, 1u)] = v;
  }
}

__device__ __forceinline__ void na_update(uint32_t v, float s, float* __restrict__ pr,
                                          const uint32_t* __restrict__ out_degree, float* __restrict__ contrib_next,
                                          const NaParams& p, double& err, uint32_t& active) {
  const float nv = __fadd_rn(p.base_pr, __fmul_rn(p.damp, s));
  const float prev = pr[v];
  pr[v] = nv;
  const uint32_t d = out_degree[v];
  contrib_next[v] = d ? __fdiv_rn(nv, (float)d) : 0.0f;
  const double e = fabs((double)__fsub_rn(nv, prev));
  err += e / (double)p.V;
  active += (e >= p.epsilon) ? 1u : 0u;
}

__global__ void __launch_bounds__(kT) na_pull_kernel(uint32_t nb_light, uint32_t nb_warp,
                                                     const uint32_t* __restrict__ idx,
                                                     const uint32_t* __restrict__ deg,
                                                     const uint32_t* __restrict__ nbr,
                                                     const uint32_t* __restrict__ out_degree,
                                                     const uint32_t* __restrict__ heavy,
                                                     const float* __restrict__ contrib,
                                                     float* __restrict__ contrib_next, float* __restrict__ pr,
                                                     NaParams p, NaCtl* __restrict__ ctl, uint32_t it) {
  __shared__ double s_err[kT / 32];
  __shared__ uint32_t s_act[kT / 32];
  __shared__ float s_part[kT / 32];
  if (ctl->stop) return;
  const uint32_t n_warp = ctl->n_warp, n_cta = ctl->n_cta;
  double err = 0.0;
  uint32_t active = 0;
  const uint32_t b = blockIdx.x;
  if (b < nb_light) {
    for (uint32_t v = b * kT + threadIdx.x; v < p.V; v += nb_light * kT) {
      const uint32_t d = deg[v];
      if (d > kWarpThr) continue;
      const uint32_t a = idx[v];
      float s = 0.0f;
      for (uint32_t j = a; j < a + d; j++) s = __fadd_rn(s, contrib[nbr[j] & 0x3FFFFFFFu]);
      na_update(v, s, pr, out_degree, contrib_next, p, err, active);
    }
  } else if (b < nb_light + nb_warp) {
    const uint32_t w0 = (b - nb_light) * (kT / 32) + (threadIdx.x >> 5);
    for (uint32_t t = w0; t < n_warp; t += nb_warp * (kT / 32)) {
      const uint32_t v = heavy[t];
      const uint32_t a = idx[v], d = deg[v];
      float s = 0.0f;
      for (uint32_t j = a + ogb::lane_id(); j < a + d; j += 32) s = __fadd_rn(s, contrib[nbr[j] & 0x3FFFFFFFu]);
#pragma unroll
      for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
      if (ogb::lane_id() == 0) na_update(v, s, pr, out_degree, contrib_next, p, err, active);
    }
  } else {
    const uint32_t cb = b - nb_light - nb_warp, ncb = gridDim.x - nb_light - nb_warp;
    for (uint32_t t = cb; t < n_cta; t += ncb) {
      const uint32_t v = heavy[n_warp + t];
      const uint32_t a = idx[v], d = deg[v];
      float s = 0.0f;
      for (uint32_t j = a + threadIdx.x; j < a + d; j += kT) s = __fadd_rn(s, contrib[nbr[j] & 0x3FFFFFFFu]);
#pragma unroll
      for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
      if (ogb::lane_id() == 0) s_part[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int w = 0; w < kT / 32; w++) tot = __fadd_rn(tot, s_part[w]);
        na_update(v, tot, pr, out_degree, contrib_next, p, err, active);
      }
      __syncthreads();
    }
  }
  // block reduction of error / active; the last block of the iteration sets
  // the stop flag when no vertex is active
  for (int o = 16; o; o >>= 1) {
    err += __shfl_down_sync(0xffffffffu, err, o);
    active += __shfl_down_sync(0xffffffffu, active, o);
  }
  if (ogb::lane_id() == 0) {
    s_err[threadIdx.x >> 5] = err;
    s_act[threadIdx.x >> 5] = active;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0;
    uint32_t a = 0;
    for (int w = 0; w < kT / 32; w++) {
      e += s_err[w];
      a += s_act[w];
    }
    if (e != 0.0) atomicAdd(&ctl->err[it], e);
    if (a) atomicAdd(&ctl->active[it], a);
    __threadfence();
    if (atomicAdd(&ctl->blocks_done[it], 1u) == gridDim.x - 1) {
      __threadfence();
      if (atomicAdd(&ctl->active[it], 0u) == 0u) {
        ctl->stop_iter = it;
        ctl->stop = 1;
      }
    }
  }
}

__global__ void na_finish_kernel(uint32_t V, float* __restrict__ pr, const NaCtl* __restrict__ ctl,
                                 uint32_t max_iters, ogb_pr_info* __restrict__ out) {
  const float fv = (float)V;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    pr[v] = __fdiv_rn(pr[v], fv);
  if (out && blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t executed = ctl->stop ? ctl->stop_iter + 1 : max_iters;
    out->iterations = ctl->stop ? ctl->stop_iter : max_iters;
    out->executed = executed;
    out->converged = ctl->stop;
    out->activeVertices = executed ? ctl->active[executed - 1] : 0;
    out->error_total = executed ? ctl->err[executed - 1] : 0.0;
    out->ms = 0.0;
    out->launches = 0;
    out->pad = 0;
  }
}

// Once per device, with that device current: the device address of the
// scratch array (the host-side name is only a stand-in for the symbol).
int noalloc_setup(int dev, DevInfo** out) {
  if (dev < 0 || dev >= kMaxDevices) return ogb::fail(ogb::ERR_ARG, "noalloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_dev_mu);
  DevInfo& di = g_dev[dev];
  if (!di.scratch) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return ogb::fail(ogb::ERR_CUDA, "noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || sms <= 0)
      return ogb::fail(ogb::ERR_CUDA, "noalloc: cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
    di.sms = sms;
    di.scratch = static_cast<unsigned char*>(p);
  }
  *out = &di;
  return ogb::OK;
}

}  // namespace

extern "C" int ogb_pagerank_pull_noalloc(uint32_t num_vertices, const uint32_t* d_in_edges_idx,
                                         const uint32_t* d_in_degree, const uint32_t* d_in_neighbors,
                                         const uint32_t* d_out_degree, uint32_t max_iterations, double epsilon,
                                         float* d_ranks, ogb_pr_info* d_info, void* stream) {
  using namespace ogb;
  const uint32_t V = num_vertices;
  if (V == 0 || V > kMaxV)
    return fail(ERR_RANGE, "ogb_pagerank_pull_noalloc: num_vertices=%u outside 1..%u (the fixed scratch holds %u)", V,
                kMaxV, kMaxV);
  if (max_iterations > kMaxIters)
    return fail(ERR_ARG, "ogb_pagerank_pull_noalloc: at most %u iterations", kMaxIters);
  if (!d_in_edges_idx || !d_in_degree || !d_in_neighbors || !d_out_degree || !d_ranks)
    return fail(ERR_ARG, "ogb_pagerank_pull_noalloc: null array");
  int dev = 0;
  OGB_CUDA(cudaGetDevice(&dev));
  DevInfo* di = nullptr;
  OGB_TRY(noalloc_setup(dev, &di));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float* c0 = reinterpret_cast<float*>(di->scratch + kOffContrib0);
  float* c1 = reinterpret_cast<float*>(di->scratch + kOffContrib1);
  uint32_t* heavy = reinterpret_cast<uint32_t*>(di->scratch + kOffHeavy);
  NaCtl* ctl = reinterpret_cast<NaCtl*>(di->scratch + kOffCtl);

  NaParams p;
  p.damp = 0.85f;
  p.base_pr = 1.0f - p.damp;
  p.epsilon = epsilon;
  p.V = V;
  const int sms = di->sms;
  // the control block must start at zero; everything else is overwritten
  OGB_CUDA(cudaMemsetAsync(ctl, 0, sizeof(NaCtl), s));
  na_init_kernel<<<sms * 8, 256, 0, s>>>(V, d_out_degree, p.base_pr, d_ranks, c0);
  na_heavy_count_kernel<<<sms * 8, 256, 0, s>>>(V, d_in_degree, ctl);
  na_heavy_fill_kernel<<<sms * 8, 256, 0, s>>>(V, d_in_degree, heavy, ctl);
  OGB_CUDA(cudaGetLastError());
  const uint32_t nb_light = (uint32_t)std::min<uint64_t>((uint64_t)sms * 8, (V + kT - 1) / kT);
  const uint32_t nb_warp = sms * 8, nb_cta = sms * 2;
  float* cur = c0;
  float* nxt = c1;
  for (uint32_t it = 0; it < max_iterations; it++) {
    na_pull_kernel<<<nb_light + nb_warp + nb_cta, kT, 0, s>>>(nb_light, nb_warp, d_in_edges_idx, d_in_degree,
                                                             d_in_neighbors, d_out_degree, heavy, cur, nxt, d_ranks,
                                                             p, ctl, it);
    float* t = cur;
    cur = nxt;
    nxt = t;
  }
  na_finish_kernel<<<sms * 8, 256, 0, s>>>(V, d_ranks, ctl, max_iterations, d_info);
  OGB_CUDA(cudaGetLastError());
  return OK;
}
