// dd.cu -- data-driven PageRank, SPMV and the sort of vertices by rank.
//
// References (00_graph_bench/src/...):
//  * pageRankDataDrivenPullGraphCSR      algorithms/openmp/pageRank.c:2405-2564  (pushpull 6)
//  * pageRankDataDrivenPushGraphCSR      algorithms/openmp/pageRank.c:2566-2721  (pushpull 7)
//  * pageRankDataDrivenPullPushGraphCSR  algorithms/openmp/pageRank.c:2723-2919  (pushpull 8)
//  * SPMVPullGraphCSR / SPMVPushGraphCSR algorithms/openmp/SPMV.c:616-810
//  * radixSortEdgesByPageRank            preprocess/reorder.c:165-221
//
// Semantics kept:
//  * data-driven pull: every iteration first takes contrib[u] = pr[u] /
//    out_degree[u] for all vertices (0 without out-edges), then each vertex on
//    the current worklist sums its in-neighbours' contribs, computes
//    0.15 + 0.85 s, adds |new - old| / V to the error, and only when that
//    change is >= epsilon stores the new rank, counts itself active and puts
//    its out-neighbours on the next worklist.  Stop when no vertex was
//    active; ranks are divided by V at the end.  Deterministic: with the
//    summation order below the result is reproducible bit for bit;
//  * data-driven push: residuals start at (1 - d) d sum(1 / out_degree) over
//    in-neighbours; an active vertex takes its residual r, adds it to its
//    rank (error |new/V - old/V|) and pushes d r / out_degree to each
//    out-neighbour; an out-neighbour whose residual crosses epsilon (before
//    <= epsilon, after >= epsilon) counts as active and joins the next
//    worklist.  The reference runs this with unsynchronised reads of the
//    residuals (its result depends on thread timing); here the residual is
//    taken with an atomic exchange and every push is an atomic add whose
//    returned value decides the crossing, so no push is lost.  A self loop's
//    push is dropped, as in a sequential run of the reference (which zeroes
//    the vertex's residual after its own pushes).  Pull-push (8) sums
//    in-neighbours' current ranks / out-degree instead and, like the
//    reference, adds the delta a second time on a crossing;
//  * SPMV: x[v] = 1 / out_degree[v] (0.001 without out-edges); every
//    iteration adds w * x[src] to y[dst] for every edge, y never reset
//    (w = the edge weight in the WEIGHTED layout, else 0.0001); pull sums
//    the in-row, push uses float atomics;
//  * rank sort: stable ascending sort of the labels by the key
//    (uint32_t)(rank * 2^20 + 0.5f) (FloatToFixed32SORT, fixedPoint.h:33).
//
// Summation order of a row (pull sums): rows of at most kWarpThr edges are
// summed by one thread in CSR order (the reference's order); rows of at most
// kCtaThr edges by a warp (lane l adds elements l, l + 32, ... in order, then
// a butterfly fold); longer rows in chunks of kChunk edges, each chunk by
// kCtaThreads threads (strided the same way, warps folded, the warp sums
// added in warp order), the chunk sums added in chunk order.  The same split
// as the PageRank pull kernel at its default thresholds; the oracle
// reproduces it.  SPMV adds a row's sum to y (light rows add each term to y
// directly, as the reference does).
#include "graph.cuh"
#include "sort.cuh"

#include <algorithm>
#include <cstddef>
#include <mutex>
#include <vector>

namespace ogb {

namespace {

constexpr int kT = 256;
constexpr uint32_t kWarpThr = 32, kCtaThr = 2048, kChunk = 8192;
constexpr uint32_t kCtaThreads = kT;
constexpr uint32_t kMarkThr = 32;       // out-rows longer than this are deferred to a warp
constexpr uint32_t kOutBig = 1024;      // deferred out-rows longer than this go by chunks
constexpr uint32_t kOutChunk = 1024;    // edges per chunk of a long out-row
constexpr uint32_t kDdMaxIters = 1024;

struct DdCtl {
  double err[kDdMaxIters];
  uint32_t active[kDdMaxIters];
  uint32_t done_a[kDdMaxIters];   // blocks of the iteration's first kernel that finished
  uint32_t done_b[kDdMaxIters];   // blocks of its second kernel that finished
  uint32_t stop, stop_iter;
  uint32_t n_med, n_heavy, cur_med, cur_heavy;  // kept across runs of one graph build
  uint32_t n_och;                               // chunks of the long out-rows
};

struct DdWork {
  uint32_t V = 0;
  uint32_t built = 0;  // build id of the graph the row classes belong to
  bool ready = false;
  // defer: out-row of v pushed / marked by the deferred-row kernel this
  // iteration; dvec: its push delta; selfcnt: self loops per vertex; och:
  // {v, j0, j1} chunks of the out-rows longer than kOutBig
  DevBuf ctl, contrib, flags0, flags1, resid, med, heavy, defer, dvec, selfcnt, och, xin;
  uint32_t n_och = 0;
  DdCtl* h_ctl = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~DdWork() {
    if (h_ctl) cudaFreeHost(h_ctl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

// One work area per device graph, kept in a small table keyed by the graph
// (the graph's destructor releases it through dd_work_free).
struct DdSlot {
  const DevGraph* g;
  DdWork* w;
};
std::mutex g_dd_mu;
std::vector<DdSlot> g_dd;

__global__ void dd_count_kernel(uint32_t V, const uint2* __restrict__ rows, DdCtl* __restrict__ ctl) {
  uint32_t cm = 0, ch = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    cm += (d > kWarpThr && d <= kCtaThr);
    ch += (d > kCtaThr);
  }
  warp_atomic_add_total(&ctl->n_med, cm);
  warp_atomic_add_total(&ctl->n_heavy, ch);
}

// Self loops per vertex (counted once per graph build).
__global__ void dd_self_kernel(uint32_t E, const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst,
                               uint32_t* __restrict__ selfcnt) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < E; j += gridDim.x * blockDim.x) {
    const uint32_t u = src[j] & 0x3FFFFFFFu;
    if (u == (dst[j] & 0x3FFFFFFFu)) atomicAdd(&selfcnt[u], 1u);
  }
}

// Chunk counts of the long out-rows, then the chunks {v, j0, j1} at their
// scanned offsets.
__global__ void dd_och_count_kernel(uint32_t V, const uint2* __restrict__ rows_f, uint32_t* __restrict__ nch) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows_f[v].y;
    nch[v] = d > kOutBig ? (d + kOutChunk - 1) / kOutChunk : 0u;
  }
}
__global__ void dd_och_fill_kernel(uint32_t V, const uint2* __restrict__ rows_f, const uint32_t* __restrict__ off,
                                   uint4* __restrict__ och) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint2 r = rows_f[v];
    if (r.y <= kOutBig) continue;
    uint32_t k = off[v];
    for (uint32_t c = 0; c < r.y; c += kOutChunk, k++) och[k] = make_uint4(v, r.x + c, r.x + min(r.y, c + kOutChunk), 0u);
  }
}

__global__ void dd_fill_kernel(uint32_t V, const uint2* __restrict__ rows, uint32_t* __restrict__ med,
                               uint32_t* __restrict__ heavy, DdCtl* __restrict__ ctl) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    if (d > kCtaThr)
      heavy[atomicAdd(&ctl->cur_heavy, 1u)] = v;
    else if (d > kWarpThr)
      med[atomicAdd(&ctl->cur_med, 1u)] = v;
  }
}

// ---- row sums in the GPU summation order -------------------------------------

// Sum of term(j) over the row [a, a + d) by one warp (d <= kCtaThr): lane l
// adds elements l, l + 32, ... in order, then a butterfly fold; every lane
// returns the sum.
// Sequential sum s + term(j0) + term(j0 + step) + ... over [j0, j1), the
// terms fetched four at a time ahead of their additions (same order).
template <class Term>
__device__ __forceinline__ float strided_sum4(float s, uint32_t j0, uint32_t j1, uint32_t step, const Term& term) {
  uint32_t j = j0;
  for (; j + 3 * step < j1; j += 4 * step) {
    const float t0 = term(j), t1 = term(j + step), t2 = term(j + 2 * step), t3 = term(j + 3 * step);
    s = __fadd_rn(s, t0);
    s = __fadd_rn(s, t1);
    s = __fadd_rn(s, t2);
    s = __fadd_rn(s, t3);
  }
  for (; j < j1; j += step) s = __fadd_rn(s, term(j));
  return s;
}

template <class Term>
__device__ __forceinline__ float warp_row_sum(uint32_t a, uint32_t d, const Term& term) {
  float s = strided_sum4(0.0f, a + lane_id(), a + d, 32u, term);
#pragma unroll
  for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
}

// Sum over a long row by the whole CTA (kCtaThreads threads): chunks of
// kChunk edges, each chunk strided over the threads, warps folded, warp sums
// added in warp order; chunk sums added in chunk order.  The total is valid
// in thread 0.  Called by every thread of the CTA.
template <class Term>
__device__ float cta_row_sum(uint32_t a, uint32_t d, const Term& term, float* s_part) {
  float tot = 0.0f;
  for (uint32_t c = 0; c < d; c += kChunk) {
    const uint32_t len = min(kChunk, d - c);
    float s = strided_sum4(0.0f, a + c + threadIdx.x, a + c + len, kCtaThreads, term);
#pragma unroll
    for (int o = 16; o; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
    if (lane_id() == 0) s_part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      float ch = 0.0f;
      for (uint32_t w = 0; w < kCtaThreads / 32; w++) ch = __fadd_rn(ch, s_part[w]);
      tot = __fadd_rn(tot, ch);
    }
    __syncthreads();
  }
  return tot;
}

// One pass over the rows of the inverse CSR in three classes: blocks
// [0, nb_light) take the rows of at most kWarpThr edges (a thread each, in
// CSR order), the next nb_med blocks the medium list (a warp each), the rest
// the heavy list (a CTA each).  For each row with P.want(v): s = the row sum
// of P.term(j) in the order above, light rows starting from P.start(v),
// others P.start(v) + sum; then P.finish(v, s) (by lane 0 / thread 0 for the
// warp and CTA rows).
template <class P>
__device__ void rows_pass(const uint2* __restrict__ rows, const uint32_t* __restrict__ med,
                          const uint32_t* __restrict__ heavy, uint32_t n_med, uint32_t n_heavy, uint32_t V,
                          uint32_t nb_light, uint32_t nb_med, P& pol) {
  __shared__ float s_part[kT / 32];
  const uint32_t b = blockIdx.x;
  if (b < nb_light) {
    for (uint32_t v = b * kT + threadIdx.x; v < V; v += nb_light * kT) {
      const uint2 r = rows[v];
      if (r.y > kWarpThr || !pol.want(v)) continue;
      const float s = strided_sum4(pol.start(v), r.x, r.x + r.y, 1u, [&](uint32_t j) { return pol.term(j); });
      pol.finish(v, s);
    }
  } else if (b < nb_light + nb_med) {
    const uint32_t w0 = (b - nb_light) * (kT / 32) + (threadIdx.x >> 5);
    for (uint32_t t = w0; t < n_med; t += nb_med * (kT / 32)) {
      const uint32_t v = med[t];
      if (!pol.want(v)) continue;  // warp-uniform
      const uint2 r = rows[v];
      const float s = warp_row_sum(r.x, r.y, [&](uint32_t j) { return pol.term(j); });
      if (lane_id() == 0) pol.finish(v, __fadd_rn(pol.start(v), s));
    }
  } else {
    const uint32_t cb = b - nb_light - nb_med, ncb = gridDim.x - nb_light - nb_med;
    for (uint32_t t = cb; t < n_heavy; t += ncb) {
      const uint32_t v = heavy[t];
      if (!pol.want(v)) continue;  // CTA-uniform
      const uint2 r = rows[v];
      const float s = cta_row_sum(r.x, r.y, [&](uint32_t j) { return pol.term(j); }, s_part);
      if (threadIdx.x == 0) pol.finish(v, __fadd_rn(pol.start(v), s));
    }
  }
}

// Per-block error / active totals into ctl; the last block of the kernel
// (counter `done`) returns true in thread 0.
__device__ bool block_totals(double err, uint32_t act, double* g_err, uint32_t* g_act, uint32_t* done) {
  __shared__ double s_e[kT / 32];
  __shared__ uint32_t s_a[kT / 32];
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    err += __shfl_down_sync(0xffffffffu, err, o);
    act += __shfl_down_sync(0xffffffffu, act, o);
  }
  if (lane_id() == 0) {
    s_e[threadIdx.x >> 5] = err;
    s_a[threadIdx.x >> 5] = act;
  }
  __syncthreads();
  bool last = false;
  if (threadIdx.x == 0) {
    double e = 0.0;
    uint32_t a = 0;
    for (uint32_t w = 0; w < blockDim.x / 32; w++) {
      e += s_e[w];
      a += s_a[w];
    }
    if (e != 0.0) atomicAdd(g_err, e);
    if (a) atomicAdd(g_act, a);
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
    if (last) __threadfence();
  }
  return last;
}

struct DdParams {
  uint32_t V;
  float damp, base_pr;
  double epsilon;
};

// ---- data-driven pull (6) -----------------------------------------------------

// Put u on the next worklist.  Most marks of an iteration hit a vertex that
// is marked already (RMAT hubs are in-neighbours of many active vertices):
// the flag is read first, from L1 / L2, and only a clear flag is written.
__device__ __forceinline__ void mark(uint8_t* next, uint32_t u) {
  if (!next[u]) next[u] = 1;
}

__global__ void dd_contrib_kernel(uint32_t V, const uint32_t* __restrict__ out_degree, const float* __restrict__ pr,
                                  float* __restrict__ contrib, uint8_t* __restrict__ next,
                                  uint8_t* __restrict__ defer, const DdCtl* __restrict__ ctl) {
  if (ctl->stop) return;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = out_degree[v];
    contrib[v] = d ? __fdiv_rn(pr[v], (float)d) : 0.0f;
    next[v] = 0;
    defer[v] = 0;
  }
}

struct PullPolicy {
  const uint8_t* cur;
  uint8_t* next;
  const float* contrib;
  const uint32_t* nbr;
  float* pr;
  const uint2* rows_f;
  const uint32_t* nbr_f;
  uint8_t* defer;
  DdParams p;
  double err = 0.0;
  uint32_t act = 0;
  __device__ bool want(uint32_t v) const { return cur[v] != 0; }
  __device__ float start(uint32_t) const { return 0.0f; }
  __device__ float term(uint32_t j) const { return contrib[nbr[j] & 0x3FFFFFFFu]; }
  __device__ void finish(uint32_t v, float s) {
    const float nv = __fadd_rn(p.base_pr, __fmul_rn(p.damp, s));
    const float old = pr[v];
    const double e = fabs((double)__fsub_rn(nv, old));
    err += e / (double)p.V;
    if (e >= p.epsilon) {
      pr[v] = nv;
      act++;
      const uint2 r = rows_f[v];
      if (r.y <= kMarkThr) {
        const uint32_t e = r.x + r.y;
        uint32_t j = r.x;
        for (; j + 3 < e; j += 4) {  // four neighbour ids in flight
          const uint32_t u0 = nbr_f[j], u1 = nbr_f[j + 1], u2 = nbr_f[j + 2], u3 = nbr_f[j + 3];
          mark(next, u0 & 0x3FFFFFFFu);
          mark(next, u1 & 0x3FFFFFFFu);
          mark(next, u2 & 0x3FFFFFFFu);
          mark(next, u3 & 0x3FFFFFFFu);
        }
        for (; j < e; j++) mark(next, nbr_f[j] & 0x3FFFFFFFu);
      } else {
        defer[v] = 1;
      }
    }
  }
};

__global__ void __launch_bounds__(kT) dd_pull_kernel(const uint2* __restrict__ rows, const uint32_t* __restrict__ med,
                                                     const uint32_t* __restrict__ heavy, uint32_t nb_light,
                                                     uint32_t nb_med, PullPolicy pol, DdCtl* __restrict__ ctl,
                                                     uint32_t it) {
  if (ctl->stop) return;
  rows_pass(rows, med, heavy, ctl->n_med, ctl->n_heavy, pol.p.V, nb_light, nb_med, pol);
  if (block_totals(pol.err, pol.act, &ctl->err[it], &ctl->active[it], &ctl->done_a[it])) {
    if (ld_volatile_u32(&ctl->active[it]) == 0) {
      ctl->stop_iter = it;
      ctl->stop = 1;
    }
  }
}

// ---- data-driven push (7) and pull-push (8) --------------------------------

// Initial residuals: (1 - d) d * sum over in-neighbours u of 1 / out_degree[u].
struct ResidPolicy {
  const uint32_t* nbr;
  const uint32_t* out_degree;
  float* resid;
  float coef;
  __device__ bool want(uint32_t) const { return true; }
  __device__ float start(uint32_t) const { return 0.0f; }
  __device__ float term(uint32_t j) const {
    const uint32_t d = out_degree[nbr[j] & 0x3FFFFFFFu];
    return d ? __fdiv_rn(1.0f, (float)d) : 0.0f;
  }
  __device__ void finish(uint32_t v, float s) { resid[v] = __fmul_rn(coef, s); }
};

__global__ void __launch_bounds__(kT) dd_resid_kernel(const uint2* __restrict__ rows, const uint32_t* __restrict__ med,
                                                      const uint32_t* __restrict__ heavy, uint32_t nb_light,
                                                      uint32_t nb_med, ResidPolicy pol, const DdCtl* __restrict__ ctl,
                                                      uint32_t V) {
  rows_pass(rows, med, heavy, ctl->n_med, ctl->n_heavy, V, nb_light, nb_med, pol);
}

// One push of delta into resid[u]: the returned old value decides whether u
// crossed epsilon (before <= eps, after >= eps); pull-push (twice) then adds
// the delta a second time, as the reference does.
__device__ __forceinline__ uint32_t push_cross(uint32_t u, float prev, float delta, float* resid, uint8_t* next,
                                               double eps, bool twice) {
  if ((double)fabsf(__fadd_rn(prev, delta)) >= eps && (double)prev <= eps) {
    if (twice) atomicAdd(&resid[u], delta);
    next[u] = 1;
    return 1;
  }
  return 0;
}

// The pushes of the out-row range [j0, j1) of v by `nl` lanes from `lane`,
// four pushes in flight per lane.  A self loop's push is dropped (see the
// header; self_loops counts it).  Returns the crossings counted.  In
// pull-push a neighbour repeated within one group of four sees the group's
// earlier push before that push's second add rather than after it: the adds
// commute, and a residual that crossed epsilon is above it, so the later
// push counts no crossing either way.
__device__ __forceinline__ uint32_t push_range(uint32_t v, uint32_t j0, uint32_t j1, float delta, uint32_t lane,
                                               uint32_t nl, const uint32_t* __restrict__ nbr_f, float* resid,
                                               uint8_t* next, double eps, bool twice) {
  uint32_t act = 0;
  for (uint32_t j = j0 + lane; j < j1; j += 4 * nl) {
    uint32_t u[4];
    float prev[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t jj = j + k * nl;
      u[k] = jj < j1 ? (nbr_f[jj] & 0x3FFFFFFFu) : v;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) prev[k] = u[k] != v ? atomicAdd(&resid[u[k]], delta) : 0.0f;
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (u[k] != v) act += push_cross(u[k], prev[k], delta, resid, next, eps, twice);
  }
  return act;
}

// A vertex's `ns` self loops, counted as a sequential run of the reference
// counts them (the vertex's own residual, read before it is zeroed).
__device__ __forceinline__ uint32_t self_loops(uint32_t v, uint32_t ns, float r, float delta, uint8_t* next,
                                               double eps, bool twice) {
  uint32_t act = 0;
  float acc = r;
  for (uint32_t k = 0; k < ns; k++) {
    const float prev = acc;
    acc = __fadd_rn(acc, delta);
    if ((double)fabsf(acc) >= eps && (double)prev <= eps) {
      act++;
      if (twice) acc = __fadd_rn(acc, delta);
      next[v] = 1;
    }
  }
  return act;
}

// Update of one active vertex given its new rank and the residual it took
// (atomically, before): error, rank store (and, for pull-push, the rank /
// out-degree its out-neighbours' pulls read), and the pushes (out-rows of at
// most kMarkThr edges here, longer ones deferred with their delta).
__device__ __forceinline__ void push_vertex(uint32_t v, float nv, float old, float r, const uint2* rows_f,
                                            const uint32_t* nbr_f, const uint32_t* selfcnt, float* pr, float* contrib,
                                            float* resid, uint8_t* next, uint8_t* defer, float* dvec,
                                            const DdParams& p, bool twice, double& err, uint32_t& act) {
  const float fv = (float)p.V;
  err += (double)fabsf(__fsub_rn(__fdiv_rn(nv, fv), __fdiv_rn(old, fv)));
  pr[v] = nv;
  const uint2 row = rows_f[v];
  if (!row.y) return;  // no pushes (the reference's delta divides by zero here and is never used)
  if (contrib) contrib[v] = __fdiv_rn(nv, (float)row.y);
  const float delta = __fmul_rn(p.damp, __fdiv_rn(r, (float)row.y));
  const uint32_t ns = selfcnt[v];
  if (ns) act += self_loops(v, ns, r, delta, next, p.epsilon, twice);
  if (row.y <= kMarkThr) {
    act += push_range(v, row.x, row.x + row.y, delta, 0, 1, nbr_f, resid, next, p.epsilon, twice);
  } else {
    dvec[v] = delta;
    defer[v] = 1;
  }
}

__global__ void __launch_bounds__(kT) dd_push_kernel(uint32_t V, const uint8_t* __restrict__ cur, uint8_t* next,
                                                     const uint2* __restrict__ rows_f,
                                                     const uint32_t* __restrict__ nbr_f,
                                                     const uint32_t* __restrict__ selfcnt, float* pr, float* resid,
                                                     uint8_t* defer, float* dvec, DdParams p,
                                                     DdCtl* __restrict__ ctl, uint32_t it) {
  if (ctl->stop) return;
  double err = 0.0;
  uint32_t act = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    if (!cur[v]) continue;
    const float r = atomicExch(&resid[v], 0.0f);
    const float old = pr[v];
    const float nv = __fadd_rn(r, old);  // the reference's aResiduals[v] + pageRanks[v]
    push_vertex(v, nv, old, r, rows_f, nbr_f, selfcnt, pr, nullptr, resid, next, defer, dvec, p, false, err, act);
  }
  block_totals(err, act, &ctl->err[it], &ctl->active[it], &ctl->done_a[it]);
}

// Pull-push (8): the row sum of current ranks / out-degree, then the pushes.
// contrib[u] holds rank[u] / out_degree[u], rewritten by every rank update
// (a vertex with in-neighbours' reads racing its update sees the old or the
// new value, as the reference's reads of pageRanks[u] do), so a term is one
// gather and no division.
struct PullPushPolicy {
  const uint8_t* cur;
  uint8_t* next;
  const uint32_t* nbr;
  float* contrib;
  float* pr;
  float* resid;
  const uint2* rows_f;
  const uint32_t* nbr_f;
  const uint32_t* selfcnt;
  uint8_t* defer;
  float* dvec;
  DdParams p;
  double err = 0.0;
  uint32_t act = 0;
  __device__ bool want(uint32_t v) const { return cur[v] != 0; }
  __device__ float start(uint32_t) const { return 0.0f; }
  __device__ float term(uint32_t j) const { return contrib[nbr[j] & 0x3FFFFFFFu]; }
  __device__ void finish(uint32_t v, float s) {
    const float nv = __fadd_rn(p.base_pr, __fmul_rn(p.damp, s));
    const float old = pr[v];
    const float r = atomicExch(&resid[v], 0.0f);
    push_vertex(v, nv, old, r, rows_f, nbr_f, selfcnt, pr, contrib, resid, next, defer, dvec, p, true, err, act);
  }
};

__global__ void __launch_bounds__(kT) dd_pullpush_kernel(const uint2* __restrict__ rows,
                                                         const uint32_t* __restrict__ med,
                                                         const uint32_t* __restrict__ heavy, uint32_t nb_light,
                                                         uint32_t nb_med, PullPushPolicy pol,
                                                         DdCtl* __restrict__ ctl, uint32_t it) {
  if (ctl->stop) return;
  rows_pass(rows, med, heavy, ctl->n_med, ctl->n_heavy, pol.p.V, nb_light, nb_med, pol);
  block_totals(pol.err, pol.act, &ctl->err[it], &ctl->active[it], &ctl->done_a[it]);
}

// The deferred out-rows of an iteration (defer[v] set): first the chunks of
// the rows longer than kOutBig, a warp per chunk; then every other deferred
// row, a warp per row, found by a warp scan of the flags of 32 vertices at a
// time.  kPush: the pushes of delta dvec[v] (crossings counted, the last
// block decides the stop); otherwise the worklist marks of the pull.
template <bool kPush>
__global__ void __launch_bounds__(kT) dd_defer_kernel(uint32_t V, const uint2* __restrict__ rows_f,
                                                      const uint32_t* __restrict__ nbr_f,
                                                      const uint8_t* __restrict__ defer,
                                                      const float* __restrict__ dvec, const uint4* __restrict__ och,
                                                      float* resid, uint8_t* next, double eps, bool twice,
                                                      DdCtl* __restrict__ ctl, uint32_t it) {
  if (ctl->stop) return;
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * kT + threadIdx.x) >> 5, nw = (gridDim.x * kT) >> 5;
  const uint32_t n_och = ctl->n_och;
  uint32_t act = 0;
  for (uint32_t c = gw; c < n_och; c += nw) {
    const uint4 e = och[c];
    if (!defer[e.x]) continue;  // warp-uniform
    if (kPush)
      act += push_range(e.x, e.y, e.z, dvec[e.x], lane, 32, nbr_f, resid, next, eps, twice);
    else
      for (uint32_t j = e.y + lane; j < e.z; j += 32) mark(next, nbr_f[j] & 0x3FFFFFFFu);
  }
  for (uint32_t base = gw * 32; base < V; base += nw * 32) {
    const uint32_t v = base + lane;
    uint2 r = make_uint2(0u, 0u);
    if (v < V && defer[v]) r = rows_f[v];
    uint32_t m = __ballot_sync(0xffffffffu, r.y > 0 && r.y <= kOutBig);
    while (m) {
      const uint32_t l = (uint32_t)__ffs(m) - 1;
      m &= m - 1;
      const uint32_t vv = base + l;
      const uint32_t a = __shfl_sync(0xffffffffu, r.x, l), d = __shfl_sync(0xffffffffu, r.y, l);
      if (kPush)
        act += push_range(vv, a, a + d, dvec[vv], lane, 32, nbr_f, resid, next, eps, twice);
      else
        for (uint32_t j = a + lane; j < a + d; j += 32) mark(next, nbr_f[j] & 0x3FFFFFFFu);
    }
  }
  if (!kPush) return;
  if (block_totals(0.0, act, &ctl->err[it], &ctl->active[it], &ctl->done_b[it])) {
    if (ld_volatile_u32(&ctl->active[it]) == 0) {
      ctl->stop_iter = it;
      ctl->stop = 1;
    }
  }
}

__global__ void dd_init_kernel(uint32_t V, float base_pr, float* __restrict__ pr, uint8_t* __restrict__ cur,
                               uint8_t* __restrict__ next) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    pr[v] = base_pr;
    cur[v] = 1;
    next[v] = 0;
  }
}

__global__ void dd_clear_kernel(uint32_t V, uint8_t* __restrict__ next, uint8_t* __restrict__ defer,
                                const DdCtl* __restrict__ ctl) {
  if (ctl->stop) return;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    next[v] = 0;
    defer[v] = 0;
  }
}

__global__ void dd_normalize_kernel(uint32_t V, float* __restrict__ pr) {
  const float fv = (float)V;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    pr[v] = __fdiv_rn(pr[v], fv);
}

// ---- SPMV ---------------------------------------------------------------------

__global__ void spmv_init_kernel(uint32_t V, const uint32_t* __restrict__ out_degree, float* __restrict__ x,
                                 float* __restrict__ y) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t d = out_degree[v];
    x[v] = d ? __fdiv_rn(1.0f, (float)d) : 0.001f;
    y[v] = 0.0f;
  }
}

struct SpmvPullPolicy {
  const uint32_t* nbr;
  const float* w;  // null: every weight is kSpmvDefaultWeight
  const float* x;
  float* y;
  __device__ bool want(uint32_t) const { return true; }
  __device__ float start(uint32_t v) const { return y[v]; }
  __device__ float term(uint32_t j) const {
    return __fmul_rn(w ? w[j] : 0.0001f, x[nbr[j] & 0x3FFFFFFFu]);
  }
  __device__ void finish(uint32_t v, float s) { y[v] = s; }
};

__global__ void __launch_bounds__(kT) spmv_pull_kernel(const uint2* __restrict__ rows, const uint32_t* __restrict__ med,
                                                       const uint32_t* __restrict__ heavy, uint32_t nb_light,
                                                       uint32_t nb_med, SpmvPullPolicy pol,
                                                       const DdCtl* __restrict__ ctl, uint32_t V) {
  rows_pass(rows, med, heavy, ctl->n_med, ctl->n_heavy, V, nb_light, nb_med, pol);
}

// Push: rows of at most kWarpThr out-edges by a thread, rows up to kOutBig
// by a warp, longer ones in chunks of kOutChunk edges, a warp per chunk
// (order does not matter: float atomics, as the reference's omp atomic).
__device__ __forceinline__ float spmv_term(const float* __restrict__ w, uint32_t j, float xv) {
  return __fmul_rn(w ? w[j] : 0.0001f, xv);
}

__global__ void __launch_bounds__(kT) spmv_push_kernel(uint32_t V, const uint2* __restrict__ rows_f,
                                                       const uint32_t* __restrict__ nbr_f, const float* __restrict__ w,
                                                       const float* __restrict__ x, float* __restrict__ y,
                                                       const uint4* __restrict__ och, const DdCtl* __restrict__ ctl) {
  const uint32_t lane = lane_id();
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t n_och = ctl->n_och;
  for (uint32_t c = gw; c < n_och; c += nw) {
    const uint4 e = och[c];
    const float xv = x[e.x];
    for (uint32_t j = e.y + lane; j < e.z; j += 32) atomicAdd(&y[nbr_f[j] & 0x3FFFFFFFu], spmv_term(w, j, xv));
  }
  for (uint32_t base = gw * 32; base < V; base += nw * 32) {
    const uint32_t v = base + lane;
    uint2 r = make_uint2(0u, 0u);
    if (v < V) r = rows_f[v];
    if (r.y && r.y <= kWarpThr) {
      const float xv = x[v];
      for (uint32_t j = r.x; j < r.x + r.y; j++) atomicAdd(&y[nbr_f[j] & 0x3FFFFFFFu], spmv_term(w, j, xv));
    }
    uint32_t longm = __ballot_sync(0xffffffffu, r.y > kWarpThr && r.y <= kOutBig);
    while (longm) {
      const uint32_t l = (uint32_t)__ffs(longm) - 1;
      longm &= longm - 1;
      const uint32_t vv = base + l;
      const uint32_t a = __shfl_sync(0xffffffffu, r.x, l), d = __shfl_sync(0xffffffffu, r.y, l);
      const float xv = x[vv];
      for (uint32_t j = a + lane; j < a + d; j += 32) atomicAdd(&y[nbr_f[j] & 0x3FFFFFFFu], spmv_term(w, j, xv));
    }
  }
}

// ---- sort by rank ---------------------------------------------------------------

__global__ void rank_keys_kernel(uint32_t n, const float* __restrict__ ranks, uint32_t* __restrict__ keys) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keys[i] = __float2uint_rz(__fadd_rn(__fmul_rn(ranks[i], 1048576.0f), ranks[i] >= 0.0f ? 0.5f : -0.5f));
}

// ---- host side -------------------------------------------------------------------

int dd_work_get(DevGraph& g, DdWork** out, cudaStream_t s) {
  DdWork* w = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_dd_mu);
    for (auto& e : g_dd)
      if (e.g == &g) w = e.w;
    if (!w) {
      w = new DdWork();
      g_dd.push_back({&g, w});
    }
  }
  const uint32_t V = g.V;
  if (w->V != V || !w->ctl.p) {
    OGB_TRY(w->ctl.alloc(sizeof(DdCtl)));
    OGB_TRY(w->contrib.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->flags0.alloc((size_t)V + 16));
    OGB_TRY(w->flags1.alloc((size_t)V + 16));
    OGB_TRY(w->resid.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->med.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->heavy.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->defer.alloc((size_t)V + 16));
    OGB_TRY(w->dvec.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->selfcnt.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->xin.alloc((size_t)V * 4 + 16));
    w->V = V;
    w->ready = false;
  }
  if (!w->h_ctl) OGB_CUDA(cudaMallocHost(&w->h_ctl, sizeof(DdCtl)));
  if (!w->ev0) {
    OGB_CUDA(cudaEventCreate(&w->ev0));
    OGB_CUDA(cudaEventCreate(&w->ev1));
  }
  DdCtl* ctl = w->ctl.as<DdCtl>();
  if (w->ready && w->built == g.build_id) {
    // per-run counters only; the row classes and chunk count stay
    OGB_CUDA(cudaMemsetAsync(w->ctl.p, 0, offsetof(DdCtl, n_med), s));
    *out = w;
    return OK;
  }
  // once per graph build: the inverse rows' classes, the self loops, and the
  // chunks of the long out-rows
  OGB_CUDA(cudaMemsetAsync(w->ctl.p, 0, sizeof(DdCtl), s));
  OGB_CUDA(cudaMemsetAsync(w->defer.p, 0, (size_t)V + 16, s));
  OGB_CUDA(cudaMemsetAsync(w->selfcnt.p, 0, (size_t)V * 4 + 16, s));
  const int grid = sm_count() * 8;
  dd_count_kernel<<<grid, kT, 0, s>>>(V, g.inv.d_rows(), ctl);
  dd_fill_kernel<<<grid, kT, 0, s>>>(V, g.inv.d_rows(), w->med.as<uint32_t>(), w->heavy.as<uint32_t>(), ctl);
  dd_self_kernel<<<grid, kT, 0, s>>>(g.E, g.fwd.d_src(), g.fwd.d_dst(), w->selfcnt.as<uint32_t>());
  OGB_CUDA(cudaGetLastError());
  DevBuf tmp;
  OGB_TRY(tmp.alloc(((size_t)V * 2 + 4 + scan_tmp_words(V)) * 4));
  uint32_t* nch = tmp.as<uint32_t>();
  uint32_t* off = nch + V + 2;
  uint32_t* stmp = off + V + 2;
  dd_och_count_kernel<<<grid, kT, 0, s>>>(V, g.fwd.d_rows(), nch);
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(scan_exclusive_u32(nch, off, V, stmp, s));
  uint32_t total = 0;
  OGB_CUDA(cudaMemcpyAsync(&total, off + V, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  OGB_TRY(w->och.alloc((size_t)total * 16 + 16));
  dd_och_fill_kernel<<<grid, kT, 0, s>>>(V, g.fwd.d_rows(), off, w->och.as<uint4>());
  OGB_CUDA(cudaGetLastError());
  w->n_och = total;
  OGB_CUDA(cudaMemcpyAsync(&ctl->n_och, &w->n_och, 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaStreamSynchronize(s));  // the host copy source and tmp outlive the copies
  w->built = g.build_id;
  w->ready = true;
  *out = w;
  return OK;
}

struct Grid3 {
  uint32_t light, med, heavy;
  uint32_t total() const { return light + med + heavy; }
};

Grid3 rows_grid(uint32_t V) {
  const uint32_t sms = sm_count();
  Grid3 g;
  g.light = std::max<uint32_t>(1, std::min<uint32_t>(sms * 8, ceil_div(V, kT)));
  g.med = sms * 8;
  g.heavy = sms * 2;
  return g;
}

}  // namespace

void dd_work_free(const DevGraph* g) {
  std::lock_guard<std::mutex> lk(g_dd_mu);
  for (size_t i = 0; i < g_dd.size(); i++) {
    if (g_dd[i].g == g) {
      delete g_dd[i].w;
      g_dd.erase(g_dd.begin() + (long)i);
      return;
    }
  }
}

int pagerank_dd_run(DevGraph& g, uint32_t mode, uint32_t max_iters, double epsilon, float* ranks, PrResult* res,
                    cudaStream_t s) {
  if (mode < PR_DD_PULL || mode > PR_DD_PULLPUSH) return fail(ERR_ARG, "data-driven pagerank: mode %u", mode);
  if (max_iters > kDdMaxIters) return fail(ERR_ARG, "data-driven pagerank: at most %u iterations", kDdMaxIters);
  const uint32_t V = g.V;
  if (V == 0) return fail(ERR_ARG, "pagerank: empty graph");
  DdWork* w = nullptr;
  OGB_TRY(dd_work_get(g, &w, s));
  DdCtl* ctl = w->ctl.as<DdCtl>();
  DdParams p;
  p.V = V;
  p.damp = 0.85f;
  p.base_pr = 1.0f - p.damp;  // float, as newPageRankStatsGraphCSR (pageRank.c:47-75)
  p.epsilon = epsilon;
  const int sms = sm_count();
  const Grid3 G = rows_grid(V);
  uint8_t* cur = w->flags0.as<uint8_t>();
  uint8_t* nxt = w->flags1.as<uint8_t>();
  float* resid = w->resid.as<float>();
  OGB_CUDA(cudaEventRecord(w->ev0, s));
  dd_init_kernel<<<sms * 8, kT, 0, s>>>(V, p.base_pr, ranks, cur, nxt);
  uint32_t launches = 1;
  if (mode != PR_DD_PULL) {
    // (1.0f - damp) * damp, then times the row sum (pageRank.c:2614), in float
    const float coef = (1.0f - p.damp) * p.damp;
    ResidPolicy rp{g.inv.d_dst(), g.fwd.d_out_degree(), resid, coef};
    dd_resid_kernel<<<G.total(), kT, 0, s>>>(g.inv.d_rows(), w->med.as<uint32_t>(), w->heavy.as<uint32_t>(), G.light,
                                             G.med, rp, ctl, V);
    launches++;
    if (mode == PR_DD_PULLPUSH) {  // the starting ranks / out-degree (flags cleared on the way)
      dd_contrib_kernel<<<sms * 8, kT, 0, s>>>(V, g.fwd.d_out_degree(), ranks, w->contrib.as<float>(), nxt,
                                               w->defer.as<uint8_t>(), ctl);
      launches++;
    }
  }
  OGB_CUDA(cudaGetLastError());
  for (uint32_t it = 0; it < max_iters; it++) {
    uint8_t* defer = w->defer.as<uint8_t>();
    float* dvec = w->dvec.as<float>();
    const uint4* och = w->och.as<uint4>();
    if (mode == PR_DD_PULL) {
      dd_contrib_kernel<<<sms * 8, kT, 0, s>>>(V, g.fwd.d_out_degree(), ranks, w->contrib.as<float>(), nxt, defer,
                                               ctl);
      PullPolicy pol{cur, nxt, w->contrib.as<float>(), g.inv.d_dst(), ranks, g.fwd.d_rows(), g.fwd.d_dst(), defer, p};
      dd_pull_kernel<<<G.total(), kT, 0, s>>>(g.inv.d_rows(), w->med.as<uint32_t>(), w->heavy.as<uint32_t>(),
                                               G.light, G.med, pol, ctl, it);
      dd_defer_kernel<false><<<sms * 8, kT, 0, s>>>(V, g.fwd.d_rows(), g.fwd.d_dst(), defer, dvec, och, resid, nxt,
                                                    epsilon, false, ctl, it);
    } else {
      dd_clear_kernel<<<sms * 8, kT, 0, s>>>(V, nxt, defer, ctl);
      if (mode == PR_DD_PUSH) {
        dd_push_kernel<<<sms * 8, kT, 0, s>>>(V, cur, nxt, g.fwd.d_rows(), g.fwd.d_dst(), w->selfcnt.as<uint32_t>(),
                                               ranks, resid, defer, dvec, p, ctl, it);
      } else {
        PullPushPolicy pol{cur,   nxt,  g.inv.d_dst(), w->contrib.as<float>(), ranks, resid, g.fwd.d_rows(),
                           g.fwd.d_dst(), w->selfcnt.as<uint32_t>(), defer, dvec, p};
        dd_pullpush_kernel<<<G.total(), kT, 0, s>>>(g.inv.d_rows(), w->med.as<uint32_t>(), w->heavy.as<uint32_t>(),
                                                     G.light, G.med, pol, ctl, it);
      }
      dd_defer_kernel<true><<<sms * 8, kT, 0, s>>>(V, g.fwd.d_rows(), g.fwd.d_dst(), defer, dvec, och, resid, nxt,
                                                   epsilon, mode == PR_DD_PULLPUSH, ctl, it);
    }
    OGB_CUDA(cudaGetLastError());
    launches += 3;
    std::swap(cur, nxt);
  }
  dd_normalize_kernel<<<sms * 8, kT, 0, s>>>(V, ranks);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaEventRecord(w->ev1, s));
  OGB_CUDA(cudaMemcpyAsync(w->h_ctl, ctl, sizeof(DdCtl), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&ms, w->ev0, w->ev1));
  PrResult r;
  r.ms = ms;
  r.launches = launches + 1;
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

int spmv_run(DevGraph& g, uint32_t mode, uint32_t iterations, float* x, float* y, double* ms_out, cudaStream_t s) {
  if (mode > 1) return fail(ERR_ARG, "spmv: mode %u", mode);
  const uint32_t V = g.V;
  if (V == 0) return fail(ERR_ARG, "spmv: empty graph");
  DdWork* w = nullptr;
  OGB_TRY(dd_work_get(g, &w, s));
  const int sms = sm_count();
  spmv_init_kernel<<<sms * 8, kT, 0, s>>>(V, g.fwd.d_out_degree(), x, y);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaEventRecord(w->ev0, s));
  if (mode == 0) {
    const Grid3 G = rows_grid(V);
    SpmvPullPolicy pol{g.inv.d_dst(), g.weighted ? g.inv.d_w() : nullptr, x, y};
    for (uint32_t it = 0; it < iterations; it++)
      spmv_pull_kernel<<<G.total(), kT, 0, s>>>(g.inv.d_rows(), w->med.as<uint32_t>(), w->heavy.as<uint32_t>(),
                                                 G.light, G.med, pol, w->ctl.as<DdCtl>(), V);
  } else {
    for (uint32_t it = 0; it < iterations; it++)
      spmv_push_kernel<<<sms * 8, kT, 0, s>>>(V, g.fwd.d_rows(), g.fwd.d_dst(), g.weighted ? g.fwd.d_w() : nullptr, x,
                                               y, w->och.as<uint4>(), w->ctl.as<DdCtl>());
  }
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaEventRecord(w->ev1, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&ms, w->ev0, w->ev1));
  if (ms_out) *ms_out = ms;
  return OK;
}

int rank_sort(const float* ranks, uint32_t* labels, uint32_t n, cudaStream_t s) {
  if (n == 0) return OK;
  static SortWorkspace* ws = new SortWorkspace();
  DevBuf keys, keys_out, labels_out;
  OGB_TRY(keys.alloc((size_t)n * 4));
  OGB_TRY(keys_out.alloc((size_t)n * 4));
  OGB_TRY(labels_out.alloc((size_t)n * 4));
  const int grid = (int)std::min<uint32_t>(sm_count() * 8, std::max<uint32_t>(1, ceil_div(n, 256)));
  rank_keys_kernel<<<grid, 256, 0, s>>>(n, ranks, keys.as<uint32_t>());
  OGB_CUDA(cudaGetLastError());
  KV in{keys.as<uint32_t>(), labels, nullptr};
  KV out{keys_out.as<uint32_t>(), labels_out.as<uint32_t>(), nullptr};
  OGB_TRY(sort_pairs(in, out, n, *ws, s, 32));
  OGB_TRY(sort_check(*ws, s));
  OGB_CUDA(cudaMemcpyAsync(labels, labels_out.p, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}


// ---- one pull iteration over a range of vertices (1-D partitioned PageRank) --
//
// A rank of a 1-D partition owns the destination vertices [lo, hi) (their
// inverse-CSR rows) and holds the whole contrib vector of the previous
// iteration.  One step: for v in [lo, hi): s = sum of contrib over v's
// in-row (the order above: the same per-row order as the single-GPU pull
// kernel, whatever the partition), rank 0.15 + 0.85 s, contrib_next[v] =
// rank / out_degree (0 without out-edges); |change| / V and the count of
// changes >= epsilon are added to *err / *active.  The caller all-gathers
// contrib_next's slices between steps (pageRank.c:984-1044 per iteration),
// or passes the other ranks' contrib_next buffers as peers: the step then
// stores each owned contrib into every one of them as it is computed (the
// all-gather fused into the step: over NVLink when the peers are other
// GPUs' memory), and the caller only needs a barrier between steps.

namespace {

struct RangeWork {
  uint32_t lo = 0, hi = 0, build = 0;
  bool ready = false;
  DevBuf ctl, med, heavy;
};
std::mutex g_range_mu;
std::vector<std::pair<const DevGraph*, RangeWork*>> g_range;

__global__ void range_count_kernel(uint32_t lo, uint32_t hi, const uint2* __restrict__ rows,
                                   DdCtl* __restrict__ ctl) {
  uint32_t cm = 0, ch = 0;
  for (uint32_t v = lo + blockIdx.x * blockDim.x + threadIdx.x; v < hi; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    cm += (d > kWarpThr && d <= kCtaThr);
    ch += (d > kCtaThr);
  }
  warp_atomic_add_total(&ctl->n_med, cm);
  warp_atomic_add_total(&ctl->n_heavy, ch);
}

__global__ void range_fill_kernel(uint32_t lo, uint32_t hi, const uint2* __restrict__ rows,
                                  uint32_t* __restrict__ med, uint32_t* __restrict__ heavy,
                                  DdCtl* __restrict__ ctl) {
  for (uint32_t v = lo + blockIdx.x * blockDim.x + threadIdx.x; v < hi; v += gridDim.x * blockDim.x) {
    const uint32_t d = rows[v].y;
    if (d > kCtaThr)
      heavy[atomicAdd(&ctl->cur_heavy, 1u)] = v;
    else if (d > kWarpThr)
      med[atomicAdd(&ctl->cur_med, 1u)] = v;
  }
}

struct RangePolicy {
  uint32_t lo;
  const uint32_t* nbr;
  const uint32_t* out_degree;
  const float* contrib;
  float* pr;
  float* contrib_next;
  DdParams p;
  float* const* peers = nullptr;  // fused exchange: contrib_next also stored into each of these
  uint32_t npeers = 0;
  double err = 0.0;
  uint32_t act = 0;
  __device__ bool want(uint32_t) const { return true; }
  __device__ float start(uint32_t) const { return 0.0f; }
  __device__ float term(uint32_t j) const { return contrib[nbr[j] & 0x3FFFFFFFu]; }
  __device__ void finish(uint32_t v, float s) {
    const float nv = __fadd_rn(p.base_pr, __fmul_rn(p.damp, s));
    const float prev = pr[v];
    pr[v] = nv;
    const uint32_t d = out_degree[v];
    const float c = d ? __fdiv_rn(nv, (float)d) : 0.0f;
    contrib_next[v] = c;
    for (uint32_t k = 0; k < npeers; k++) peers[k][v] = c;
    const double e = fabs((double)__fsub_rn(nv, prev));
    err += e / (double)p.V;
    act += (e >= p.epsilon) ? 1u : 0u;
  }
};

// rows_pass over [lo, hi): the light blocks walk [lo, hi), the lists hold
// the range's medium and heavy rows.
__global__ void __launch_bounds__(kT) range_step_kernel(const uint2* __restrict__ rows, uint32_t lo, uint32_t hi,
                                                        const uint32_t* __restrict__ med,
                                                        const uint32_t* __restrict__ heavy, uint32_t nb_light,
                                                        uint32_t nb_med, RangePolicy pol,
                                                        const DdCtl* __restrict__ ctl, double* g_err,
                                                        uint32_t* g_act) {
  // shift the light rows' vertex numbering to the range: rows_pass walks
  // [0, n) of the shifted arrays
  struct Shift {
    RangePolicy& q;
    uint32_t lo;
    __device__ bool want(uint32_t) const { return true; }
    __device__ float start(uint32_t) const { return 0.0f; }
    __device__ float term(uint32_t j) const { return q.term(j); }
    __device__ void finish(uint32_t v, float s) { q.finish(v + lo, s); }
  };
  Shift sh{pol, lo};
  if (blockIdx.x < nb_light) {
    rows_pass(rows + lo, nullptr, nullptr, 0, 0, hi - lo, nb_light, 0, sh);
  } else {
    // medium / heavy lists hold absolute vertex ids: run them unshifted
    rows_pass(rows, med, heavy, ctl->n_med, ctl->n_heavy, 0, nb_light, nb_med, pol);
  }
  // peer stores (other GPUs' memory over NVLink) ordered before anything
  // this thread does after the step, the caller's barrier included
  if (pol.npeers) __threadfence_system();
  double err = pol.err;
  uint32_t act = pol.act;
  __shared__ double s_e[kT / 32];
  __shared__ uint32_t s_a[kT / 32];
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    err += __shfl_down_sync(0xffffffffu, err, o);
    act += __shfl_down_sync(0xffffffffu, act, o);
  }
  if (lane_id() == 0) {
    s_e[threadIdx.x >> 5] = err;
    s_a[threadIdx.x >> 5] = act;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0.0;
    uint32_t a = 0;
    for (uint32_t w = 0; w < kT / 32; w++) {
      e += s_e[w];
      a += s_a[w];
    }
    if (e != 0.0) atomicAdd(g_err, e);
    if (a) atomicAdd(g_act, a);
  }
}

__global__ void range_init_kernel(uint32_t V, const uint32_t* __restrict__ out_degree, float base_pr,
                                  float* __restrict__ pr, float* __restrict__ contrib) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    pr[v] = base_pr;
    const uint32_t d = out_degree[v];
    contrib[v] = d ? __fdiv_rn(base_pr, (float)d) : 0.0f;
  }
}

}  // namespace

void range_work_free(const DevGraph* g) {
  std::lock_guard<std::mutex> lk(g_range_mu);
  for (size_t i = 0; i < g_range.size(); i++) {
    if (g_range[i].first == g) {
      delete g_range[i].second;
      g_range.erase(g_range.begin() + (long)i);
      return;
    }
  }
}

int pagerank_range_init(DevGraph& g, float* ranks, float* contrib, cudaStream_t s) {
  if (g.V == 0) return fail(ERR_ARG, "pagerank range: empty graph");
  const float base = 1.0f - 0.85f;
  range_init_kernel<<<sm_count() * 8, kT, 0, s>>>(g.V, g.fwd.d_out_degree(), base, ranks, contrib);
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int pagerank_range_step(DevGraph& g, uint32_t lo, uint32_t hi, const float* contrib, float* ranks,
                        float* contrib_next, double epsilon, double* d_err, uint32_t* d_active, cudaStream_t s,
                        float* const* peers, uint32_t npeers) {
  if (lo > hi || hi > g.V) return fail(ERR_RANGE, "pagerank range [%u, %u) outside [0, %u)", lo, hi, g.V);
  if (npeers && !peers) return fail(ERR_ARG, "pagerank range: %u peers without their addresses", npeers);
  if (lo == hi) return OK;
  RangeWork* w = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_range_mu);
    for (auto& e : g_range)
      if (e.first == &g) w = e.second;
    if (!w) {
      w = new RangeWork();
      g_range.emplace_back(&g, w);
    }
  }
  DdCtl* ctl = nullptr;
  if (!w->ready || w->lo != lo || w->hi != hi || w->build != g.build_id) {
    OGB_TRY(w->ctl.alloc(sizeof(DdCtl)));
    OGB_TRY(w->med.alloc((size_t)(hi - lo) * 4 + 16));
    OGB_TRY(w->heavy.alloc((size_t)(hi - lo) * 4 + 16));
    ctl = w->ctl.as<DdCtl>();
    OGB_CUDA(cudaMemsetAsync(ctl, 0, sizeof(DdCtl), s));
    const int grid = sm_count() * 8;
    range_count_kernel<<<grid, kT, 0, s>>>(lo, hi, g.inv.d_rows(), ctl);
    range_fill_kernel<<<grid, kT, 0, s>>>(lo, hi, g.inv.d_rows(), w->med.as<uint32_t>(), w->heavy.as<uint32_t>(), ctl);
    OGB_CUDA(cudaGetLastError());
    w->lo = lo;
    w->hi = hi;
    w->build = g.build_id;
    w->ready = true;
  }
  ctl = w->ctl.as<DdCtl>();
  DdParams p;
  p.V = g.V;
  p.damp = 0.85f;
  p.base_pr = 1.0f - p.damp;
  p.epsilon = epsilon;
  RangePolicy pol{lo, g.inv.d_dst(), g.fwd.d_out_degree(), contrib, ranks, contrib_next, p, peers, npeers};
  const Grid3 G = rows_grid(hi - lo);
  range_step_kernel<<<G.total(), kT, 0, s>>>(g.inv.d_rows(), lo, hi, w->med.as<uint32_t>(), w->heavy.as<uint32_t>(),
                                             G.light, G.med, pol, ctl, d_err, d_active);
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int pagerank_range_finish(DevGraph& g, float* ranks, cudaStream_t s) {
  dd_normalize_kernel<<<sm_count() * 8, kT, 0, s>>>(g.V, ranks);
  OGB_CUDA(cudaGetLastError());
  return OK;
}

}  // namespace ogb
