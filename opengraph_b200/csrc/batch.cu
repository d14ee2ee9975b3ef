// batch.cu -- batched traversals over one device graph.
//
// Multi-source BFS (no reference counterpart; each lane must equal the
// reference's single-root BFS depths, BFS.c:476-626): up to 64 searches at
// once, one bit-lane per root.  Per vertex, three 64-bit words: the lanes
// that have visited it, the lanes whose frontier holds it, and the lanes that
// reach it in the level being built.  A level is either
//  * push (top-down): the frontier's out-edges, edge-balanced (a device scan
//    of the frontier vertices' out-degrees, then a warp per 32 consecutive
//    edges, each lane locating its edge's vertex by binary search); each
//    edge ORs the frontier word of its source, minus the target's visited
//    lanes, into the target's next word (64-bit atomicOr);
//  * pull (bottom-up): every vertex with a lane still unvisited ORs the
//    frontier words of its in-neighbours, stopping once every unvisited lane
//    is covered; rows of at most kMsLight in-edges by a thread (four edges
//    per step), longer rows by a warp;
// then one dense pass turns the next words into the new frontier, sets the
// visited lanes, writes the depths of the lanes each vertex gained (a warp
// per vertex row, coalesced) and counts the new frontier and its out-edges
// for the direction choice.
// Depths are u16 per (vertex, lane), row-major by vertex (128 bytes per
// vertex, 0xFFFF = unreached).  The search is level-synchronous in every
// lane, so every lane's depths are those of a single-root BFS.
#include "graph.cuh"

#include <algorithm>
#include <vector>

namespace ogb {

constexpr uint32_t kMsLight = 32;    // pull: rows up to this many in-edges by one thread
constexpr uint32_t kMsAlpha = 14;    // push while the frontier's out-edges < E / kMsAlpha

struct MsCtl {
  uint32_t nlist;              // vertices of the new frontier
  uint32_t pad;
  unsigned long long mf;       // their out-edges
  unsigned long long reached;  // (vertex, lane) pairs reached by the level
  unsigned long long edges;    // edges read by the level
};

struct MsWork {
  uint32_t V = 0, heavy_build = 0;
  bool heavy_ready = false;
  DevBuf F, N, vis, list, cnt, off, heavy, ctl, scan_tmp;
  uint32_t n_heavy = 0;
  MsCtl* h_ctl = nullptr;
  cudaEvent_t ev_init = nullptr, ev0 = nullptr, ev1 = nullptr;
  ~MsWork() {
    if (h_ctl) cudaFreeHost(h_ctl);
    if (ev_init) cudaEventDestroy(ev_init);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

void ms_work_free(MsWork* w) { delete w; }

// ------------------------------------------------------------ kernels ------

__global__ void msk_roots(const uint32_t* __restrict__ verts, const unsigned long long* __restrict__ masks,
                          uint32_t n, unsigned long long* __restrict__ F, unsigned long long* __restrict__ vis,
                          uint16_t* __restrict__ depth, uint32_t* __restrict__ list,
                          const uint32_t* __restrict__ out_degree, MsCtl* __restrict__ ctl) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = verts[i];
    const unsigned long long m = masks[i];
    F[v] = m;
    vis[v] = m;
    list[i] = v;
    unsigned long long b = m;
    while (b) {
      const int lane = __ffsll((long long)b) - 1;
      depth[(size_t)v * 64 + lane] = 0;
      b &= b - 1;
    }
    atomicAdd(&ctl->mf, (unsigned long long)out_degree[v]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->nlist = n;
}

// push: out-degree of each frontier vertex (scanned into edge offsets)
__global__ void msk_frontier_degree(const uint32_t* __restrict__ list, uint32_t n, const uint2* __restrict__ rows,
                                    uint32_t* __restrict__ cnt) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    cnt[i] = rows[list[i]].y;
}

// push, a frontier list of at most kMsSmallScan entries: its out-degrees
// scanned by one CTA (entry i's first edge in off[i], the total in off[n]) --
// one launch instead of a degree pass and a three-kernel device scan.
constexpr uint32_t kMsSmallScan = 8192;
__global__ void __launch_bounds__(1024) msk_small_scan(const uint32_t* __restrict__ list, uint32_t n,
                                                        const uint2* __restrict__ rows, uint32_t* __restrict__ off) {
  constexpr uint32_t K = kMsSmallScan / 1024;  // entries per thread
  __shared__ uint32_t s_w[32];
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t d[K], sum = 0;
#pragma unroll
  for (uint32_t k = 0; k < K; k++) {
    const uint32_t i = threadIdx.x * K + k;
    d[k] = i < n ? rows[list[i]].y : 0u;
    sum += d[k];
  }
  uint32_t x = sum;
#pragma unroll
  for (uint32_t o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_w[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = s_w[lane];
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    s_w[lane] = t;  // inclusive warp totals
  }
  __syncthreads();
  uint32_t e = (warp ? s_w[warp - 1] : 0u) + x - sum;
#pragma unroll
  for (uint32_t k = 0; k < K; k++) {
    const uint32_t i = threadIdx.x * K + k;
    if (i < n) off[i] = e;
    e += d[k];
  }
  if (threadIdx.x == blockDim.x - 1) off[n] = e;  // the list's out-edges
}

// push: the frontier's out-edges, edge-balanced: a warp takes 32 consecutive
// edges of the frontier's edge range; lane 0 finds the first edge's vertex
// by binary search over the offsets, each lane then its own edge's vertex
// from there.
__global__ void __launch_bounds__(256) msk_push(const uint32_t* __restrict__ list, uint32_t n,
                                                const uint32_t* __restrict__ off, const uint2* __restrict__ rows,
                                                const uint32_t* __restrict__ nbr,
                                                const unsigned long long* __restrict__ F,
                                                const unsigned long long* __restrict__ vis,
                                                unsigned long long* __restrict__ N, MsCtl* __restrict__ ctl) {
  const uint32_t lane = lane_id();
  const uint32_t total = off[n];
  const uint32_t gw = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x / 32);
  for (uint32_t e0 = gw * 32; e0 < total; e0 += nw * 32) {
    uint32_t i0 = 0;
    if (lane == 0) {
      uint32_t lo = 0, hi = n - 1;  // last i with off[i] <= e0
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= e0)
          lo = mid;
        else
          hi = mid - 1;
      }
      i0 = lo;
    }
    i0 = __shfl_sync(0xffffffffu, i0, 0);
    const uint32_t e = e0 + lane;
    if (e < total) {
      uint32_t lo = i0, hi = n - 1;  // entries without out-edges share an offset, so no tighter bound
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= e)
          lo = mid;
        else
          hi = mid - 1;
      }
      const uint32_t u = list[lo];
      const uint32_t w = __ldg(&nbr[rows[u].x + (e - off[lo])]) & 0x3FFFFFFFu;
      const unsigned long long m = F[u] & ~vis[w];
      if (m) atomicOr(&N[w], m);
    }
  }
  if (gw == 0 && lane == 0) atomicAdd(&ctl->edges, (unsigned long long)total);
}

// pull, light rows: a thread per vertex, four in-edges per step, stop once
// every unvisited lane is covered
__global__ void __launch_bounds__(256) msk_pull_light(uint32_t V, unsigned long long lanes,
                                                      const uint2* __restrict__ rows, const uint32_t* __restrict__ nbr,
                                                      const unsigned long long* __restrict__ F,
                                                      const unsigned long long* __restrict__ vis,
                                                      unsigned long long* __restrict__ N, MsCtl* __restrict__ ctl) {
  uint32_t edges = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const unsigned long long pending = lanes & ~vis[v];
    if (!pending) continue;
    const uint2 r = rows[v];
    if (r.y == 0 || r.y > kMsLight) continue;
    unsigned long long acc = 0;
    uint32_t j = r.x;
    const uint32_t end = r.x + r.y;
    for (; j < end; j += 4) {
      unsigned long long f[4];
#pragma unroll
      for (int k = 0; k < 4; k++) f[k] = (j + k < end) ? F[__ldg(&nbr[j + k]) & 0x3FFFFFFFu] : 0ull;
      acc |= f[0] | f[1] | f[2] | f[3];
      if ((acc & pending) == pending) {
        j += 4;
        break;
      }
    }
    edges += min(j, end) - r.x;
    const unsigned long long n = acc & pending;
    if (n) N[v] = n;
  }
  warp_atomic_add_total64(&ctl->edges, edges);
}

// pull, long rows: a warp per vertex of the heavy list, lanes strided, the
// warp's OR checked every 128 edges
__global__ void __launch_bounds__(256) msk_pull_heavy(const uint32_t* __restrict__ heavy, uint32_t n_heavy,
                                                      unsigned long long lanes, const uint2* __restrict__ rows,
                                                      const uint32_t* __restrict__ nbr,
                                                      const unsigned long long* __restrict__ F,
                                                      const unsigned long long* __restrict__ vis,
                                                      unsigned long long* __restrict__ N, MsCtl* __restrict__ ctl) {
  const uint32_t lane = lane_id();
  const uint32_t gw = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x / 32);
  uint32_t edges = 0;
  for (uint32_t t = gw; t < n_heavy; t += nw) {
    const uint32_t v = heavy[t];
    const unsigned long long pending = lanes & ~vis[v];
    if (!pending) continue;
    const uint2 r = rows[v];
    const uint32_t end = r.x + r.y;
    unsigned long long acc = 0;
    uint32_t j = r.x;
    for (; j < end; j += 128) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint32_t jj = j + k * 32 + lane;
        if (jj < end) acc |= F[__ldg(&nbr[jj]) & 0x3FFFFFFFu];
      }
      // the warp's OR
      unsigned int lo = (unsigned int)acc, hi = (unsigned int)(acc >> 32);
      lo = __reduce_or_sync(0xffffffffu, lo);
      hi = __reduce_or_sync(0xffffffffu, hi);
      acc = ((unsigned long long)hi << 32) | lo;
      if ((acc & pending) == pending) {
        j += 128;
        break;
      }
    }
    if (lane == 0) {
      edges += min(j, end) - r.x;
      const unsigned long long n = acc & pending;
      if (n) N[v] = n;
    }
  }
  if (lane == 0 && edges) atomicAdd(&ctl->edges, (unsigned long long)edges);
}

// Next words -> new frontier: visited lanes, the depths of the newly reached
// lanes, the frontier list and its out-edges.  N is left all zero.  A warp
// covers 32 consecutive vertices; for each of them that gained lanes, the
// whole warp writes its depths (lane l: depth lanes l and l + 32 of the
// vertex's 128-byte row, 2-byte stores, no read -- every (vertex, lane) is
// written once).
__global__ void __launch_bounds__(256) msk_finish(uint32_t V, uint16_t level, unsigned long long* __restrict__ F,
                                                  unsigned long long* __restrict__ N,
                                                  unsigned long long* __restrict__ vis,
                                                  uint16_t* __restrict__ depth, const uint32_t* __restrict__ out_degree,
                                                  uint32_t* __restrict__ list, MsCtl* __restrict__ ctl) {
  __shared__ BlockAppend<1024> q;
  __shared__ unsigned long long s_red[8];
  ba_init(q);
  const uint32_t lane = lane_id();
  unsigned long long mf = 0, reached = 0;
  for (uint32_t base = blockIdx.x * 1024; base < V; base += gridDim.x * 1024) {
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) {
      const uint32_t w0 = base + k * 256 + (threadIdx.x & ~31u);
      const uint32_t v = w0 + lane;
      unsigned long long n = 0;
      if (v < V) {
        const unsigned long long nx = N[v];
        if (nx) {
          const unsigned long long vi = vis[v];
          n = nx & ~vi;
          N[v] = 0;
          if (n) {
            vis[v] = vi | n;
            mf += out_degree[v];
            reached += (unsigned long long)__popcll(n);
            ba_push(q, v);
          }
        }
        F[v] = n;
      }
      uint32_t has = __ballot_sync(0xffffffffu, n != 0);
      while (has) {
        const uint32_t j = (uint32_t)__ffs(has) - 1;
        has &= has - 1;
        const unsigned long long f = __shfl_sync(0xffffffffu, n, j);
        uint16_t* row = depth + (size_t)(w0 + j) * 64;
        if ((f >> lane) & 1ull) row[lane] = level;
        if ((f >> (lane + 32)) & 1ull) row[lane + 32] = level;
      }
    }
    ba_flush(q, list, &ctl->nlist);
  }
  block_add_total<unsigned long long>(&ctl->mf, mf, s_red);
  block_add_total<unsigned long long>(&ctl->reached, reached, s_red);
}

// vertices with more than kMsLight in-edges (built once per graph)
__global__ void msk_heavy_list(uint32_t V, const uint2* __restrict__ rows, uint32_t* __restrict__ heavy,
                               uint32_t* __restrict__ count) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    if (rows[v].y > kMsLight) heavy[warp_atomic_inc(count)] = v;
}

// ------------------------------------------------------------ driver -------

static int ms_work_get(DevGraph& g, MsWork** out, cudaStream_t s) {
  if (!g.ms) g.ms = new MsWork();
  MsWork* w = g.ms;
  const uint32_t V = g.V;
  if (w->V != V || !w->F.p) {
    OGB_TRY(w->F.alloc((size_t)V * 8 + 16));
    OGB_TRY(w->N.alloc((size_t)V * 8 + 16));
    OGB_TRY(w->vis.alloc((size_t)V * 8 + 16));
    OGB_TRY(w->list.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->cnt.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->off.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->heavy.alloc((size_t)V * 4 + 16));
    OGB_TRY(w->scan_tmp.alloc(scan_tmp_words(V) * 4));
    OGB_TRY(w->ctl.alloc(sizeof(MsCtl) + 16));
    w->V = V;
    w->heavy_ready = false;
  }
  if (!w->h_ctl) OGB_CUDA(cudaMallocHost(&w->h_ctl, sizeof(MsCtl)));
  if (!w->ev0) {
    OGB_CUDA(cudaEventCreate(&w->ev_init));
    OGB_CUDA(cudaEventCreate(&w->ev0));
    OGB_CUDA(cudaEventCreate(&w->ev1));
  }
  if (!w->heavy_ready || w->heavy_build != g.build_id) {
    uint32_t* c = w->ctl.as<uint32_t>();
    OGB_CUDA(cudaMemsetAsync(c, 0, 4, s));
    msk_heavy_list<<<sm_count() * 8, 256, 0, s>>>(V, g.inv.d_rows(), w->heavy.as<uint32_t>(), c);
    OGB_CUDA(cudaGetLastError());
    OGB_CUDA(cudaMemcpyAsync(&w->n_heavy, c, 4, cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaStreamSynchronize(s));
    w->heavy_ready = true;
    w->heavy_build = g.build_id;
  }
  *out = w;
  return OK;
}

int msbfs_run(DevGraph& g, const uint32_t* roots, uint32_t nroots, uint16_t* depth, MsResult* res,
              cudaStream_t s) {
  const uint32_t V = g.V;
  if (nroots == 0 || nroots > 64) return fail(ERR_ARG, "msbfs: %u roots (1..64)", nroots);
  for (uint32_t i = 0; i < nroots; i++)
    if (roots[i] >= V) return fail(ERR_ARG, "msbfs: root %u out of range (V=%u)", roots[i], V);
  MsWork* w = nullptr;
  OGB_TRY(ms_work_get(g, &w, s));
  // distinct root vertices and their lanes
  std::vector<uint32_t> verts;
  std::vector<unsigned long long> masks;
  for (uint32_t i = 0; i < nroots; i++) {
    auto it = std::find(verts.begin(), verts.end(), roots[i]);
    if (it == verts.end()) {
      verts.push_back(roots[i]);
      masks.push_back(1ull << i);
    } else {
      masks[it - verts.begin()] |= 1ull << i;
    }
  }
  const unsigned long long lanes = nroots == 64 ? ~0ull : ((1ull << nroots) - 1);
  DevBuf d_roots;
  OGB_TRY(d_roots.alloc(verts.size() * 12 + 32));
  uint32_t* d_verts = d_roots.as<uint32_t>();
  unsigned long long* d_masks = reinterpret_cast<unsigned long long*>(d_roots.as<char>() + ((verts.size() * 4 + 15) & ~15ull));
  OGB_CUDA(cudaMemcpyAsync(d_verts, verts.data(), verts.size() * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(d_masks, masks.data(), masks.size() * 8, cudaMemcpyHostToDevice, s));

  const int sms = sm_count();
  unsigned long long* F = w->F.as<unsigned long long>();
  unsigned long long* N = w->N.as<unsigned long long>();
  unsigned long long* vis = w->vis.as<unsigned long long>();
  MsCtl* ctl = w->ctl.as<MsCtl>();
  const uint2* rows_f = g.fwd.d_rows();
  const uint2* rows_i = g.inv.d_rows();

  // initialisation (timed apart, as the single-root search's precedes its
  // timed part): depths unreached, per-vertex words cleared, the roots set
  OGB_CUDA(cudaEventRecord(w->ev_init, s));
  OGB_CUDA(cudaMemsetAsync(depth, 0xFF, (size_t)V * 64 * 2, s));
  OGB_CUDA(cudaMemsetAsync(F, 0, (size_t)V * 8, s));
  OGB_CUDA(cudaMemsetAsync(N, 0, (size_t)V * 8, s));
  OGB_CUDA(cudaMemsetAsync(vis, 0, (size_t)V * 8, s));
  OGB_CUDA(cudaMemsetAsync(ctl, 0, sizeof(MsCtl), s));
  msk_roots<<<1, 64, 0, s>>>(d_verts, d_masks, (uint32_t)verts.size(), F, vis, depth, w->list.as<uint32_t>(),
                             g.fwd.d_out_degree(), ctl);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaEventRecord(w->ev0, s));
  OGB_CUDA(cudaMemcpyAsync(w->h_ctl, ctl, sizeof(MsCtl), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  uint32_t nlist = w->h_ctl->nlist;
  unsigned long long mf = w->h_ctl->mf;
  MsResult r;
  r.reached = verts.size() ? __builtin_popcountll(lanes) : 0;
  uint32_t level = 0, launches = 6;
  while (nlist > 0) {
    if (level >= 0xFFFE) return fail(ERR_UNSUPPORTED, "msbfs: more than 65534 levels");
    level++;
    OGB_CUDA(cudaMemsetAsync(ctl, 0, sizeof(MsCtl), s));
    const bool push = mf < (unsigned long long)g.E / kMsAlpha;
    if (push) {
      if (nlist <= kMsSmallScan) {
        msk_small_scan<<<1, 1024, 0, s>>>(w->list.as<uint32_t>(), nlist, rows_f, w->off.as<uint32_t>());
        launches += 1;
      } else {
        msk_frontier_degree<<<std::min<uint32_t>(sms * 8, ceil_div(nlist, 256)), 256, 0, s>>>(
            w->list.as<uint32_t>(), nlist, rows_f, w->cnt.as<uint32_t>());
        OGB_TRY(scan_exclusive_u32(w->cnt.as<uint32_t>(), w->off.as<uint32_t>(), nlist, w->scan_tmp.as<uint32_t>(),
                                   s));
        launches += 4;
      }
      msk_push<<<sms * 8, 256, 0, s>>>(w->list.as<uint32_t>(), nlist, w->off.as<uint32_t>(), rows_f, g.fwd.d_dst(), F,
                                      vis, N, ctl);
      launches += 1;
      r.push_levels++;
    } else {
      msk_pull_light<<<sms * 8, 256, 0, s>>>(V, lanes, rows_i, g.inv.d_dst(), F, vis, N, ctl);
      if (w->n_heavy)
        msk_pull_heavy<<<sms * 8, 256, 0, s>>>(w->heavy.as<uint32_t>(), w->n_heavy, lanes, rows_i, g.inv.d_dst(), F,
                                              vis, N, ctl);
      launches += 2;
      r.pull_levels++;
    }
    msk_finish<<<sms * 8, 256, 0, s>>>(V, (uint16_t)level, F, N, vis, depth, g.fwd.d_out_degree(),
                                       w->list.as<uint32_t>(), ctl);
    OGB_CUDA(cudaGetLastError());
    OGB_CUDA(cudaMemcpyAsync(w->h_ctl, ctl, sizeof(MsCtl), cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaStreamSynchronize(s));
    launches += 2;
    nlist = w->h_ctl->nlist;
    mf = w->h_ctl->mf;
    r.reached += w->h_ctl->reached;
    r.edges_examined += w->h_ctl->edges;
  }
  OGB_CUDA(cudaEventRecord(w->ev1, s));
  OGB_CUDA(cudaEventSynchronize(w->ev1));
  float ms = 0.f, init_ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&ms, w->ev0, w->ev1));
  OGB_CUDA(cudaEventElapsedTime(&init_ms, w->ev_init, w->ev0));
  r.levels = level;
  r.ms = ms;
  r.init_ms = init_ms;
  r.launches = launches;
  if (res) *res = r;
  return OK;
}


// ===========================================================================
// Batched personalized PageRank (no reference counterpart: the reference's
// pull PageRank, pageRank.c:984-1044, with the teleport term base_pr
// replaced by (1 - d) on the seed vertex only, one vector per seed).  Up to
// 32 seeds at once; ranks are row-major by vertex, 32 floats (128 bytes) per
// vertex, so every in-edge gathers one full cache line: the 32 contribs of
// its source.  Per iteration, for every vertex v and seed k:
//   s_k = sum of c_k[u] over the in-edges (u, v)
//   r'_k[v] = (v == seed_k ? 1 - d : 0) + d * s_k,  c'_k[v] = r'_k[v] / out_degree(v)
//   err_k += |r'_k[v] - r_k[v]|   (fp64)
// starting from r_k = e_seed_k; the run stops when every seed's err_k is
// below epsilon, or after max_iterations.  A warp takes a vertex (or a chunk
// of a long row): its four 8-lane groups walk the row's edges in turn, each
// lane owning 4 seeds (one float4 of the row), four edges per group in
// flight; the groups' sums are folded at the end.  Rows longer than
// kPprChunk edges are cut into chunks (handed out one per claim, before the
// other vertices, 64 per claim) whose sums the warp finishing the last one
// adds in chunk order.  Dangling vertices' rank is not redistributed,
// as in the reference.
// ===========================================================================

constexpr uint32_t kPprSeeds = 32;
constexpr uint32_t kPprChunk = 512;
constexpr uint32_t kPprMaxIters = 1024;

struct PprCtl {
  double err[kPprMaxIters][kPprSeeds];
  uint32_t stop, stop_iter;
  uint32_t claim_chunk[kPprMaxIters];  // chunks handed out, one per claim
  uint32_t claim_row[kPprMaxIters];    // other vertices handed out, 64 per claim
};

struct PprChunk {
  uint32_t v, j0, j1, k;  // vertex, edge range, index of the vertex among the chunked ones
};

struct PprWork {
  uint32_t V = 0, build = 0;
  bool ready = false;
  DevBuf R, C0, C1, ctl, chunks, vfirst, vcount, done, partials, light;
  uint32_t n_chunks = 0, n_cut = 0, n_light = 0;
  PprCtl* h_ctl = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~PprWork() {
    if (h_ctl) cudaFreeHost(h_ctl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

void ppr_work_free(PprWork* w) { delete w; }

__global__ void pprk_seed(const uint32_t* __restrict__ seeds, uint32_t nseeds, const uint32_t* __restrict__ out_degree,
                          float* __restrict__ R, float* __restrict__ C) {
  const uint32_t k = threadIdx.x;
  if (k < nseeds) {
    const uint32_t v = seeds[k];
    R[(size_t)v * kPprSeeds + k] = 1.0f;
    const uint32_t d = out_degree[v];
    C[(size_t)v * kPprSeeds + k] = d ? __fdiv_rn(1.0f, (float)d) : 0.0f;
  }
}

// Sum of the 32-float contrib rows of in-edges [j0, j1) (each lane: 4 seeds):
// group g of 8 lanes takes edges g, g+4, g+8, g+12, then the next 16, four
// rows in flight per group; the four groups are folded at the end.
__device__ __forceinline__ float4 ppr_row_sum(const uint32_t* __restrict__ nbr, const float4* __restrict__ C4,
                                              uint32_t j0, uint32_t j1, uint32_t grp, uint32_t sub) {
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (uint32_t j = j0 + grp; j < j1; j += 16) {
    uint32_t u[4];
#pragma unroll
    for (int q = 0; q < 4; q++) u[q] = (j + 4 * q < j1) ? (__ldg(&nbr[j + 4 * q]) & 0x3FFFFFFFu) : 0xFFFFFFFFu;
    float4 c[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      c[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (u[q] != 0xFFFFFFFFu) c[q] = __ldg(&C4[(size_t)u[q] * 8 + sub]);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      acc.x += c[q].x;
      acc.y += c[q].y;
      acc.z += c[q].z;
      acc.w += c[q].w;
    }
  }
  // fold the four groups (lanes sub, sub + 8, sub + 16, sub + 24)
#pragma unroll
  for (int o = 8; o < 32; o <<= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
    acc.z += __shfl_xor_sync(0xffffffffu, acc.z, o);
    acc.w += __shfl_xor_sync(0xffffffffu, acc.w, o);
  }
  return acc;
}

struct PprParams {
  float damp, base;
  double eps;
  uint32_t nseeds;
  const uint32_t* seeds;
};

// Update of vertex v from its sums (lanes 0..7 hold seeds 4l..4l+3).
__device__ __forceinline__ void ppr_update(uint32_t v, float4 s, uint32_t sub, const PprParams& p,
                                           const uint32_t* __restrict__ out_degree, float* __restrict__ R,
                                           float* __restrict__ Cn, double* err4) {
  const uint32_t d = out_degree[v];
  float4* R4 = reinterpret_cast<float4*>(R) + (size_t)v * 8 + sub;
  float4* C4 = reinterpret_cast<float4*>(Cn) + (size_t)v * 8 + sub;
  const float4 old = *R4;
  float sv[4] = {s.x, s.y, s.z, s.w}, ov[4] = {old.x, old.y, old.z, old.w}, nv[4], cv[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const uint32_t k = sub * 4 + i;
    const float tele = (k < p.nseeds && p.seeds[k] == v) ? p.base : 0.0f;
    nv[i] = __fadd_rn(tele, __fmul_rn(p.damp, sv[i]));
    cv[i] = d ? __fdiv_rn(nv[i], (float)d) : 0.0f;
    err4[i] += fabs((double)nv[i] - (double)ov[i]);
  }
  *R4 = make_float4(nv[0], nv[1], nv[2], nv[3]);
  *C4 = make_float4(cv[0], cv[1], cv[2], cv[3]);
}

__global__ void __launch_bounds__(256) pprk_iter(const PprChunk* __restrict__ chunks, uint32_t n_chunks,
                                                 const uint32_t* __restrict__ vfirst,
                                                 const uint32_t* __restrict__ vcount, uint32_t* __restrict__ done,
                                                 float4* __restrict__ partials, const uint32_t* __restrict__ light,
                                                 uint32_t n_light, const uint2* __restrict__ rows,
                                                 const uint32_t* __restrict__ nbr,
                                                 const uint32_t* __restrict__ out_degree, const float* __restrict__ C,
                                                 float* __restrict__ Cn, float* __restrict__ R, PprParams p,
                                                 PprCtl* __restrict__ ctl, uint32_t it) {
  __shared__ double s_err[8][kPprSeeds];
  if (ctl->stop) return;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t grp = lane >> 3, sub = lane & 7;
  const float4* C4 = reinterpret_cast<const float4*>(C);
  double err4[4] = {0, 0, 0, 0};
  // chunks of long rows, one per claim
  for (;;) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(&ctl->claim_chunk[it], 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_chunks) break;
    const PprChunk ci = chunks[t];
    const float4 s = ppr_row_sum(nbr, C4, ci.j0, ci.j1, grp, sub);
    uint32_t last = 0;
    if (lane < 8) partials[(size_t)t * 8 + sub] = s;
    __threadfence();
    __syncwarp();
    if (lane == 0) last = (atomicAdd(&done[ci.k], 1u) == vcount[ci.k] - 1) ? 1u : 0u;
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
      __threadfence();
      const uint32_t f = vfirst[ci.k], cnt = vcount[ci.k];
      float4 tot = make_float4(0.f, 0.f, 0.f, 0.f);
      for (uint32_t c = 0; c < cnt; c++) {
        const float4 q = __ldcg(&partials[(size_t)(f + c) * 8 + sub]);
        tot.x += q.x;
        tot.y += q.y;
        tot.z += q.z;
        tot.w += q.w;
      }
      if (lane < 8) ppr_update(ci.v, tot, sub, p, out_degree, R, Cn, err4);
      if (lane == 0) done[ci.k] = 0;
    }
  }
  // the other vertices, 64 per claim
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&ctl->claim_row[it], 64u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n_light) break;
    const uint32_t end = min(base + 64, n_light);
    for (uint32_t t = base; t < end; t++) {
      const uint32_t v = light[t];
      const uint2 r = rows[v];
      const float4 s = ppr_row_sum(nbr, C4, r.x, r.x + r.y, grp, sub);
      if (lane < 8) ppr_update(v, s, sub, p, out_degree, R, Cn, err4);
    }
  }
  // per-seed error: lanes 0..7 hold seeds 4l..4l+3
  if (lane < 8)
    for (int i = 0; i < 4; i++) s_err[warp][lane * 4 + i] = err4[i];
  __syncthreads();
  if (threadIdx.x < kPprSeeds) {
    double e = 0.0;
    for (int w = 0; w < 8; w++) e += s_err[w][threadIdx.x];
    if (e != 0.0) atomicAdd(&ctl->err[it][threadIdx.x], e);
  }
}

// the run stops after an iteration in which every seed changed by < eps (L1)
__global__ void pprk_check(PprCtl* __restrict__ ctl, uint32_t it, uint32_t nseeds, double eps) {
  if (threadIdx.x != 0 || ctl->stop) return;
  bool all = true;
  for (uint32_t k = 0; k < nseeds; k++) all = all && (ctl->err[it][k] < eps);
  if (all) {
    ctl->stop = 1;
    ctl->stop_iter = it;
  }
}

static int ppr_work_get(DevGraph& g, PprWork** out, cudaStream_t s) {
  if (!g.ppr) g.ppr = new PprWork();
  PprWork* w = g.ppr;
  const uint32_t V = g.V;
  if (w->V != V || !w->R.p) {
    OGB_TRY(w->R.alloc((size_t)V * kPprSeeds * 4 + 64));
    OGB_TRY(w->C0.alloc((size_t)V * kPprSeeds * 4 + 64));
    OGB_TRY(w->C1.alloc((size_t)V * kPprSeeds * 4 + 64));
    OGB_TRY(w->ctl.alloc(sizeof(PprCtl) + 64));
    w->V = V;
    w->ready = false;
  }
  if (!w->h_ctl) OGB_CUDA(cudaMallocHost(&w->h_ctl, sizeof(PprCtl)));
  if (!w->ev0) {
    OGB_CUDA(cudaEventCreate(&w->ev0));
    OGB_CUDA(cudaEventCreate(&w->ev1));
  }
  if (!w->ready || w->build != g.build_id) {
    // rows from the inverse CSR: rows over kPprChunk in-edges become chunks
    const uint2* rows = g.inv.d_rows();
    std::vector<uint2> h_rows(V);
    OGB_CUDA(cudaMemcpyAsync(h_rows.data(), rows, (size_t)V * 8, cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> light;
    std::vector<PprChunk> chunks;
    std::vector<uint32_t> first, count;
    light.reserve(V);
    for (uint32_t v = 0; v < V; v++) {
      const uint2 r = h_rows[v];
      if (r.y > kPprChunk) {
        const uint32_t k = (uint32_t)first.size();
        first.push_back((uint32_t)chunks.size());
        for (uint32_t c = 0; c < r.y; c += kPprChunk) chunks.push_back({v, r.x + c, r.x + std::min(r.y, c + kPprChunk), k});
        count.push_back((uint32_t)chunks.size() - first.back());
      } else {
        light.push_back(v);
      }
    }
    w->n_light = (uint32_t)light.size();
    w->n_chunks = (uint32_t)chunks.size();
    w->n_cut = (uint32_t)first.size();
    OGB_TRY(w->light.alloc((size_t)w->n_light * 4 + 16));
    OGB_TRY(w->chunks.alloc((size_t)w->n_chunks * sizeof(PprChunk) + 16));
    OGB_TRY(w->partials.alloc((size_t)w->n_chunks * kPprSeeds * 4 + 16));
    OGB_TRY(w->vfirst.alloc((size_t)w->n_cut * 4 + 16));
    OGB_TRY(w->vcount.alloc((size_t)w->n_cut * 4 + 16));
    OGB_TRY(w->done.alloc((size_t)w->n_cut * 4 + 16));
    if (w->n_light) OGB_CUDA(cudaMemcpyAsync(w->light.p, light.data(), light.size() * 4, cudaMemcpyHostToDevice, s));
    if (w->n_chunks)
      OGB_CUDA(cudaMemcpyAsync(w->chunks.p, chunks.data(), chunks.size() * sizeof(PprChunk), cudaMemcpyHostToDevice, s));
    if (w->n_cut) {
      OGB_CUDA(cudaMemcpyAsync(w->vfirst.p, first.data(), first.size() * 4, cudaMemcpyHostToDevice, s));
      OGB_CUDA(cudaMemcpyAsync(w->vcount.p, count.data(), count.size() * 4, cudaMemcpyHostToDevice, s));
    }
    OGB_CUDA(cudaMemsetAsync(w->done.p, 0, (size_t)w->n_cut * 4 + 16, s));
    OGB_CUDA(cudaStreamSynchronize(s));
    w->ready = true;
    w->build = g.build_id;
  }
  *out = w;
  return OK;
}

int ppr_run(DevGraph& g, const uint32_t* seeds, uint32_t nseeds, uint32_t max_iters, double epsilon, float* ranks,
            PprResult* res, cudaStream_t s) {
  const uint32_t V = g.V;
  if (nseeds == 0 || nseeds > kPprSeeds) return fail(ERR_ARG, "ppr: %u seeds (1..%u)", nseeds, kPprSeeds);
  if (max_iters > kPprMaxIters) return fail(ERR_ARG, "ppr: at most %u iterations", kPprMaxIters);
  for (uint32_t i = 0; i < nseeds; i++)
    if (seeds[i] >= V) return fail(ERR_ARG, "ppr: seed %u out of range (V=%u)", seeds[i], V);
  PprWork* w = nullptr;
  OGB_TRY(ppr_work_get(g, &w, s));
  DevBuf d_seeds;
  OGB_TRY(d_seeds.alloc(kPprSeeds * 4));
  OGB_CUDA(cudaMemcpyAsync(d_seeds.p, seeds, nseeds * 4, cudaMemcpyHostToDevice, s));
  PprCtl* ctl = w->ctl.as<PprCtl>();
  float* C = w->C0.as<float>();
  float* Cn = w->C1.as<float>();
  float* R = w->R.as<float>();
  PprParams p;
  p.damp = 0.85f;
  p.base = 1.0f - p.damp;
  p.eps = epsilon;
  p.nseeds = nseeds;
  p.seeds = d_seeds.as<uint32_t>();
  const int sms = sm_count();
  OGB_CUDA(cudaEventRecord(w->ev0, s));
  OGB_CUDA(cudaMemsetAsync(ctl, 0, sizeof(PprCtl), s));
  OGB_CUDA(cudaMemsetAsync(R, 0, (size_t)V * kPprSeeds * 4, s));
  OGB_CUDA(cudaMemsetAsync(C, 0, (size_t)V * kPprSeeds * 4, s));
  pprk_seed<<<1, 32, 0, s>>>(p.seeds, nseeds, g.fwd.d_out_degree(), R, C);
  OGB_CUDA(cudaGetLastError());
  for (uint32_t it = 0; it < max_iters; it++) {
    pprk_iter<<<sms * 8, 256, 0, s>>>(w->chunks.as<PprChunk>(), w->n_chunks, w->vfirst.as<uint32_t>(),
                                      w->vcount.as<uint32_t>(), w->done.as<uint32_t>(), w->partials.as<float4>(),
                                      w->light.as<uint32_t>(), w->n_light, g.inv.d_rows(), g.inv.d_dst(),
                                      g.fwd.d_out_degree(), C, Cn, R, p, ctl, it);
    pprk_check<<<1, 32, 0, s>>>(ctl, it, nseeds, epsilon);
    OGB_CUDA(cudaGetLastError());
    std::swap(C, Cn);
  }
  OGB_CUDA(cudaEventRecord(w->ev1, s));
  if (ranks) OGB_CUDA(cudaMemcpyAsync(ranks, R, (size_t)V * kPprSeeds * 4, cudaMemcpyDeviceToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(w->h_ctl, ctl, sizeof(PprCtl), cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&ms, w->ev0, w->ev1));
  PprResult r;
  r.ms = ms;
  r.executed = w->h_ctl->stop ? w->h_ctl->stop_iter + 1 : max_iters;
  r.converged = w->h_ctl->stop;
  r.launches = 2 + 2 * max_iters;
  for (uint32_t k = 0; k < nseeds; k++) r.err_last[k] = r.executed ? w->h_ctl->err[r.executed - 1][k] : 0.0;
  if (res) *res = r;
  return OK;
}


// ===========================================================================
// Many graphs in one launch (no reference counterpart: each graph's results
// equal the reference path run on that graph alone).  The graphs are packed
// into one disjoint union (vertex ids shifted by each graph's offset, one
// sort builds every graph's CSR side by side), so the single-graph kernels
// and their load balancing serve the whole batch:
//  * BFS: one search from every graph's root at once -- one cooperative
//    launch for the whole batch; each vertex gets its depth from its own
//    graph's root (no edges cross graphs); parents are returned in local ids;
//  * PageRank pull: every graph keeps its own stop rule and normalization
//    (a per-graph reduction after each iteration freezes a graph whose
//    vertices all changed by < epsilon); the whole run is one CUDA graph.
// ===========================================================================

struct GraphBatch {
  DevGraph g;
  uint32_t ngraphs = 0;
  std::vector<uint32_t> voff;  // host copy of the vertex offsets
  DevBuf d_voff, d_eoff, gid, frozen, stop_iter, executed, active_last, err_last, delta;
  cudaGraphExec_t pr_exec = nullptr;
  uint32_t pr_iters = 0, pr_warp = 0, pr_cta = 0, pr_build = 0;
  double pr_eps = -1.0;
  float* pr_ranks = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~GraphBatch() {
    if (pr_exec) cudaGraphExecDestroy(pr_exec);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

GraphBatch* batch_new() { return new GraphBatch(); }
void batch_free(GraphBatch* b) { delete b; }
uint32_t batch_ngraphs(const GraphBatch* b) { return b->ngraphs; }
const uint32_t* batch_voff(const GraphBatch* b) { return b->voff.data(); }
DevGraph& batch_graph(GraphBatch* b) { return b->g; }

// local ids -> union ids (edge e of graph g: + voff[g]); an id outside its
// graph sets *err
__global__ void bk_shift(uint64_t E, const uint64_t* __restrict__ eoff, const uint32_t* __restrict__ voff,
                         uint32_t ng, uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t* err) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = ng - 1;  // last g with eoff[g] <= e
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (eoff[mid] <= e)
        lo = mid;
      else
        hi = mid - 1;
    }
    const uint32_t n = voff[lo + 1] - voff[lo];
    if (src[e] >= n || dst[e] >= n) *err = 1;
    src[e] += voff[lo];
    dst[e] += voff[lo];
  }
}

__global__ void bk_gid(uint32_t V, const uint32_t* __restrict__ voff, uint32_t ng, uint32_t* __restrict__ gid) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = ng - 1;  // last g with voff[g] <= v
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (voff[mid] <= v)
        lo = mid;
      else
        hi = mid - 1;
    }
    gid[v] = lo;
  }
}

__global__ void bk_localize(uint32_t V, const uint32_t* __restrict__ gid, const uint32_t* __restrict__ voff,
                            int32_t* __restrict__ parents) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const int32_t p = parents[v];
    if (p >= 0) parents[v] = p - (int32_t)voff[gid[v]];
  }
}

int batch_create(GraphBatch& b, uint32_t ngraphs, const uint32_t* nv, const uint64_t* eoff, const uint32_t* src,
                 const uint32_t* dst, uint32_t sort_type, cudaStream_t s) {
  if (ngraphs == 0) return fail(ERR_ARG, "batch: no graphs");
  if (sort_type > 3) return fail(ERR_ARG, "batch: sort type %u", sort_type);
  b.voff.assign(ngraphs + 1, 0);
  uint64_t V = 0;
  for (uint32_t i = 0; i < ngraphs; i++) {
    if (eoff[i + 1] < eoff[i]) return fail(ERR_ARG, "batch: edge offsets decrease at graph %u", i);
    V += nv[i];
    if (V > (1u << 30)) return fail(ERR_RANGE, "batch: more than 2^30 vertices in all");
    b.voff[i + 1] = (uint32_t)V;
  }
  const uint64_t E = eoff[ngraphs] - eoff[0];
  if (eoff[0] != 0) return fail(ERR_ARG, "batch: edge offsets must start at 0");
  if (E > 0xFFFFFFFFull) return fail(ERR_RANGE, "batch: more than 2^32 - 1 edges in all");
  b.ngraphs = ngraphs;
  OGB_TRY(b.d_voff.alloc((size_t)(ngraphs + 1) * 4));
  OGB_TRY(b.d_eoff.alloc((size_t)(ngraphs + 1) * 8));
  OGB_CUDA(cudaMemcpyAsync(b.d_voff.p, b.voff.data(), (size_t)(ngraphs + 1) * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemcpyAsync(b.d_eoff.p, eoff, (size_t)(ngraphs + 1) * 8, cudaMemcpyHostToDevice, s));
  DevBuf us, ud, derr;
  OGB_TRY(us.alloc(E * 4 + 16));
  OGB_TRY(ud.alloc(E * 4 + 16));
  OGB_TRY(derr.alloc(16));
  OGB_CUDA(cudaMemsetAsync(derr.p, 0, 4, s));
  if (E) {
    OGB_CUDA(cudaMemcpyAsync(us.p, src, E * 4, cudaMemcpyHostToDevice, s));
    OGB_CUDA(cudaMemcpyAsync(ud.p, dst, E * 4, cudaMemcpyHostToDevice, s));
    bk_shift<<<sm_count() * 8, 256, 0, s>>>(E, b.d_eoff.as<uint64_t>(), b.d_voff.as<uint32_t>(), ngraphs,
                                           us.as<uint32_t>(), ud.as<uint32_t>(), derr.as<uint32_t>());
    OGB_CUDA(cudaGetLastError());
  }
  uint32_t herr = 0;
  OGB_CUDA(cudaMemcpyAsync(&herr, derr.p, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  if (herr) return fail(ERR_RANGE, "batch: an edge id is not below its graph's vertex count");
  OGB_TRY(graph_build(b.g, us.as<uint32_t>(), ud.as<uint32_t>(), nullptr, (uint32_t)E, (uint32_t)V, sort_type, s));
  OGB_TRY(graph_check(b.g, s));
  OGB_TRY(b.gid.alloc(V * 4 + 16));
  bk_gid<<<sm_count() * 8, 256, 0, s>>>((uint32_t)V, b.d_voff.as<uint32_t>(), ngraphs, b.gid.as<uint32_t>());
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(b.frozen.alloc((size_t)ngraphs * 4 + 16));
  OGB_TRY(b.stop_iter.alloc((size_t)ngraphs * 4 + 16));
  OGB_TRY(b.executed.alloc((size_t)ngraphs * 4 + 16));
  OGB_TRY(b.active_last.alloc((size_t)ngraphs * 4 + 16));
  OGB_TRY(b.err_last.alloc((size_t)ngraphs * 8 + 16));
  OGB_TRY(b.delta.alloc(V * 4 + 16));
  if (!b.ev0) {
    OGB_CUDA(cudaEventCreate(&b.ev0));
    OGB_CUDA(cudaEventCreate(&b.ev1));
  }
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

int batch_bfs(GraphBatch& b, const uint32_t* roots, int32_t* parents, uint32_t* distances, BfsResult* res,
              cudaStream_t s) {
  std::vector<uint32_t> r(b.ngraphs);
  for (uint32_t i = 0; i < b.ngraphs; i++) {
    if (roots[i] >= b.voff[i + 1] - b.voff[i]) return fail(ERR_ARG, "batch bfs: root %u of graph %u out of range", roots[i], i);
    r[i] = roots[i] + b.voff[i];
  }
  OGB_TRY(bfs_run_roots(b.g, r.data(), b.ngraphs, BFS_DO, parents, distances, res, false, false, s));
  bk_localize<<<sm_count() * 8, 256, 0, s>>>(b.g.V, b.gid.as<uint32_t>(), b.d_voff.as<uint32_t>(), parents);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

int batch_pagerank(GraphBatch& b, uint32_t max_iters, double epsilon, float* ranks, BatchPrGraph* per_graph,
                   double* ms_out, uint32_t* captured, cudaStream_t s) {
  uint32_t wt = 0, ct = 0, cth = 0, ch = 0;
  pagerank_get_bins(&wt, &ct, &cth, &ch);
  if (b.pr_exec && (b.pr_iters != max_iters || b.pr_eps != epsilon || b.pr_ranks != ranks || b.pr_warp != wt ||
                    b.pr_cta != ct || b.pr_build != b.g.build_id)) {
    cudaGraphExecDestroy(b.pr_exec);
    b.pr_exec = nullptr;
  }
  PrBatchDev d;
  d.voff = b.d_voff.as<uint32_t>();
  d.gid = b.gid.as<uint32_t>();
  d.frozen = b.frozen.as<uint32_t>();
  d.stop_iter = b.stop_iter.as<uint32_t>();
  d.executed = b.executed.as<uint32_t>();
  d.active_last = b.active_last.as<uint32_t>();
  d.err_last = b.err_last.as<double>();
  d.delta = b.delta.as<float>();
  bool rebuilt = false;
  // capture happens outside the timed region
  if (!b.pr_exec) {
    OGB_TRY(pagerank_batch_run(b.g, d, b.ngraphs, max_iters, epsilon, ranks, &b.pr_exec, &rebuilt, s));
    OGB_CUDA(cudaStreamSynchronize(s));
    b.pr_iters = max_iters;
    b.pr_eps = epsilon;
    b.pr_ranks = ranks;
    b.pr_warp = wt;
    b.pr_cta = ct;
    b.pr_build = b.g.build_id;
  }
  OGB_CUDA(cudaEventRecord(b.ev0, s));
  OGB_TRY(pagerank_batch_run(b.g, d, b.ngraphs, max_iters, epsilon, ranks, &b.pr_exec, nullptr, s));
  OGB_CUDA(cudaEventRecord(b.ev1, s));
  std::vector<uint32_t> stop(b.ngraphs), exe(b.ngraphs), act(b.ngraphs);
  std::vector<double> err(b.ngraphs);
  OGB_CUDA(cudaMemcpyAsync(stop.data(), d.stop_iter, (size_t)b.ngraphs * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(exe.data(), d.executed, (size_t)b.ngraphs * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(act.data(), d.active_last, (size_t)b.ngraphs * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaMemcpyAsync(err.data(), d.err_last, (size_t)b.ngraphs * 8, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&ms, b.ev0, b.ev1));
  if (ms_out) *ms_out = ms;
  if (captured) *captured = rebuilt ? 1u : 0u;
  if (per_graph)
    for (uint32_t i = 0; i < b.ngraphs; i++) {
      const bool conv = stop[i] != 0xFFFFFFFFu;
      per_graph[i].converged = conv ? 1u : 0u;
      per_graph[i].iterations = conv ? stop[i] : max_iters;
      per_graph[i].executed = exe[i];
      per_graph[i].activeVertices = act[i];
      per_graph[i].error_total = err[i];
    }
  return OK;
}

// Bin thresholds for this batch: each candidate (warp_thr, cta_thr) runs a
// few pull iterations over the union (its per-graph layout is rebuilt for
// it, outside the timing); the fastest is kept as the library's setting.
int batch_autotune(GraphBatch& b, uint32_t iters, TuneResult* out, cudaStream_t s) {
  static const uint32_t cand[][2] = {{16, 1024}, {32, 2048}, {64, 2048}, {64, 4096}, {128, 4096}, {32, 8192}};
  const uint32_t n = sizeof(cand) / sizeof(cand[0]);
  float* ranks = nullptr;
  DevBuf rb;
  OGB_TRY(rb.alloc((size_t)b.g.V * 4 + 16));
  ranks = rb.as<float>();
  double best = 1e30;
  uint32_t bi = 0;
  for (uint32_t i = 0; i < n; i++) {
    pagerank_set_bins(cand[i][0], cand[i][1]);
    PrResult r;
    OGB_TRY(pagerank_run(b.g, PR_PULL, 1, 0.0, ranks, nullptr, &r, s));  // builds the layout
    OGB_TRY(pagerank_run(b.g, PR_PULL, iters, 0.0, ranks, nullptr, &r, s));
    const double ms = r.ms / iters;
    if (out) {
      out->warp_thr[i] = cand[i][0];
      out->cta_thr[i] = cand[i][1];
      out->ms[i] = ms;
    }
    if (ms < best) {
      best = ms;
      bi = i;
    }
  }
  pagerank_set_bins(cand[bi][0], cand[bi][1]);
  if (out) {
    out->n = n;
    out->best = bi;
  }
  return OK;
}

}  // namespace ogb
