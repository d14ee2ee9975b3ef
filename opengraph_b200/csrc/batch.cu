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
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~MsWork() {
    if (h_ctl) cudaFreeHost(h_ctl);
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

  OGB_CUDA(cudaEventRecord(w->ev0, s));
  OGB_CUDA(cudaMemsetAsync(depth, 0xFF, (size_t)V * 64 * 2, s));
  OGB_CUDA(cudaMemsetAsync(F, 0, (size_t)V * 8, s));
  OGB_CUDA(cudaMemsetAsync(N, 0, (size_t)V * 8, s));
  OGB_CUDA(cudaMemsetAsync(vis, 0, (size_t)V * 8, s));
  OGB_CUDA(cudaMemsetAsync(ctl, 0, sizeof(MsCtl), s));
  msk_roots<<<1, 64, 0, s>>>(d_verts, d_masks, (uint32_t)verts.size(), F, vis, depth, w->list.as<uint32_t>(),
                             g.fwd.d_out_degree(), ctl);
  OGB_CUDA(cudaGetLastError());
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
      msk_frontier_degree<<<std::min<uint32_t>(sms * 8, ceil_div(nlist, 256)), 256, 0, s>>>(
          w->list.as<uint32_t>(), nlist, rows_f, w->cnt.as<uint32_t>());
      OGB_TRY(scan_exclusive_u32(w->cnt.as<uint32_t>(), w->off.as<uint32_t>(), nlist, w->scan_tmp.as<uint32_t>(), s));
      msk_push<<<sms * 8, 256, 0, s>>>(w->list.as<uint32_t>(), nlist, w->off.as<uint32_t>(), rows_f, g.fwd.d_dst(), F,
                                      vis, N, ctl);
      launches += 5;
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
  float ms = 0.f;
  OGB_CUDA(cudaEventElapsedTime(&ms, w->ev0, w->ev1));
  r.levels = level;
  r.ms = ms;
  r.launches = launches;
  if (res) *res = r;
  return OK;
}

}  // namespace ogb
