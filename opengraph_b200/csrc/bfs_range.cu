// bfs_range.cu -- one rank's share of a 1-D partitioned direction-optimizing
// BFS (several GPUs, one process each; no counterpart in the reference, whose
// single shared-memory loop is BFS.c:476-626).
//
// A rank owns the vertices [lo, hi): their parents and depths, the out-rows
// it expands in top-down steps and the in-rows it scans in bottom-up steps.
// The frontier and the visited set are one byte per vertex over all V and the
// same on every rank.  A step is two calls with an exchange between them,
// made by the caller (opengraph_b200.parallel):
//   expand  -- top-down: for every unvisited out-neighbour w of an owned
//              frontier vertex u, cand[w] = min(cand[w], u) (bfsr_td,
//              bfsr_td_rows); bottom-up: every owned unvisited vertex with
//              in-edges takes the first in-neighbour in the frontier, in CSR
//              order, as its parent (BFS.c:703-754) and sets its next byte
//              (bfsr_bu; rows of more than 32 in-edges by a warp each,
//              bfsr_bu_long);
//   (exchange: top-down a min all-reduce of cand (4 V bytes), bottom-up a
//    max all-reduce of next (V bytes), across the ranks)
//   settle  -- top-down: next[v] = (cand[v] was set); each owner gives its
//              newly reached vertices their depth and cand as parent -- the
//              smallest frontier in-neighbour, where the reference's
//              top-down parent is whichever frontier vertex wins a race
//              (BFS.c:672) -- and counts them and the sum of
//              max(out_degree, 1) over them, the reference's mf (BFS.c:675);
//              both directions: visited |= next (bfsr_settle).
// cand is kNoCand everywhere between steps: init fills it, a top-down
// settle puts back what the step changed.
// counts (4 u64): expand zeroes them; [0] vertices this rank reached in the
// step, [1] their mf share (top-down), [2] in-edges examined (bottom-up),
// [3] nonzero if a step queue overflowed (cannot happen: the queues are
// sized for the worst case; the caller checks it with the others, so a step
// needs no synchronization of its own).
// Depths are exact for any partition (the search is level-synchronous), and
// so are the bottom-up parents; the top-down parents do not depend on the
// partition either.
//
// The scans over vertex bytes read 4 bytes at a time when the buffers are
// 4-byte aligned (and cand 16-byte aligned), else one at a time.
//
// Fused exchange (bfs_range_expand_peers / bfs_range_claim_peers), with the
// cand array and two alternating next buffers in memory every rank maps (for
// example symmetric memory over NVLink): a top-down expand sends each
// candidate straight to the cand array of w's owner (remote atomicMin); after
// a barrier each owner claims its vertices from its own cand, writes its
// owned next bytes and stores them into every rank's next buffer; after a
// second barrier each rank merges visited |= next (bfs_range_settle with
// direction 1).  A bottom-up step zeroes only its owned next bytes, finds its
// parents as above, and broadcasts its owned next bytes the same way.  No
// all-reduce of cand or next: each byte crosses the links once per reader.
#include "graph.cuh"

#include <algorithm>

namespace ogb {

namespace {

constexpr uint32_t kThreadRow = 32;      // rows up to this many edges: one thread
constexpr uint32_t kRowChunk = 4096;     // longer top-down rows: queued chunks of this many edges, one warp each
constexpr uint32_t kNoParent = 0xFFFFFFFFu;
constexpr int32_t kNoCand = 0x7F7F7F7F;  // cand of a vertex no frontier vertex reached (ids are < 2^30);
                                         // every byte 0x7F, so one memset writes it

// Work queue of a step: a count, then {vertex, first edge, end edge or
// degree, 0} per item.
struct RangeQueue {
  uint32_t n, pad[3];
  uint4 item[1];
};

// Calls f(v) for every v in [lo, hi) whose byte is nonzero (kSet) or zero
// (!kSet), the calling thread taking 4 consecutive vertices per round.
template <bool kVec, bool kSet, class F>
__device__ __forceinline__ void for_bytes(const uint8_t* __restrict__ bytes, uint32_t lo, uint32_t hi, uint32_t V,
                                          F f) {
  const uint32_t w0 = lo >> 2, w1 = (hi + 3) >> 2;
  for (uint32_t w = w0 + blockIdx.x * blockDim.x + threadIdx.x; w < w1; w += gridDim.x * blockDim.x) {
    const uint32_t v0 = w << 2;
    uint32_t x;
    if (kVec && v0 + 4 <= V) {
      x = *reinterpret_cast<const uint32_t*>(bytes + v0);
    } else {
      x = 0;
      for (uint32_t k = 0; k < 4 && v0 + k < V; k++) x |= (uint32_t)bytes[v0 + k] << (8 * k);
    }
    for (uint32_t k = 0; k < 4; k++) {
      const uint32_t v = v0 + k;
      if (v < lo || v >= hi) continue;
      const bool set = (x >> (8 * k)) & 0xFFu;
      if (set == kSet) f(v);
    }
  }
}

__device__ __forceinline__ void flag_overflow(unsigned long long* counts) { atomicOr(&counts[3], 1ull); }

__global__ void bfsr_init_kernel(uint32_t lo, uint32_t hi, uint32_t root, const uint32_t* __restrict__ out_degree,
                                 int32_t* __restrict__ parents, uint32_t* __restrict__ dist) {
  for (uint32_t v = lo + blockIdx.x * blockDim.x + threadIdx.x; v < hi; v += gridDim.x * blockDim.x) {
    const uint32_t d = out_degree[v];
    parents[v] = v == root ? (int32_t)root : (d ? -(int32_t)d : -1);
    dist[v] = 0;
  }
}

// Where a top-down step's candidate for w goes: this rank's cand array, or
// (fused exchange) the cand array of w's owner, mapped from another GPU.
struct CandLocal {
  int32_t* cand;
  __device__ __forceinline__ int32_t* at(uint32_t w) const { return cand + w; }
  static constexpr bool kPeers = false;
};
struct CandPeers {
  int32_t* const* cand;     // per rank: its cand array (V entries)
  const uint32_t* bounds;   // owner ranges: rank r owns [bounds[r], bounds[r + 1])
  uint32_t nparts;
  __device__ __forceinline__ int32_t* at(uint32_t w) const {
    uint32_t lo = 0, hi = nparts;  // the owner is in [lo, hi)
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (w >= __ldg(&bounds[mid])) lo = mid; else hi = mid;
    }
    return cand[lo] + w;
  }
  static constexpr bool kPeers = true;
};

// Top-down, the owned frontier vertices: short rows by their thread, longer
// rows queued in chunks.
template <bool kVec, class T>
__global__ void bfsr_td_kernel(uint32_t V, uint32_t lo, uint32_t hi, const uint8_t* __restrict__ frontier,
                               const uint8_t* __restrict__ visited, const uint2* __restrict__ rows,
                               const uint32_t* __restrict__ nbr, T cand, RangeQueue* q,
                               uint32_t qcap, unsigned long long* __restrict__ counts) {
  for_bytes<kVec, true>(frontier, lo, hi, V, [&](uint32_t u) {
    const uint2 r = rows[u];
    if (r.y <= kThreadRow) {
      for (uint32_t j = r.x; j < r.x + r.y; j++) {
        const uint32_t w = __ldg(&nbr[j]) & 0x3FFFFFFFu;
        if (!visited[w]) atomicMin(cand.at(w), (int32_t)u);  // result unused: a reduction, no round trip
      }
    } else {
      const uint32_t nc = (r.y + kRowChunk - 1) / kRowChunk;
      const uint32_t k0 = atomicAdd(&q->n, nc);
      if (k0 + nc > qcap) {
        flag_overflow(counts);
        return;
      }
      for (uint32_t k = 0; k < nc; k++)
        q->item[k0 + k] = make_uint4(u, r.x + k * kRowChunk, r.x + min(r.y, (k + 1) * kRowChunk), 0u);
    }
  });
  if (T::kPeers) __threadfence_system();  // the remote atomics before the caller's barrier
}

// Top-down, the queued chunks: a warp per chunk, lanes strided over its edges.
template <class T>
__global__ void bfsr_td_rows_kernel(const uint8_t* __restrict__ visited, const uint32_t* __restrict__ nbr,
                                    T cand, const RangeQueue* q, uint32_t qcap) {
  const uint32_t lane = lane_id();
  const uint32_t gw = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x / 32);
  const uint32_t n = min(q->n, qcap);
  for (uint32_t t = gw; t < n; t += nw) {
    const uint4 it = q->item[t];
    for (uint32_t j = it.y + lane; j < it.z; j += 32) {
      const uint32_t w = __ldg(&nbr[j]) & 0x3FFFFFFFu;
      if (!visited[w]) atomicMin(cand.at(w), (int32_t)it.x);
    }
  }
  if (T::kPeers) __threadfence_system();
}

// The first in-neighbour of a vertex in the frontier, in CSR order of its
// in-row r (kNoParent if none); `examined` grows by the in-edges read up to
// and including it.  Four neighbour loads in flight per round.
__device__ __forceinline__ uint32_t first_frontier_in(uint2 r, const uint32_t* __restrict__ nbr,
                                                      const uint8_t* __restrict__ frontier, uint32_t& examined) {
  const uint32_t end = r.x + r.y;
  for (uint32_t j = r.x; j < end; j += 4) {
    uint32_t u[4];
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) u[k] = j + k < end ? (__ldg(&nbr[j + k]) & 0x3FFFFFFFu) : kNoParent;
    uint8_t f[4];
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) f[k] = u[k] != kNoParent ? frontier[u[k]] : 0;
#pragma unroll
    for (uint32_t k = 0; k < 4; k++)
      if (f[k]) {
        examined += j + k + 1 - r.x;
        return u[k];
      }
  }
  examined += r.y;
  return kNoParent;
}

// The same for a row of more than kThreadRow in-edges, by a whole warp (r
// the same in every lane): 64 in-neighbours per round, the lowest lane whose
// neighbour is in the frontier wins, so the result is the first in CSR order.
__device__ __forceinline__ uint32_t warp_first_frontier_in(uint2 r, const uint32_t* __restrict__ nbr,
                                                           const uint8_t* __restrict__ frontier, uint32_t lane,
                                                           uint32_t& examined) {
  const uint32_t end = r.x + r.y;
  for (uint32_t j = r.x; j < end; j += 64) {
    const uint32_t a = j + lane, b = j + 32 + lane;
    const uint32_t ua = a < end ? (__ldg(&nbr[a]) & 0x3FFFFFFFu) : kNoParent;
    const uint32_t ub = b < end ? (__ldg(&nbr[b]) & 0x3FFFFFFFu) : kNoParent;
    const bool fa = ua != kNoParent && frontier[ua];
    const bool fb = ub != kNoParent && frontier[ub];
    const uint32_t ma = __ballot_sync(0xFFFFFFFFu, fa), mb = __ballot_sync(0xFFFFFFFFu, fb);
    if (ma | mb) {
      const uint32_t l = ma ? __ffs(ma) - 1 : __ffs(mb) - 1;
      examined += (ma ? j : j + 32) + l + 1 - r.x;
      return __shfl_sync(0xFFFFFFFFu, ma ? ua : ub, l);
    }
  }
  examined += r.y;
  return kNoParent;
}

// Bottom-up, the owned unvisited vertices with in-edges: rows of up to
// kThreadRow in-edges by their thread, longer ones queued for bfsr_bu_long.
template <bool kVec>
__global__ void bfsr_bu_kernel(uint32_t V, uint32_t lo, uint32_t hi, const uint8_t* __restrict__ frontier,
                               const uint8_t* __restrict__ visited, uint32_t depth, const uint2* __restrict__ rows_i,
                               const uint32_t* __restrict__ nbr_i, int32_t* __restrict__ parents,
                               uint32_t* __restrict__ dist, uint8_t* __restrict__ next,
                               unsigned long long* __restrict__ counts, RangeQueue* q, uint32_t qcap) {
  uint32_t found = 0, examined = 0;
  for_bytes<kVec, false>(visited, lo, hi, V, [&](uint32_t v) {
    const uint2 r = rows_i[v];
    if (!r.y) return;
    if (r.y > kThreadRow) {
      const uint32_t k = atomicAdd(&q->n, 1u);
      if (k < qcap)
        q->item[k] = make_uint4(v, r.x, r.y, 0u);
      else
        flag_overflow(counts);
      return;
    }
    const uint32_t p = first_frontier_in(r, nbr_i, frontier, examined);
    if (p == kNoParent) return;
    parents[v] = (int32_t)p;
    dist[v] = depth;
    next[v] = 1;
    found++;
  });
  warp_atomic_add_total64(&counts[0], found);
  warp_atomic_add_total64(&counts[2], examined);
}

// Bottom-up, the queued long rows, a warp each.
__global__ void bfsr_bu_long_kernel(const uint8_t* __restrict__ frontier, uint32_t depth,
                                    const uint32_t* __restrict__ nbr_i, int32_t* __restrict__ parents,
                                    uint32_t* __restrict__ dist, uint8_t* __restrict__ next,
                                    unsigned long long* __restrict__ counts, const RangeQueue* q, uint32_t qcap) {
  const uint32_t lane = lane_id();
  const uint32_t gw = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x / 32);
  const uint32_t n = min(q->n, qcap);
  uint32_t found = 0, examined = 0;
  for (uint32_t t = gw; t < n; t += nw) {
    const uint4 it = q->item[t];
    const uint32_t p = warp_first_frontier_in(make_uint2(it.y, it.z), nbr_i, frontier, lane, examined);
    if (p != kNoParent && lane == 0) {
      parents[it.x] = (int32_t)p;
      dist[it.x] = depth;
      next[it.x] = 1;
      found++;
    }
  }
  if (lane == 0) {  // a warp's counts are in its lane 0
    if (found) atomicAdd(&counts[0], (unsigned long long)found);
    if (examined) atomicAdd(&counts[2], (unsigned long long)examined);
  }
}

// One vertex of a top-down settle: returns its next byte.
__device__ __forceinline__ uint32_t settle_td_vertex(uint32_t v, int32_t c, uint32_t lo, uint32_t hi,
                                                     uint32_t depth, const uint32_t* __restrict__ out_degree,
                                                     int32_t* __restrict__ parents, uint32_t* __restrict__ dist,
                                                     uint32_t& found, unsigned long long& mf) {
  if (c == kNoCand) return 0;
  if (v >= lo && v < hi) {
    const uint32_t d = out_degree[v];
    parents[v] = c;
    dist[v] = depth;
    found++;
    mf += d ? d : 1u;
  }
  return 1;
}

// After the exchange, over all V.  Top-down: next from cand, the owned newly
// reached vertices settled, cand reset to kNoCand for the next top-down
// step; both: visited |= next.
template <bool kVec, bool kTopDown>
__global__ void bfsr_settle_kernel(uint32_t V, uint32_t lo, uint32_t hi, uint32_t depth,
                                   int32_t* __restrict__ cand, uint8_t* __restrict__ next,
                                   uint8_t* __restrict__ visited, const uint32_t* __restrict__ out_degree,
                                   int32_t* __restrict__ parents, uint32_t* __restrict__ dist,
                                   unsigned long long* __restrict__ counts) {
  uint32_t found = 0;
  unsigned long long mf = 0;
  const uint32_t nw = (V + 3) >> 2;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
    const uint32_t v0 = w << 2;
    if (kVec && v0 + 4 <= V) {
      uint32_t nx;
      if (kTopDown) {
        const int4 c = *reinterpret_cast<const int4*>(cand + v0);
        if ((c.x & c.y & c.z & c.w) != kNoCand)
          *reinterpret_cast<int4*>(cand + v0) = make_int4(kNoCand, kNoCand, kNoCand, kNoCand);
        nx = settle_td_vertex(v0, c.x, lo, hi, depth, out_degree, parents, dist, found, mf) |
             settle_td_vertex(v0 + 1, c.y, lo, hi, depth, out_degree, parents, dist, found, mf) << 8 |
             settle_td_vertex(v0 + 2, c.z, lo, hi, depth, out_degree, parents, dist, found, mf) << 16 |
             settle_td_vertex(v0 + 3, c.w, lo, hi, depth, out_degree, parents, dist, found, mf) << 24;
        *reinterpret_cast<uint32_t*>(next + v0) = nx;
      } else {
        nx = *reinterpret_cast<const uint32_t*>(next + v0);
      }
      if (nx) *reinterpret_cast<uint32_t*>(visited + v0) |= nx;
    } else {
      for (uint32_t v = v0; v < v0 + 4 && v < V; v++) {
        uint32_t nx;
        if (kTopDown) {
          nx = settle_td_vertex(v, cand[v], lo, hi, depth, out_degree, parents, dist, found, mf);
          if (nx) cand[v] = kNoCand;
          next[v] = (uint8_t)nx;
        } else {
          nx = next[v];
        }
        if (nx) visited[v] = 1;
      }
    }
  }
  if (kTopDown) {
    warp_atomic_add_total64(&counts[0], found);
    const uint32_t active = __activemask();
    unsigned long long t = mf;
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(active, t, o);
    if ((int)lane_id() == __ffs(active) - 1 && t) atomicAdd(&counts[1], t);
  }
}

// Fused exchange, top-down: the owned vertices with a candidate (in this
// rank's cand, which every rank's expand fed) are reached: parent, depth,
// counts; their next bytes are written (0 or 1 over the whole owned range)
// and cand is put back to kNoCand.
__global__ void bfsr_claim_owned_kernel(uint32_t lo, uint32_t hi, uint32_t depth, int32_t* __restrict__ cand,
                                        uint8_t* __restrict__ next, const uint32_t* __restrict__ out_degree,
                                        int32_t* __restrict__ parents, uint32_t* __restrict__ dist,
                                        unsigned long long* __restrict__ counts) {
  uint32_t found = 0;
  unsigned long long mf = 0;
  for (uint32_t v = lo + blockIdx.x * blockDim.x + threadIdx.x; v < hi; v += gridDim.x * blockDim.x) {
    const int32_t c = cand[v];
    const uint32_t nx = settle_td_vertex(v, c, lo, hi, depth, out_degree, parents, dist, found, mf);
    next[v] = (uint8_t)nx;
    if (nx) cand[v] = kNoCand;
  }
  warp_atomic_add_total64(&counts[0], found);
  const uint32_t active = __activemask();
  unsigned long long t = mf;
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(active, t, o);
  if ((int)lane_id() == __ffs(active) - 1 && t) atomicAdd(&counts[1], t);
}

// Fused exchange: this rank's next bytes of its owned range [lo, hi) copied
// into every rank's next buffer (peer stores; 4 bytes at a time inside the
// range, single bytes on its ragged ends, so no other owner's byte is
// written), then ordered before the caller's barrier.
__global__ void bfsr_broadcast_kernel(uint32_t lo, uint32_t hi, const uint8_t* __restrict__ src,
                                      uint8_t* const* __restrict__ peers, uint32_t npeers) {
  const uint32_t a = (lo + 3) & ~3u, b = hi & ~3u;  // whole words [a, b)
  const uint32_t stride = gridDim.x * blockDim.x, tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < b) {
    for (uint32_t w = a / 4 + tid; w < b / 4; w += stride) {
      const uint32_t x = reinterpret_cast<const uint32_t*>(src)[w];
      for (uint32_t p = 0; p < npeers; p++) reinterpret_cast<uint32_t*>(peers[p])[w] = x;
    }
  }
  // the ends: [lo, min(a, hi)) and [max(b, a, lo), hi)
  const uint32_t e0 = min(a, hi), e1 = max(max(b, a), lo);
  for (uint32_t v = lo + tid; v < e0; v += stride)
    for (uint32_t p = 0; p < npeers; p++) peers[p][v] = src[v];
  for (uint32_t v = e1 + tid; v < hi; v += stride)
    for (uint32_t p = 0; p < npeers; p++) peers[p][v] = src[v];
  __threadfence_system();
}

bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

}  // namespace

// The step queue of a graph.  Top-down: a row of more than kThreadRow edges
// gives at most 1 + edges / kRowChunk chunks, and at most
// min(V, E / (kThreadRow + 1)) rows are that long; bottom-up: one item per
// such row.  E / kRowChunk + min(V, E / (kThreadRow + 1)) items hold any step.
static int range_queue(DevGraph& g, RangeQueue** q, uint32_t* cap) {
  const size_t c = (size_t)g.E / kRowChunk + std::min<size_t>(g.V, (size_t)g.E / (kThreadRow + 1)) + 16;
  OGB_TRY(g.range_q.alloc(16 + c * 16));
  *q = g.range_q.as<RangeQueue>();
  *cap = (uint32_t)std::min<size_t>(c, 0xFFFFFFFFu);
  return OK;
}

static int range_check(const DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction) {
  if (lo > hi || hi > g.V) return fail(ERR_ARG, "bfs range: [%u, %u) is not inside [0, %u)", lo, hi, g.V);
  if (direction > 1) return fail(ERR_ARG, "bfs range: direction %u (0 top-down, 1 bottom-up)", direction);
  return OK;
}

template <class T>
static int launch_td(DevGraph& g, uint32_t lo, uint32_t hi, const uint8_t* frontier, const uint8_t* visited, T cand,
                     RangeQueue* q, uint32_t cap, unsigned long long* counts, bool vec, cudaStream_t s) {
  const int grid = sm_count() * 8;
  if (vec)
    bfsr_td_kernel<true, T><<<grid, 256, 0, s>>>(g.V, lo, hi, frontier, visited, g.fwd.d_rows(), g.fwd.d_dst(), cand,
                                                 q, cap, counts);
  else
    bfsr_td_kernel<false, T><<<grid, 256, 0, s>>>(g.V, lo, hi, frontier, visited, g.fwd.d_rows(), g.fwd.d_dst(),
                                                  cand, q, cap, counts);
  bfsr_td_rows_kernel<T><<<grid, 256, 0, s>>>(visited, g.fwd.d_dst(), cand, q, cap);
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int bfs_range_init(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t root, int32_t* parents, uint32_t* dist,
                   uint8_t* frontier, uint8_t* visited, int32_t* cand, unsigned long long* counts, cudaStream_t s) {
  OGB_TRY(range_check(g, lo, hi, 0));
  if (root >= g.V) return fail(ERR_ARG, "bfs range: root %u out of range (V=%u)", root, g.V);
  // counts = {1, out_degree(root), 0, 0} on the root's owner, zeros elsewhere:
  // summed over the ranks, the first frontier and its mf (BFS.c:511).  Only
  // the owner's out-row of the root is whole when the graph is partitioned.
  OGB_CUDA(cudaMemsetAsync(counts, 0, 32, s));
  if (root >= lo && root < hi) {
    OGB_CUDA(cudaMemsetAsync(counts, 1, 1, s));
    OGB_CUDA(cudaMemcpyAsync(counts + 1, g.fwd.d_out_degree() + root, 4, cudaMemcpyDeviceToDevice, s));
  }
  OGB_CUDA(cudaMemsetAsync(frontier, 0, g.V, s));
  OGB_CUDA(cudaMemsetAsync(visited, 0, g.V, s));
  OGB_CUDA(cudaMemsetAsync(frontier + root, 1, 1, s));
  OGB_CUDA(cudaMemsetAsync(visited + root, 1, 1, s));
  OGB_CUDA(cudaMemsetAsync(cand, 0x7F, (size_t)g.V * 4, s));  // every word kNoCand
  if (hi > lo) bfsr_init_kernel<<<sm_count() * 8, 256, 0, s>>>(lo, hi, root, g.fwd.d_out_degree(), parents, dist);
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int bfs_range_expand(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                     const uint8_t* frontier, const uint8_t* visited, uint8_t* next, int32_t* cand,
                     int32_t* parents, uint32_t* dist, unsigned long long* counts, cudaStream_t s) {
  OGB_TRY(range_check(g, lo, hi, direction));
  OGB_CUDA(cudaMemsetAsync(counts, 0, 32, s));
  if (direction == 1) {
    if (g.V) OGB_CUDA(cudaMemsetAsync(next, 0, g.V, s));
  }
  if (hi == lo) return OK;
  const int grid = sm_count() * 8;
  RangeQueue* q = nullptr;
  uint32_t cap = 0;
  OGB_TRY(range_queue(g, &q, &cap));
  OGB_CUDA(cudaMemsetAsync(q, 0, 16, s));
  const bool vec = aligned(frontier, 4) && aligned(visited, 4);
  if (direction == 1) {
    if (vec)
      bfsr_bu_kernel<true><<<grid, 256, 0, s>>>(g.V, lo, hi, frontier, visited, depth, g.inv.d_rows(),
                                                g.inv.d_dst(), parents, dist, next, counts, q, cap);
    else
      bfsr_bu_kernel<false><<<grid, 256, 0, s>>>(g.V, lo, hi, frontier, visited, depth, g.inv.d_rows(),
                                                 g.inv.d_dst(), parents, dist, next, counts, q, cap);
    bfsr_bu_long_kernel<<<grid, 256, 0, s>>>(frontier, depth, g.inv.d_dst(), parents, dist, next, counts, q, cap);
  } else {
    OGB_TRY(launch_td(g, lo, hi, frontier, visited, CandLocal{cand}, q, cap, counts, vec, s));
  }
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int bfs_range_expand_peers(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                           const uint8_t* frontier, const uint8_t* visited, uint8_t* next, int32_t* const* cand_peers,
                           const uint32_t* bounds, uint32_t nparts, int32_t* parents, uint32_t* dist,
                           unsigned long long* counts, cudaStream_t s) {
  OGB_TRY(range_check(g, lo, hi, direction));
  if (nparts < 1 || !cand_peers || !bounds) return fail(ERR_ARG, "bfs range: no peers");
  OGB_CUDA(cudaMemsetAsync(counts, 0, 32, s));
  if (direction == 1 && hi > lo) OGB_CUDA(cudaMemsetAsync(next + lo, 0, hi - lo, s));  // only the owned bytes
  if (hi == lo) return OK;
  RangeQueue* q = nullptr;
  uint32_t cap = 0;
  OGB_TRY(range_queue(g, &q, &cap));
  OGB_CUDA(cudaMemsetAsync(q, 0, 16, s));
  const bool vec = aligned(frontier, 4) && aligned(visited, 4);
  const int grid = sm_count() * 8;
  if (direction == 1) {
    if (vec)
      bfsr_bu_kernel<true><<<grid, 256, 0, s>>>(g.V, lo, hi, frontier, visited, depth, g.inv.d_rows(),
                                                g.inv.d_dst(), parents, dist, next, counts, q, cap);
    else
      bfsr_bu_kernel<false><<<grid, 256, 0, s>>>(g.V, lo, hi, frontier, visited, depth, g.inv.d_rows(),
                                                 g.inv.d_dst(), parents, dist, next, counts, q, cap);
    bfsr_bu_long_kernel<<<grid, 256, 0, s>>>(frontier, depth, g.inv.d_dst(), parents, dist, next, counts, q, cap);
  } else {
    OGB_TRY(launch_td(g, lo, hi, frontier, visited, CandPeers{cand_peers, bounds, nparts}, q, cap, counts, vec, s));
  }
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int bfs_range_claim_peers(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth, int32_t* cand,
                          uint8_t* next, uint8_t* const* next_peers, uint32_t npeers, int32_t* parents,
                          uint32_t* dist, unsigned long long* counts, cudaStream_t s) {
  OGB_TRY(range_check(g, lo, hi, direction));
  if (npeers < 1 || !next_peers) return fail(ERR_ARG, "bfs range: no peers");
  if (!aligned(next, 4)) return fail(ERR_ARG, "bfs range: next buffers must be 4-byte aligned");
  if (hi == lo) return OK;
  const int grid = sm_count() * 8;
  if (direction == 0)
    bfsr_claim_owned_kernel<<<grid, 256, 0, s>>>(lo, hi, depth, cand, next, g.fwd.d_out_degree(), parents, dist,
                                                 counts);
  bfsr_broadcast_kernel<<<grid, 256, 0, s>>>(lo, hi, next, next_peers, npeers);
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int bfs_range_settle(DevGraph& g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth, int32_t* cand,
                     uint8_t* next, uint8_t* visited, int32_t* parents, uint32_t* dist, unsigned long long* counts,
                     cudaStream_t s) {
  OGB_TRY(range_check(g, lo, hi, direction));
  if (!g.V) return OK;
  const int grid = sm_count() * 8;
  const bool vec = aligned(next, 4) && aligned(visited, 4) && (direction == 1 || aligned(cand, 16));
  const uint32_t* od = g.fwd.d_out_degree();
  if (direction == 0) {
    if (vec)
      bfsr_settle_kernel<true, true><<<grid, 256, 0, s>>>(g.V, lo, hi, depth, cand, next, visited, od, parents, dist,
                                                          counts);
    else
      bfsr_settle_kernel<false, true><<<grid, 256, 0, s>>>(g.V, lo, hi, depth, cand, next, visited, od, parents,
                                                           dist, counts);
  } else {
    if (vec)
      bfsr_settle_kernel<true, false><<<grid, 256, 0, s>>>(g.V, lo, hi, depth, cand, next, visited, od, parents,
                                                           dist, counts);
    else
      bfsr_settle_kernel<false, false><<<grid, 256, 0, s>>>(g.V, lo, hi, depth, cand, next, visited, od, parents,
                                                            dist, counts);
  }
  OGB_CUDA(cudaGetLastError());
  return OK;
}

}  // namespace ogb
