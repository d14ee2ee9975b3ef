// compact.cu -- single-pass stable stream compaction of edge lists, and the
// duplicate/self-loop removal built on it.
//
// Reference: removeDulpicatesSelfLoopEdges (00_graph_bench/src/structures/
// edgeList.c:138-211) walks the sorted list once, skips self loops, and
// keeps an edge only if it differs from the LAST KEPT edge.  That is two
// stable compactions: (1) drop self loops, (2) drop edges equal to their
// predecessor in the result of (1).  Each compaction is one kernel: a CTA
// flags its tile, scans the flags, resolves the tile's output offset by
// decoupled look-back and scatters the kept edges in order.
#include "graph.cuh"

namespace ogb {

namespace {
constexpr int kCT = 256;   // threads
constexpr int kCI = 8;     // items per thread (blocked)
constexpr int kCTile = kCT * kCI;
constexpr unsigned long long kCAgg = 1ull << 32;
constexpr unsigned long long kCInc = 2ull << 32;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_w, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_w[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kCT / 32 ? s_w[lane] : 0;
#pragma unroll
    for (int o = 1; o < kCT / 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kCT / 32) s_w[lane] = w;
  }
  __syncthreads();
  *total = s_w[kCT / 32 - 1];
  return (warp ? s_w[warp - 1] : 0) + x - v;
}

// mode 0: keep src != dst.  mode 1: keep i == 0 or (src,dst) != previous.
template <int MODE>
__global__ void __launch_bounds__(kCT) compact_kernel(uint32_t n, const uint32_t* __restrict__ s,
                                                      const uint32_t* __restrict__ d,
                                                      const uint32_t* __restrict__ w, uint32_t* __restrict__ os,
                                                      uint32_t* __restrict__ od, uint32_t* __restrict__ ow,
                                                      int truncate_w, unsigned long long* __restrict__ status,
                                                      uint32_t* __restrict__ ctr) {
  __shared__ uint32_t s_tile, s_prefix;
  __shared__ uint32_t s_w[kCT / 32];
  if (threadIdx.x == 0) s_tile = atomicAdd(&ctr[0], 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = (uint64_t)tile * kCTile + (uint64_t)threadIdx.x * kCI;
  uint32_t keep = 0;  // bit k: item k kept
#pragma unroll
  for (int k = 0; k < kCI; k++) {
    const uint64_t i = base + k;
    if (i < n) {
      const uint32_t a = s[i], b = d[i];
      bool kp;
      if (MODE == 0)
        kp = a != b;
      else
        kp = (i == 0) || a != s[i - 1] || b != d[i - 1];
      keep |= (kp ? 1u : 0u) << k;
    }
  }
  uint32_t tile_total = 0;
  const uint32_t excl = block_excl_scan(__popc(keep), s_w, &tile_total);
  if (threadIdx.x == 0) {
    unsigned long long* st = status + tile;
    uint32_t prefix = 0;
    if (tile == 0) {
      st_volatile_u64(st, kCInc | tile_total);
    } else {
      st_volatile_u64(st, kCAgg | tile_total);
      int64_t p = (int64_t)tile - 1;
      uint32_t spins = 0;
      while (p >= 0) {
        const unsigned long long v = ld_volatile_u64(status + p);
        const unsigned long long f = v & ~0xFFFFFFFFull;
        if (f == 0) {
          if (++spins > kSpinLimit) {
            atomicExch(&ctr[2], (uint32_t)ERR_SPIN);
            break;
          }
          continue;
        }
        prefix += (uint32_t)v;
        if (f == kCInc) break;
        --p;
      }
      st_volatile_u64(st, kCInc | (unsigned long long)(prefix + tile_total));
    }
    s_prefix = prefix;
    if ((uint64_t)(tile + 1) * kCTile >= n) ctr[1] = prefix + tile_total;  // last tile: total kept
  }
  __syncthreads();
  uint32_t o = s_prefix + excl;
#pragma unroll
  for (int k = 0; k < kCI; k++) {
    if ((keep >> k) & 1u) {
      const uint64_t i = base + k;
      os[o] = s[i];
      od[o] = d[i];
      if (w) {
        uint32_t x = w[i];
        if (truncate_w) x = __float_as_uint(__uint2float_rn(__float2uint_rz(__uint_as_float(x))));
        ow[o] = x;
      }
      o++;
    }
  }
}
}  // namespace

// Two compactions (self loops, then consecutive duplicates).  Output arrays
// must not alias the inputs; *out_count receives the kept edge count.
int dedup_device(const uint32_t* s, const uint32_t* d, const uint32_t* w, uint32_t E, uint32_t* os, uint32_t* od,
                 uint32_t* ow, int truncate_weights, uint32_t* out_count, cudaStream_t st) {
  *out_count = 0;
  if (E == 0) return OK;
  const uint32_t tiles = ceil_div(E, kCTile);
  DevBuf status, ctr, ts, td, tw;
  OGB_TRY(status.alloc((size_t)tiles * 8 + 8));
  OGB_TRY(ctr.alloc(16));
  OGB_TRY(ts.alloc((size_t)E * 4));
  OGB_TRY(td.alloc((size_t)E * 4));
  if (w) OGB_TRY(tw.alloc((size_t)E * 4));
  uint32_t h[4];
  // pass 1: self loops
  OGB_CUDA(cudaMemsetAsync(status.p, 0, (size_t)tiles * 8, st));
  OGB_CUDA(cudaMemsetAsync(ctr.p, 0, 16, st));
  compact_kernel<0><<<tiles, kCT, 0, st>>>(E, s, d, w, ts.as<uint32_t>(), td.as<uint32_t>(),
                                           w ? tw.as<uint32_t>() : nullptr, truncate_weights, status.as<unsigned long long>(),
                                           ctr.as<uint32_t>());
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaMemcpyAsync(h, ctr.p, 16, cudaMemcpyDeviceToHost, st));
  OGB_CUDA(cudaStreamSynchronize(st));
  if (h[2]) return fail(ERR_SPIN, "dedup: look-back wait gave up");
  const uint32_t n1 = h[1];
  if (n1 == 0) return OK;
  // pass 2: consecutive duplicates (weights already truncated)
  const uint32_t tiles2 = ceil_div(n1, kCTile);
  OGB_CUDA(cudaMemsetAsync(status.p, 0, (size_t)tiles2 * 8, st));
  OGB_CUDA(cudaMemsetAsync(ctr.p, 0, 16, st));
  compact_kernel<1><<<tiles2, kCT, 0, st>>>(n1, ts.as<uint32_t>(), td.as<uint32_t>(), w ? tw.as<uint32_t>() : nullptr,
                                            os, od, ow, 0, status.as<unsigned long long>(), ctr.as<uint32_t>());
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaMemcpyAsync(h, ctr.p, 16, cudaMemcpyDeviceToHost, st));
  OGB_CUDA(cudaStreamSynchronize(st));
  if (h[2]) return fail(ERR_SPIN, "dedup: look-back wait gave up");
  *out_count = h[1];
  return OK;
}

}  // namespace ogb

// The ABI layer declares this at global scope.
int dedup_device(const uint32_t* s, const uint32_t* d, const uint32_t* w, uint32_t E, uint32_t* os, uint32_t* od,
                 uint32_t* ow, int truncate_weights, uint32_t* out_count, cudaStream_t st) {
  return ogb::dedup_device(s, d, w, E, os, od, ow, truncate_weights, out_count, st);
}
