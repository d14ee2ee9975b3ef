// scan.cu -- device-wide exclusive scan of u32 arrays (three passes: tile
// sums, one-CTA scan of the tile sums, tile scans with the tile offsets).
// Used by the preparation steps (renumbered PageRank layout, BFS result
// packing), not inside an iteration.
#include "graph.cuh"

#include <algorithm>

namespace ogb {


constexpr uint32_t kScanTileN = 4096;  // 256 threads x 16

__device__ __forceinline__ uint32_t block_excl_256(uint32_t v, uint32_t* s_w, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_w[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < 8 ? s_w[lane] : 0;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < 8) s_w[lane] = t;
  }
  __syncthreads();
  *total = s_w[7];
  const uint32_t r = (warp ? s_w[warp - 1] : 0) + x - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(256) scan_tile_sum_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                                            uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_w[8];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTileN + threadIdx.x * 16;
  uint32_t t = 0;
  for (int k = 0; k < 16; k++)
    if (base + k < n) t += in[base + k];
  uint32_t total;
  block_excl_256(t, s_w, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One CTA: exclusive scan of the tile sums in place; total into sums[ntiles].
__global__ void __launch_bounds__(256) scan_sums_kernel(uint32_t* __restrict__ sums, uint32_t ntiles) {
  __shared__ uint32_t s_w[8];
  uint32_t carry = 0;
  for (uint32_t b = 0; b < ntiles; b += 256) {
    const uint32_t i = b + threadIdx.x;
    const uint32_t v = i < ntiles ? sums[i] : 0u;
    uint32_t total;
    const uint32_t e = block_excl_256(v, s_w, &total);
    if (i < ntiles) sums[i] = carry + e;
    carry += total;
  }
  if (threadIdx.x == 0) sums[ntiles] = carry;
}

__global__ void __launch_bounds__(256) scan_tile_kernel(const uint32_t* __restrict__ in, uint32_t n,
                                                        const uint32_t* __restrict__ sums, uint32_t* __restrict__ out) {
  __shared__ uint32_t s_w[8];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTileN + threadIdx.x * 16;
  uint32_t v[16], t = 0;
  for (int k = 0; k < 16; k++) {
    v[k] = base + k < n ? in[base + k] : 0u;
    t += v[k];
  }
  uint32_t total;
  uint32_t o = sums[blockIdx.x] + block_excl_256(t, s_w, &total);
  for (int k = 0; k < 16; k++)
    if (base + k < n) {
      out[base + k] = o;
      o += v[k];
    }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = sums[gridDim.x];
}

// out[0..n] = exclusive scan of in[0..n) followed by the total (out holds
// n + 1 entries); tmp holds n / kScanTileN + 2 words.
int scan_exclusive_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t s) {
  const uint32_t ntiles = std::max<uint32_t>(1, ceil_div(n, kScanTileN));
  scan_tile_sum_kernel<<<ntiles, 256, 0, s>>>(in, n, tmp);
  scan_sums_kernel<<<1, 256, 0, s>>>(tmp, ntiles);
  scan_tile_kernel<<<ntiles, 256, 0, s>>>(in, n, tmp, out);
  OGB_CUDA(cudaGetLastError());
  return OK;
}

size_t scan_tmp_words(uint32_t n) { return (size_t)n / kScanTileN + 4; }

}  // namespace ogb
