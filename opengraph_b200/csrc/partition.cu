// partition.cu -- stable split of an edge-list shard by vertex owner, for a
// graph built across several GPUs (no counterpart in the reference, which
// sorts one edge list in one process: radixsort.c:46-335, graphCSR.c:107-248).
//
// Ranks own contiguous vertex ranges [bounds[r], bounds[r+1]).  Each edge of
// a rank's shard goes to the owner of its source (pass A) and, when that is
// another rank, to the owner of its destination (pass B).  The output holds,
// per destination rank r in rank order, A_r then B_r, each in shard order, so
// one all-to-all sends every rank its segment.  A rank that builds its graph
// from the segments it receives (in sender order) gets, for each vertex it
// owns, the same out-row and the same in-row, in the same order, as the graph
// of the whole edge list: an out-row's edges all come from one pass of each
// sender, in shard order, and in-rows follow the stably sorted out-rows.
//
// Each pass is a count (per warp and owner, 1024 edges per warp), an
// exclusive scan of the counts owner-major, and a stable scatter in which a
// warp ranks each 32-edge chunk by __match_any_sync over the owners.
#include "graph.cuh"

#include <algorithm>
#include <vector>

namespace ogb {

namespace {

constexpr uint32_t kPartWarpEdges = 1024;  // edges per warp
constexpr uint32_t kPartWarps = 8;         // warps per CTA
constexpr uint32_t kPartThreads = kPartWarps * 32;
constexpr uint32_t kMaxParts = 64;
constexpr uint32_t kSkip = 0xFFFFFFFFu;

// Owner of vertex x: the r with bounds[r] <= x < bounds[r + 1] (kSkip if x
// is past the last range).
__device__ __forceinline__ uint32_t owner_of(const uint32_t* s_bounds, uint32_t nparts, uint32_t x) {
  uint32_t lo = 0, hi = nparts;  // answer in [lo, hi)
  if (x >= s_bounds[nparts]) return kSkip;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (x >= s_bounds[mid]) lo = mid; else hi = mid;
  }
  return lo;
}

// The pass's key of edge e: pass A the source's owner, pass B the
// destination's owner unless it is the source's (kSkip).  Ids past the last
// range set *err.
__device__ __forceinline__ uint32_t part_key(uint32_t pass, const uint32_t* __restrict__ src,
                                             const uint32_t* __restrict__ dst, uint32_t e, const uint32_t* s_bounds,
                                             uint32_t nparts, uint32_t* err) {
  const uint32_t os = owner_of(s_bounds, nparts, src[e]);
  const uint32_t od = owner_of(s_bounds, nparts, dst[e]);
  if (os == kSkip || od == kSkip) {
    atomicExch(err, 1u);
    return kSkip;
  }
  if (pass == 0) return os;
  return od == os ? kSkip : od;
}

__global__ void __launch_bounds__(kPartThreads) part_count_kernel(
    uint32_t pass, const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint32_t E,
    const uint32_t* __restrict__ bounds, uint32_t nparts, uint32_t nw, uint32_t* __restrict__ cnt,
    uint32_t* __restrict__ err) {
  __shared__ uint32_t s_bounds[kMaxParts + 1];
  __shared__ uint32_t s_cnt[kPartWarps][kMaxParts];
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  for (uint32_t i = threadIdx.x; i <= nparts; i += blockDim.x) s_bounds[i] = bounds[i];
  for (uint32_t i = lane; i < nparts; i += 32) s_cnt[warp][i] = 0;
  __syncthreads();
  const uint32_t gw = blockIdx.x * kPartWarps + warp;
  const uint64_t e0 = (uint64_t)gw * kPartWarpEdges;
  for (uint32_t k = lane; k < kPartWarpEdges; k += 32) {
    const uint64_t e = e0 + k;
    if (e >= E) break;
    const uint32_t key = part_key(pass, src, dst, (uint32_t)e, s_bounds, nparts, err);
    if (key != kSkip) atomicAdd(&s_cnt[warp][key], 1u);
  }
  __syncwarp();
  if (gw < nw)
    for (uint32_t b = lane; b < nparts; b += 32) cnt[(size_t)b * nw + gw] = s_cnt[warp][b];
}

// scan_a / scan_b: exclusive scans of pass A's / pass B's counts (owner-major,
// nparts * nw entries + the total).  The segment of owner b starts at
// (A counts of owners < b) + (B counts of owners < b); its A part first.
__global__ void __launch_bounds__(kPartThreads) part_scatter_kernel(
    uint32_t pass, const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, const float* __restrict__ w,
    uint32_t E, const uint32_t* __restrict__ bounds, uint32_t nparts, uint32_t nw, const uint32_t* __restrict__ scan_a,
    const uint32_t* __restrict__ scan_b, uint32_t* __restrict__ out_src, uint32_t* __restrict__ out_dst,
    float* __restrict__ out_w, uint32_t* __restrict__ err) {
  __shared__ uint32_t s_bounds[kMaxParts + 1];
  __shared__ uint32_t s_off[kPartWarps][kMaxParts];
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  const uint32_t gw = blockIdx.x * kPartWarps + warp;
  for (uint32_t i = threadIdx.x; i <= nparts; i += blockDim.x) s_bounds[i] = bounds[i];
  if (gw < nw)
    for (uint32_t b = lane; b < nparts; b += 32)
      s_off[warp][b] = pass == 0 ? scan_a[(size_t)b * nw + gw] + scan_b[(size_t)b * nw]
                                 : scan_b[(size_t)b * nw + gw] + scan_a[(size_t)(b + 1) * nw];
  __syncthreads();
  const uint64_t e0 = (uint64_t)gw * kPartWarpEdges;
  for (uint32_t k = 0; k < kPartWarpEdges; k += 32) {
    const uint64_t e = e0 + k + lane;
    if (e0 + k >= E) break;  // the same for the whole warp
    const uint32_t key = e < E ? part_key(pass, src, dst, (uint32_t)e, s_bounds, nparts, err) : kSkip;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
    if (key != kSkip) {
      const uint32_t pos = s_off[warp][key] + __popc(peers & lanemask_lt());
      out_src[pos] = src[e];
      out_dst[pos] = dst[e];
      if (w) out_w[pos] = w[e];
    }
    __syncwarp();
    if (key != kSkip && lane == (uint32_t)(__ffs(peers) - 1)) s_off[warp][key] += __popc(peers);
    __syncwarp();
  }
}

}  // namespace

int partition_edges(const uint32_t* src, const uint32_t* dst, const float* w, uint32_t E, const uint32_t* bounds,
                    uint32_t nparts, uint32_t* out_src, uint32_t* out_dst, float* out_w, uint32_t* counts,
                    cudaStream_t s) {
  if (nparts < 1 || nparts > kMaxParts) return fail(ERR_ARG, "partition: %u parts (1 to %u)", nparts, kMaxParts);
  if (!bounds || !counts) return fail(ERR_ARG, "partition: null bounds or counts");
  if (bounds[0] != 0) return fail(ERR_ARG, "partition: the first range must start at vertex 0");
  for (uint32_t r = 0; r < nparts; r++)
    if (bounds[r] > bounds[r + 1]) return fail(ERR_ARG, "partition: ranges must be ascending");
  if (E && (!src || !dst || !out_src || !out_dst || (w && !out_w))) return fail(ERR_ARG, "partition: null");
  if (E == 0) {
    std::fill(counts, counts + nparts, 0u);
    return OK;
  }
  if (2ull * E > 0xFFFFFFFFull) return fail(ERR_ARG, "partition: %u edges (at most 2^31 - 1 per shard)", E);
  const uint32_t nw = (uint32_t)(((uint64_t)E + kPartWarpEdges - 1) / kPartWarpEdges);
  const uint32_t nblocks = (nw + kPartWarps - 1) / kPartWarps;
  const size_t n = (size_t)nparts * nw;
  if (n >= 0xFFFFFFFFull) return fail(ERR_ARG, "partition: too many edges for %u parts", nparts);
  const size_t tmpw = scan_tmp_words((uint32_t)n);
  // device scratch: bounds + error word, two count arrays, two scans, scan
  // temp; each array starts on a 16-byte boundary
  auto up4 = [](size_t x) { return (x + 3) & ~(size_t)3; };
  const size_t o_cnt_a = up4(kMaxParts + 2), o_cnt_b = o_cnt_a + up4(n), o_scan_a = o_cnt_b + up4(n),
               o_scan_b = o_scan_a + up4(n + 1), o_tmp = o_scan_b + up4(n + 1), words = o_tmp + up4(tmpw);
  DevBuf buf;
  OGB_TRY(buf.alloc(words * 4));
  uint32_t* d_bounds = buf.as<uint32_t>();
  uint32_t* d_err = d_bounds + kMaxParts + 1;
  uint32_t* cnt_a = d_bounds + o_cnt_a;
  uint32_t* cnt_b = d_bounds + o_cnt_b;
  uint32_t* scan_a = d_bounds + o_scan_a;
  uint32_t* scan_b = d_bounds + o_scan_b;
  uint32_t* tmp = d_bounds + o_tmp;
  OGB_CUDA(cudaMemcpyAsync(d_bounds, bounds, (nparts + 1) * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemsetAsync(d_err, 0, 4, s));
  part_count_kernel<<<nblocks, kPartThreads, 0, s>>>(0, src, dst, E, d_bounds, nparts, nw, cnt_a, d_err);
  part_count_kernel<<<nblocks, kPartThreads, 0, s>>>(1, src, dst, E, d_bounds, nparts, nw, cnt_b, d_err);
  OGB_CUDA(cudaGetLastError());
  OGB_TRY(scan_exclusive_u32(cnt_a, scan_a, (uint32_t)n, tmp, s));
  OGB_TRY(scan_exclusive_u32(cnt_b, scan_b, (uint32_t)n, tmp, s));
  part_scatter_kernel<<<nblocks, kPartThreads, 0, s>>>(0, src, dst, w, E, d_bounds, nparts, nw, scan_a, scan_b,
                                                       out_src, out_dst, out_w, d_err);
  part_scatter_kernel<<<nblocks, kPartThreads, 0, s>>>(1, src, dst, w, E, d_bounds, nparts, nw, scan_a, scan_b,
                                                       out_src, out_dst, out_w, d_err);
  OGB_CUDA(cudaGetLastError());
  // per owner: (A + B) = the differences of the two scans at the owner boundaries
  std::vector<uint32_t> ha(nparts + 1), hb(nparts + 1);
  for (uint32_t b = 0; b <= nparts; b++) {
    OGB_CUDA(cudaMemcpyAsync(&ha[b], scan_a + (size_t)b * nw, 4, cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaMemcpyAsync(&hb[b], scan_b + (size_t)b * nw, 4, cudaMemcpyDeviceToHost, s));
  }
  uint32_t herr = 0;
  OGB_CUDA(cudaMemcpyAsync(&herr, d_err, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));  // also keeps buf alive until the kernels are done
  if (herr) return fail(ERR_RANGE, "partition: a vertex id is past the last range (%u)", bounds[nparts]);
  for (uint32_t b = 0; b < nparts; b++) counts[b] = (ha[b + 1] - ha[b]) + (hb[b + 1] - hb[b]);
  return OK;
}

}  // namespace ogb
