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
// Both passes share one count kernel (per CTA and owner: 2048 edges per
// CTA, 256 per warp) and one scatter kernel, with an exclusive scan of each
// pass's counts (owner-major) between them.  The scatter ranks each 32-edge
// chunk's edges among those going to the same owner with __match_any_sync,
// lays the CTA's output out in shared memory as one run per (owner, pass),
// and copies the runs out with consecutive threads on consecutive addresses:
// each owner's edges keep their shard order, and the global stores are
// coalesced instead of one scattered 4-byte store per edge and array.
#include "graph.cuh"

#include <algorithm>
#include <vector>

namespace ogb {

namespace {

constexpr uint32_t kPartWarps = 8;          // warps per CTA
constexpr uint32_t kPartThreads = kPartWarps * 32;
constexpr uint32_t kWarpChunks = 8;         // 32-edge chunks per warp
constexpr uint32_t kWarpEdges = 32 * kWarpChunks;
constexpr uint32_t kCtaEdges = kPartWarps * kWarpEdges;  // 2048
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

// The two keys of an edge: its source's owner (pass A) and its
// destination's owner if that is another (pass B), else kSkip.  Ids past the
// last range give kSkip for both and set *err.
__device__ __forceinline__ void part_keys(uint32_t s, uint32_t d, const uint32_t* s_bounds, uint32_t nparts,
                                          uint32_t& ka, uint32_t& kb, uint32_t* err) {
  const uint32_t os = owner_of(s_bounds, nparts, s);
  const uint32_t od = owner_of(s_bounds, nparts, d);
  if (os == kSkip || od == kSkip) {
    atomicExch(err, 1u);
    ka = kb = kSkip;
    return;
  }
  ka = os;
  kb = od == os ? kSkip : od;
}

// A warp's edges: loaded all at once (8 chunks in flight), with their keys.
struct WarpEdges {
  uint32_t s[kWarpChunks], d[kWarpChunks], ka[kWarpChunks], kb[kWarpChunks];
  float w[kWarpChunks];
};

__device__ __forceinline__ void load_warp_edges(WarpEdges& x, const uint32_t* __restrict__ src,
                                                const uint32_t* __restrict__ dst, const float* __restrict__ w,
                                                uint64_t e0, uint32_t E, uint32_t lane, const uint32_t* s_bounds,
                                                uint32_t nparts, uint32_t* err) {
#pragma unroll
  for (uint32_t c = 0; c < kWarpChunks; c++) {
    const uint64_t e = e0 + c * 32 + lane;
    x.s[c] = e < E ? src[e] : 0u;
    x.d[c] = e < E ? dst[e] : 0u;
    x.w[c] = (w && e < E) ? w[e] : 0.0f;
  }
#pragma unroll
  for (uint32_t c = 0; c < kWarpChunks; c++) {
    const uint64_t e = e0 + c * 32 + lane;
    x.ka[c] = x.kb[c] = kSkip;
    if (e < E) part_keys(x.s[c], x.d[c], s_bounds, nparts, x.ka[c], x.kb[c], err);
  }
}

// Per-warp counts of a warp's edges by owner, pass A and pass B.
__device__ __forceinline__ void count_warp_edges(const WarpEdges& x, uint32_t lane, uint32_t* cnt_a,
                                                 uint32_t* cnt_b) {
#pragma unroll
  for (uint32_t c = 0; c < kWarpChunks; c++) {
    const uint32_t pa = __match_any_sync(0xFFFFFFFFu, x.ka[c]);
    const uint32_t pb = __match_any_sync(0xFFFFFFFFu, x.kb[c]);
    if (x.ka[c] != kSkip && lane == (uint32_t)(__ffs(pa) - 1)) cnt_a[x.ka[c]] += __popc(pa);
    if (x.kb[c] != kSkip && lane == (uint32_t)(__ffs(pb) - 1)) cnt_b[x.kb[c]] += __popc(pb);
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kPartThreads) part_count_kernel(
    const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint32_t E,
    const uint32_t* __restrict__ bounds, uint32_t nparts, uint32_t nb, uint32_t* __restrict__ cnt_a,
    uint32_t* __restrict__ cnt_b, uint32_t* __restrict__ err) {
  __shared__ uint32_t s_bounds[kMaxParts + 1];
  __shared__ uint32_t s_cnt[2][kPartWarps][kMaxParts];
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  for (uint32_t i = threadIdx.x; i <= nparts; i += blockDim.x) s_bounds[i] = bounds[i];
  for (uint32_t i = lane; i < nparts; i += 32) s_cnt[0][warp][i] = s_cnt[1][warp][i] = 0;
  __syncthreads();
  WarpEdges x;
  load_warp_edges(x, src, dst, nullptr, (uint64_t)blockIdx.x * kCtaEdges + warp * kWarpEdges, E, lane, s_bounds,
                  nparts, err);
  count_warp_edges(x, lane, s_cnt[0][warp], s_cnt[1][warp]);
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < nparts; b += blockDim.x) {
    uint32_t a = 0, c = 0;
    for (uint32_t k = 0; k < kPartWarps; k++) {
      a += s_cnt[0][k][b];
      c += s_cnt[1][k][b];
    }
    cnt_a[(size_t)b * nb + blockIdx.x] = a;
    cnt_b[(size_t)b * nb + blockIdx.x] = c;
  }
}

// scan_a / scan_b: exclusive scans of pass A's / pass B's counts (owner-major,
// nparts * nb entries + the total).  Owner b's output segment starts at
// (A counts of owners < b) + (B counts of owners < b); its A part first.  In
// shared memory a CTA lays its output out the same way: segment 2b + p is
// owner b's pass-p run.
__global__ void __launch_bounds__(kPartThreads) part_scatter_kernel(
    const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, const float* __restrict__ w, uint32_t E,
    const uint32_t* __restrict__ bounds, uint32_t nparts, uint32_t nb, const uint32_t* __restrict__ scan_a,
    const uint32_t* __restrict__ scan_b, uint32_t* __restrict__ out_src, uint32_t* __restrict__ out_dst,
    float* __restrict__ out_w, uint32_t* __restrict__ err) {
  extern __shared__ uint32_t s_stage[];  // src, dst[, w] of up to 2 kCtaEdges items
  __shared__ uint32_t s_bounds[kMaxParts + 1];
  __shared__ uint32_t s_off[2][kPartWarps][kMaxParts];  // per-warp counts, then running positions
  __shared__ uint32_t s_seg[2 * kMaxParts + 1];          // segment starts in the stage
  __shared__ uint32_t s_goff[2 * kMaxParts];             // segment starts in the output
  uint32_t* st_src = s_stage;
  uint32_t* st_dst = s_stage + 2 * kCtaEdges;
  float* st_w = reinterpret_cast<float*>(s_stage + 4 * kCtaEdges);
  const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
  const uint32_t nseg = 2 * nparts;
  for (uint32_t i = threadIdx.x; i <= nparts; i += blockDim.x) s_bounds[i] = bounds[i];
  for (uint32_t i = lane; i < nparts; i += 32) s_off[0][warp][i] = s_off[1][warp][i] = 0;
  __syncthreads();
  WarpEdges x;
  load_warp_edges(x, src, dst, w, (uint64_t)blockIdx.x * kCtaEdges + warp * kWarpEdges, E, lane, s_bounds, nparts,
                  err);
  count_warp_edges(x, lane, s_off[0][warp], s_off[1][warp]);
  __syncthreads();
  // segment sizes and starts (warp 0: lane l takes segments 4l .. 4l + 3),
  // then each warp's start inside each segment
  if (warp == 0) {
    uint32_t sz[4], t = 0;
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) {
      const uint32_t g = 4 * lane + k;
      sz[k] = 0;
      if (g < nseg)
        for (uint32_t q = 0; q < kPartWarps; q++) sz[k] += s_off[g & 1][q][g >> 1];
      t += sz[k];
    }
    uint32_t incl = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    uint32_t run = incl - t;
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) {
      const uint32_t g = 4 * lane + k;
      if (g < nseg) s_seg[g] = run;
      run += sz[k];
    }
    if (lane == 31) s_seg[nseg] = incl;  // the CTA's item count (nseg <= 128 = 4 x 32)
  }
  for (uint32_t g = threadIdx.x; g < nseg; g += blockDim.x) {
    const uint32_t b = g >> 1;
    s_goff[g] = (g & 1) ? scan_b[(size_t)b * nb + blockIdx.x] + scan_a[(size_t)(b + 1) * nb]
                        : scan_a[(size_t)b * nb + blockIdx.x] + scan_b[(size_t)b * nb];
  }
  __syncthreads();
  for (uint32_t g = threadIdx.x; g < nseg; g += blockDim.x) {
    uint32_t run = s_seg[g];
    for (uint32_t q = 0; q < kPartWarps; q++) {
      const uint32_t c = s_off[g & 1][q][g >> 1];
      s_off[g & 1][q][g >> 1] = run;
      run += c;
    }
  }
  __syncthreads();
  // stage the warp's edges at their positions, chunk by chunk in shard order
  uint32_t* off_a = s_off[0][warp];
  uint32_t* off_b = s_off[1][warp];
#pragma unroll
  for (uint32_t c = 0; c < kWarpChunks; c++) {
    const uint32_t ka = x.ka[c], kb = x.kb[c];
    const uint32_t pa = __match_any_sync(0xFFFFFFFFu, ka);
    const uint32_t pb = __match_any_sync(0xFFFFFFFFu, kb);
    if (ka != kSkip) {
      const uint32_t pos = off_a[ka] + __popc(pa & lanemask_lt());
      st_src[pos] = x.s[c];
      st_dst[pos] = x.d[c];
      if (w) st_w[pos] = x.w[c];
    }
    if (kb != kSkip) {
      const uint32_t pos = off_b[kb] + __popc(pb & lanemask_lt());
      st_src[pos] = x.s[c];
      st_dst[pos] = x.d[c];
      if (w) st_w[pos] = x.w[c];
    }
    __syncwarp();
    if (ka != kSkip && lane == (uint32_t)(__ffs(pa) - 1)) off_a[ka] += __popc(pa);
    if (kb != kSkip && lane == (uint32_t)(__ffs(pb) - 1)) off_b[kb] += __popc(pb);
    __syncwarp();
  }
  __syncthreads();
  // copy the runs out: item i of the stage lies in the segment g with
  // s_seg[g] <= i < s_seg[g + 1]
  const uint32_t total = s_seg[nseg];
  for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) {
    uint32_t lo = 0, hi = nseg;  // g in [lo, hi)
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (i >= s_seg[mid]) lo = mid; else hi = mid;
    }
    const uint32_t g = s_goff[lo] + (i - s_seg[lo]);
    out_src[g] = st_src[i];
    out_dst[g] = st_dst[i];
    if (w) out_w[g] = st_w[i];
  }
}

// tot[b] = edges to owner b (both passes), tot[nparts] = the error word.
__global__ void part_totals_kernel(const uint32_t* __restrict__ scan_a, const uint32_t* __restrict__ scan_b,
                                   uint32_t nparts, uint32_t nb, const uint32_t* __restrict__ err,
                                   uint32_t* __restrict__ tot) {
  for (uint32_t b = threadIdx.x; b <= nparts; b += blockDim.x)
    tot[b] = b < nparts ? (scan_a[(size_t)(b + 1) * nb] - scan_a[(size_t)b * nb]) +
                              (scan_b[(size_t)(b + 1) * nb] - scan_b[(size_t)b * nb])
                        : *err;
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
  const uint32_t nb = (uint32_t)(((uint64_t)E + kCtaEdges - 1) / kCtaEdges);  // CTAs
  const size_t n = (size_t)nparts * nb;
  if (n >= 0xFFFFFFFFull) return fail(ERR_ARG, "partition: too many edges for %u parts", nparts);
  const size_t tmpw = scan_tmp_words((uint32_t)n);
  // device scratch: bounds + error word, totals, two count arrays, two
  // scans, scan temp; each array on a 16-byte boundary
  auto up4 = [](size_t x) { return (x + 3) & ~(size_t)3; };
  const size_t o_tot = up4(kMaxParts + 2), o_cnt_a = o_tot + up4(kMaxParts + 1), o_cnt_b = o_cnt_a + up4(n),
               o_scan_a = o_cnt_b + up4(n), o_scan_b = o_scan_a + up4(n + 1), o_tmp = o_scan_b + up4(n + 1),
               words = o_tmp + up4(tmpw);
  // grow-only, one per host thread (threads may split shards concurrently)
  static thread_local DevBuf scratch;
  OGB_TRY(scratch.alloc(words * 4));
  uint32_t* d_bounds = scratch.as<uint32_t>();
  uint32_t* d_err = d_bounds + kMaxParts + 1;
  uint32_t* d_tot = d_bounds + o_tot;
  uint32_t* cnt_a = d_bounds + o_cnt_a;
  uint32_t* cnt_b = d_bounds + o_cnt_b;
  uint32_t* scan_a = d_bounds + o_scan_a;
  uint32_t* scan_b = d_bounds + o_scan_b;
  uint32_t* tmp = d_bounds + o_tmp;
  std::vector<uint32_t> htot(nparts + 1, 0);
  int rc = OK;
  auto run = [&]() -> int {
    OGB_CUDA(cudaMemcpyAsync(d_bounds, bounds, (nparts + 1) * 4, cudaMemcpyHostToDevice, s));
    OGB_CUDA(cudaMemsetAsync(d_err, 0, 4, s));
    part_count_kernel<<<nb, kPartThreads, 0, s>>>(src, dst, E, d_bounds, nparts, nb, cnt_a, cnt_b, d_err);
    OGB_CUDA(cudaGetLastError());
    OGB_TRY(scan_exclusive_u32(cnt_a, scan_a, (uint32_t)n, tmp, s));
    OGB_TRY(scan_exclusive_u32(cnt_b, scan_b, (uint32_t)n, tmp, s));
    const size_t stage = (size_t)(w ? 6 : 4) * kCtaEdges * 4;  // 2 kCtaEdges items of 2 or 3 words
    static thread_local bool attr_set = false;
    if (!attr_set) {
      OGB_CUDA(cudaFuncSetAttribute(part_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(6 * kCtaEdges * 4)));
      attr_set = true;
    }
    part_scatter_kernel<<<nb, kPartThreads, stage, s>>>(src, dst, w, E, d_bounds, nparts, nb, scan_a, scan_b,
                                                        out_src, out_dst, out_w, d_err);
    part_totals_kernel<<<1, 64, 0, s>>>(scan_a, scan_b, nparts, nb, d_err, d_tot);
    OGB_CUDA(cudaGetLastError());
    OGB_CUDA(cudaMemcpyAsync(htot.data(), d_tot, (nparts + 1) * 4, cudaMemcpyDeviceToHost, s));
    return OK;
  };
  rc = run();
  if (rc != OK) return rc;
  OGB_CUDA(cudaStreamSynchronize(s));  // the scratch is reused by this thread's next call
  if (htot[nparts]) return fail(ERR_RANGE, "partition: a vertex id is past the last range (%u)", bounds[nparts]);
  for (uint32_t b = 0; b < nparts; b++) counts[b] = htot[b];
  return OK;
}

}  // namespace ogb
