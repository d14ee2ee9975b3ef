// sort.cu -- stable onesweep LSD radix sort for edge lists on sm_100a.
//
// Replaces the reference's 4-pass, 8-bit, per-thread-histogram LSD sort
// (00_graph_bench/src/preprocess/radixsort.c:46-135, :231-335) and its
// counting sort (countsort.c:28-270), whose outputs are identical: edges
// ordered by key, ties kept in input order.
//
// Design (one pass = one kernel, no separate upsweep):
//  * digit histograms of every 8-bit digit are built by one read of the keys;
//    digits that are constant over all keys are skipped (for V = 2^22 only
//    three passes run, the last with 6 live bits);
//  * each CTA claims a tile of kTile keys in launch order, ranks the keys of
//    the tile stably with warp match masks (order = warp, item, lane, which is
//    input order), publishes its per-digit counts and resolves the per-digit
//    prefix of all earlier tiles by decoupled look-back;
//  * keys and payloads are staged in shared memory in digit order and written
//    out so that consecutive threads store consecutive addresses of a run.
#include "sort.cuh"

#include <vector>

namespace ogb {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kTile = kSortThreads * kSortItems;
constexpr int kWarps = kSortThreads / 32;
constexpr int kMaxPasses = 8;  // 4 digits x (primary, secondary)
constexpr unsigned long long kFlagAgg = 1ull << 32;
constexpr unsigned long long kFlagInc = 2ull << 32;

// counters layout (u32): [0, kMaxPasses) tile counters, [kMaxPasses] error
// word, [kMaxPasses+1] OR of all primary keys, [kMaxPasses+2] OR of all
// secondary keys.
constexpr int kCtrErr = kMaxPasses;
constexpr int kCtrOr0 = kMaxPasses + 1;
constexpr int kCtrWords = kMaxPasses + 4;

__device__ __forceinline__ uint32_t block_exclusive_scan_256(uint32_t v, uint32_t* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < kWarps) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < kWarps; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kWarps) s_warp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  uint32_t warp_excl = warp ? s_warp[warp - 1] : 0;
  return warp_excl + x - v;
}

// Histograms of `ndig` digits of keys[0, n) into hist[ndig][256] (digit d
// = (key >> 8-aligned or narrower lay.shift[d]) & lay.mask[d]) and the OR of
// all keys into *or_out.  Each warp counts into its own copy of
// the histograms in shared memory (conflicts only inside a warp's atomic),
// and the copies are summed once at the end.
// The digits of one key: ndig groups of at most 8 bits from bit 0 up.
struct DigitLayout {
  int ndig;
  uint32_t shift[4], mask[4];
};

// Digits for keys below 2^bits: ceil(bits / 8) groups of nearly equal
// width (the lower ones one bit wider), so each pass's digit runs are as
// long as the key width allows (22 bits: 8 + 7 + 7 instead of 8 + 8 + 6).
static DigitLayout digit_layout(uint32_t bits) {
  bits = bits < 1 ? 1 : (bits > 32 ? 32 : bits);
  DigitLayout l;
  l.ndig = (int)((bits + 7) / 8);
  const uint32_t w = bits / l.ndig, extra = bits % l.ndig;
  uint32_t sh = 0;
  for (int d = 0; d < 4; d++) {
    const uint32_t wd = d < l.ndig ? w + ((uint32_t)d < extra ? 1u : 0u) : 0u;
    l.shift[d] = sh;
    l.mask[d] = wd ? (wd >= 32 ? 0xFFFFFFFFu : (1u << wd) - 1u) : 0u;
    sh += wd;
  }
  return l;
}

constexpr int kHistThreads = 256, kHistWarps = kHistThreads / 32;
__global__ void __launch_bounds__(kHistThreads) digit_hist_kernel(const uint32_t* __restrict__ keys, uint64_t n,
                                                                  int ndig, DigitLayout lay,
                                                                  uint32_t* __restrict__ hist,
                                                                  uint32_t* __restrict__ or_out) {
  __shared__ uint32_t sh[kHistWarps][4][256];
  __shared__ uint32_t s_or;
  for (int i = threadIdx.x; i < kHistWarps * 4 * 256; i += blockDim.x) (&sh[0][0][0])[i] = 0;
  if (threadIdx.x == 0) s_or = 0;
  __syncthreads();
  uint32_t(*h)[256] = sh[threadIdx.x >> 5];
  uint32_t acc_or = 0;
  const uint64_t nvec = n / 4;
  const uint4* kv = reinterpret_cast<const uint4*>(keys);
  const bool aligned = (reinterpret_cast<uintptr_t>(keys) & 15) == 0;
  uint64_t start_scalar = 0;
  if (aligned) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec;
         i += (uint64_t)gridDim.x * blockDim.x) {
      const uint4 q = __ldg(kv + i);
      const uint32_t a[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int j = 0; j < 4; j++) {
        acc_or |= a[j];
#pragma unroll
        for (int d = 0; d < 4; d++)
          if (d < ndig) atomicAdd(&h[d][(a[j] >> lay.shift[d]) & lay.mask[d]], 1u);
      }
    }
    start_scalar = nvec * 4;
  }
  for (uint64_t i = start_scalar + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    acc_or |= k;
#pragma unroll
    for (int d = 0; d < 4; d++)
      if (d < ndig) atomicAdd(&h[d][(k >> lay.shift[d]) & lay.mask[d]], 1u);
  }
  acc_or = __reduce_or_sync(0xffffffffu, acc_or);
  if ((threadIdx.x & 31) == 0) atomicOr(&s_or, acc_or);
  __syncthreads();
  for (int i = threadIdx.x; i < ndig * 256; i += blockDim.x) {
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < kHistWarps; w++) c += (&sh[w][0][0])[i];
    if (c) atomicAdd(&hist[i], c);
  }
  if (threadIdx.x == 0) atomicOr(or_out, s_or);
}

// Exclusive scan of each 256-bucket histogram (one block per histogram).
__global__ void __launch_bounds__(256) digit_scan_kernel(const uint32_t* __restrict__ hist,
                                                         uint32_t* __restrict__ base) {
  __shared__ uint32_t s_warp[kWarps];
  uint32_t v = hist[blockIdx.x * 256 + threadIdx.x];
  uint32_t e = block_exclusive_scan_256(v, s_warp);
  base[blockIdx.x * 256 + threadIdx.x] = e;
}

__device__ __forceinline__ void cp_async_u32(uint32_t* dst_smem, const uint32_t* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// One pass over one tile.  Only the keys pass through registers: once the
// tile-local digit prefix is known, each payload element is copied from
// global memory straight into its slot of the digit-ordered stage by an
// asynchronous copy, and those copies land while the look-back runs; the
// kernel holds no payload registers.  Keys and payloads are then written out
// run by run (consecutive threads, consecutive addresses).  Shared memory: a
// stage per array (32 KB unweighted: four CTAs per SM; 48 KB weighted: three).
template <bool HAS_P1>
__global__ void __launch_bounds__(kSortThreads, HAS_P1 ? 3 : 4)
onesweep_kernel(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ p0in,
                const uint32_t* __restrict__ p1in, uint32_t* __restrict__ kout,
                uint32_t* __restrict__ p0out, uint32_t* __restrict__ p1out, uint32_t n,
                uint32_t shift, uint32_t mask, const uint32_t* __restrict__ digit_base,
                unsigned long long* __restrict__ status, uint32_t* __restrict__ tile_ctr,
                uint32_t* __restrict__ err) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_whist[kWarps][256];
  __shared__ uint32_t s_local_start[256];
  __shared__ uint32_t s_global_start[256];
  __shared__ uint32_t s_warp[kWarps];
  extern __shared__ uint32_t s_dyn[];  // kTile keys, kTile payload0 [, kTile payload1]
  uint32_t* s_k = s_dyn;
  uint32_t* s_p0 = s_dyn + kTile;
  uint32_t* s_p1 = s_dyn + 2 * kTile;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
  for (int i = tid; i < kWarps * 256; i += kSortThreads) (&s_whist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t tile_base = (uint64_t)tile * kTile;
  const uint64_t warp_base = tile_base + (uint64_t)warp * 32 * kSortItems;
  // this warp's items: [0, wn) of kSortItems * 32, addressed from per-warp bases
  const uint32_t wn = n > warp_base ? (uint32_t)min((uint64_t)kSortItems * 32, (uint64_t)n - warp_base) : 0u;
  const uint32_t* kw = kin + warp_base;

  uint32_t key[kSortItems], pos[kSortItems];
#pragma unroll
  for (int i = 0; i < kSortItems; i++) {
    const uint32_t o = (uint32_t)i * 32 + lane;
    key[i] = o < wn ? kw[o] : 0xFFFFFFFFu;
  }

  // Stable warp-level ranking: order within the warp is (item, lane).
  uint32_t* wh = s_whist[warp];
#pragma unroll
  for (int i = 0; i < kSortItems; i++) {
    const uint32_t d = ((uint32_t)i * 32 + lane < wn) ? ((key[i] >> shift) & mask) : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t before = (d < 256) ? wh[d] : 0u;
    __syncwarp();
    if (d < 256 && lane == __ffs(peers) - 1) wh[d] = before + __popc(peers);
    __syncwarp();
    pos[i] = before + __popc(peers & lanemask_lt());
  }
  __syncthreads();

  // Per digit (thread = digit): exclusive prefix over warps, tile count.
  uint32_t cnt = 0;
#pragma unroll
  for (int w = 0; w < kWarps; w++) {
    uint32_t c = s_whist[w][tid];
    s_whist[w][tid] = cnt;
    cnt += c;
  }
  // digits above the mask never occur in this pass: no status, no look-back
  const bool live = (uint32_t)tid <= mask;
  unsigned long long* my_status = status + (uint64_t)tile * 256 + tid;
  if (live) st_volatile_u64(my_status, (tile == 0 ? kFlagInc : kFlagAgg) | cnt);
  const uint32_t local_start = block_exclusive_scan_256(cnt, s_warp);
  s_local_start[tid] = local_start;
  __syncthreads();

  // Stage slots (digit order within the tile): keys staged, payloads copied
  // into their slots asynchronously.
  {
    const uint32_t* p0w = p0in + warp_base;
    const uint32_t* p1w = HAS_P1 ? p1in + warp_base : nullptr;
#pragma unroll
    for (int i = 0; i < kSortItems; i++) {
      const uint32_t o = (uint32_t)i * 32 + lane;
      if (o < wn) {
        const uint32_t d = (key[i] >> shift) & mask;
        const uint32_t p = s_local_start[d] + s_whist[warp][d] + pos[i];
        s_k[p] = key[i];
        cp_async_u32(&s_p0[p], p0w + o);
        if (HAS_P1) cp_async_u32(&s_p1[p], p1w + o);
      }
    }
  }

  // Decoupled look-back over earlier tiles for this digit.
  uint32_t excl = 0;
  if (tile > 0 && live) {
    int64_t pred = (int64_t)tile - 1;
    uint32_t spins = 0;
    while (pred >= 0) {
      unsigned long long s = ld_volatile_u64(status + (uint64_t)pred * 256 + tid);
      unsigned long long flag = s & ~0xFFFFFFFFull;
      if (flag == 0) {
        if (++spins > kSpinLimit) {
          atomicExch(err, (uint32_t)ERR_SPIN);
          break;
        }
        continue;
      }
      excl += (uint32_t)s;
      if (flag == kFlagInc) break;
      --pred;
    }
    st_volatile_u64(my_status, kFlagInc | (unsigned long long)(excl + cnt));
  }
  s_global_start[tid] = digit_base[tid] + excl - local_start;
  cp_async_commit_wait_all();
  __syncthreads();

  const uint32_t valid = (uint32_t)min((uint64_t)kTile, (uint64_t)n - tile_base);
#pragma unroll 4
  for (uint32_t j = tid; j < valid; j += kSortThreads) {
    const uint32_t k = s_k[j];
    const uint32_t o = s_global_start[(k >> shift) & mask] + j;
    kout[o] = k;
    p0out[o] = s_p0[j];
    if (HAS_P1) p1out[o] = s_p1[j];
  }
}

struct PinnedCounts {
  uint32_t* h = nullptr;  // 8*256 counts + kCtrWords counters
  PinnedCounts() {
    if (cudaMallocHost(&h, (8 * 256 + kCtrWords) * sizeof(uint32_t)) != cudaSuccess) h = nullptr;
  }
};

PinnedCounts& pinned_counts() {
  static thread_local PinnedCounts pc;
  return pc;
}

struct PassPlan {
  int role;  // 0: key = primary (k), payloads (v0, v1); 1: key = secondary (v0), payloads (k, v1)
  uint32_t shift, mask;
  int hist_index;  // which 256-bucket histogram holds the digit counts
};

}  // namespace

int SortWorkspace::reserve(uint64_t n, bool weighted, int max_passes) {
  const uint64_t tiles = (n + kTile - 1) / kTile;
  OGB_TRY(hist.alloc(2 * 8 * 256 * sizeof(uint32_t)));
  OGB_TRY(status.alloc((size_t)max_passes * tiles * 256 * sizeof(unsigned long long) + 256));
  OGB_TRY(counters.alloc(kCtrWords * sizeof(uint32_t)));
  OGB_TRY(tmp_k.alloc(n * 4));
  OGB_TRY(tmp_v0.alloc(n * 4));
  if (weighted) OGB_TRY(tmp_v1.alloc(n * 4));
  return OK;
}

static int sort_impl(const KV& in, const KV& out, uint64_t n, bool lex, uint32_t key_bits, SortWorkspace& ws,
                     cudaStream_t stream) {
  if (n == 0) return OK;
  if (n > 0xFFFFFFFFull) return fail(ERR_ARG, "sort: %llu edges exceed the u32 edge count", (unsigned long long)n);
  if (in.k == out.k || in.v0 == out.v0) return fail(ERR_ARG, "sort: input and output arrays must differ");
  const bool has_p1 = in.v1 != nullptr;
  if (has_p1 && !out.v1) return fail(ERR_ARG, "sort: weighted input needs a weighted output");
  OGB_TRY(ws.reserve(n, has_p1, lex ? 8 : 4));

  uint32_t* d_hist = ws.hist.as<uint32_t>();   // [8][256] counts
  uint32_t* d_base = d_hist + 8 * 256;         // [8][256] exclusive bases
  uint32_t* d_ctr = ws.counters.as<uint32_t>();
  OGB_CUDA(cudaMemsetAsync(d_hist, 0, 8 * 256 * sizeof(uint32_t), stream));
  OGB_CUDA(cudaMemsetAsync(d_ctr, 0, kCtrWords * sizeof(uint32_t), stream));

  const int grid = sm_count() * 4;
  // hist[0..3]: primary key digits; hist[4..7]: secondary key digits (lex).
  const DigitLayout lay = digit_layout(key_bits);
  digit_hist_kernel<<<grid, 256, 0, stream>>>(in.k, n, lay.ndig, lay, d_hist, d_ctr + kCtrOr0);
  if (lex)
    digit_hist_kernel<<<grid, 256, 0, stream>>>(in.v0, n, lay.ndig, lay, d_hist + 4 * 256, d_ctr + kCtrOr0 + 1);
  OGB_CUDA(cudaGetLastError());
  digit_scan_kernel<<<lex ? 8 : 4, 256, 0, stream>>>(d_hist, d_base);
  OGB_CUDA(cudaGetLastError());

  PinnedCounts& pc = pinned_counts();
  if (!pc.h) return fail(ERR_NOMEM, "cudaMallocHost for sort counts failed");
  OGB_CUDA(cudaMemcpyAsync(pc.h, d_hist, 8 * 256 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
  OGB_CUDA(cudaStreamSynchronize(stream));

  // LSD order: secondary digits first (lex), then primary digits.
  std::vector<PassPlan> plan;
  auto add_passes = [&](int role, int hbase) {
    for (int d = 0; d < lay.ndig; d++) {
      const uint32_t* h = pc.h + (hbase + d) * 256;
      bool trivial = false;
      for (int b = 0; b < 256; b++)
        if (h[b] == n) trivial = true;
      if (!trivial) plan.push_back({role, lay.shift[d], lay.mask[d], hbase + d});
    }
  };
  if (lex) add_passes(1, 4);
  add_passes(0, 0);

  const int P = (int)plan.size();
  if (P == 0) {
    OGB_CUDA(cudaMemcpyAsync(out.k, in.k, n * 4, cudaMemcpyDeviceToDevice, stream));
    OGB_CUDA(cudaMemcpyAsync(out.v0, in.v0, n * 4, cudaMemcpyDeviceToDevice, stream));
    if (has_p1) OGB_CUDA(cudaMemcpyAsync(out.v1, in.v1, n * 4, cudaMemcpyDeviceToDevice, stream));
    return OK;
  }
  const uint64_t tiles = (n + kTile - 1) / kTile;
  const size_t dyn_smem = (size_t)(has_p1 ? 3 : 2) * kTile * sizeof(uint32_t);  // a stage per array
  static bool attr_set = false;
  if (!attr_set) {
    OGB_CUDA(cudaFuncSetAttribute(onesweep_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 3 * kTile * 4));
    OGB_CUDA(cudaFuncSetAttribute(onesweep_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kTile * 4));
    attr_set = true;
  }
  OGB_CUDA(cudaMemsetAsync(ws.status.p, 0, (size_t)P * tiles * 256 * sizeof(unsigned long long), stream));

  KV tmp{ws.tmp_k.as<uint32_t>(), ws.tmp_v0.as<uint32_t>(), has_p1 ? ws.tmp_v1.as<uint32_t>() : nullptr};
  KV cur = in;
  for (int i = 0; i < P; i++) {
    const KV dst = ((P - 1 - i) % 2 == 0) ? out : tmp;
    const PassPlan& pp = plan[i];
    const uint32_t* kin = pp.role == 0 ? cur.k : cur.v0;
    const uint32_t* p0in = pp.role == 0 ? cur.v0 : cur.k;
    uint32_t* kout = pp.role == 0 ? dst.k : dst.v0;
    uint32_t* p0out = pp.role == 0 ? dst.v0 : dst.k;
    unsigned long long* st = ws.status.as<unsigned long long>() + (uint64_t)i * tiles * 256;
    if (has_p1)
      onesweep_kernel<true><<<(unsigned)tiles, kSortThreads, dyn_smem, stream>>>(
          kin, p0in, cur.v1, kout, p0out, dst.v1, (uint32_t)n, pp.shift, pp.mask, d_base + pp.hist_index * 256, st,
          d_ctr + i, d_ctr + kCtrErr);
    else
      onesweep_kernel<false><<<(unsigned)tiles, kSortThreads, dyn_smem, stream>>>(
          kin, p0in, nullptr, kout, p0out, nullptr, (uint32_t)n, pp.shift, pp.mask, d_base + pp.hist_index * 256, st,
          d_ctr + i, d_ctr + kCtrErr);
    OGB_CUDA(cudaGetLastError());
    cur = dst;
  }
  return OK;
}

int sort_pairs(const KV& in, const KV& out, uint64_t n, SortWorkspace& ws, cudaStream_t stream, uint32_t key_bits) {
  return sort_impl(in, out, n, false, key_bits, ws, stream);
}

int sort_pairs_lex(const KV& in, const KV& out, uint64_t n, SortWorkspace& ws, cudaStream_t stream,
                   uint32_t key_bits) {
  return sort_impl(in, out, n, true, key_bits, ws, stream);
}

// Reads the error word of the last sorts on `stream` (synchronizes).
int sort_check(SortWorkspace& ws, cudaStream_t stream) {
  if (!ws.counters.p) return OK;
  uint32_t e = 0;
  OGB_CUDA(cudaMemcpyAsync(&e, ws.counters.as<uint32_t>() + kCtrErr, 4, cudaMemcpyDeviceToHost, stream));
  OGB_CUDA(cudaStreamSynchronize(stream));
  if (e) return fail((int)e, "radix sort: decoupled look-back wait gave up");
  return OK;
}

}  // namespace ogb
