// common.cuh -- shared helpers of the B200 CSR hot path: status codes, CUDA
// error capture, device buffers and warp primitives.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>

namespace ogb {

// Status codes of the device API (ogb200_device.h).  0 = success.
enum Status : int {
  OK = 0,
  ERR_CUDA = 1,          // a CUDA runtime call failed
  ERR_ARG = 2,           // invalid argument (size, root, null pointer)
  ERR_SPIN = 3,          // a bounded device wait gave up (look-back never resolved)
  ERR_RANGE = 4,         // vertex id out of the supported range
  ERR_NOMEM = 5,         // allocation failed
  ERR_UNSUPPORTED = 6,   // variant not provided by this library
  ERR_STATE = 7,         // a device-side consistency check failed (counters disagree)
};

// Last error message of the calling thread (set by fail()).
void set_last_error(const std::string& msg);
const char* last_error();

int fail(int code, const char* fmt, ...);

#define OGB_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess)                                                    \
      return ::ogb::fail(::ogb::ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, \
                         #call, cudaGetErrorString(_e));                      \
  } while (0)

#define OGB_TRY(call)            \
  do {                           \
    int _s = (call);             \
    if (_s != ::ogb::OK) return _s; \
  } while (0)

// Library stream: every reference-facing call runs on it.
cudaStream_t lib_stream();

// Number of SMs of the current device (cached per device).
int sm_count();

// A device allocation that frees itself.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  int alloc(size_t n) {
    if (n <= bytes && p) return OK;
    release();
    if (n == 0) return OK;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      p = nullptr;
      bytes = 0;
      return fail(ERR_NOMEM, "cudaMalloc(%zu): %s", n, cudaGetErrorString(e));
    }
    bytes = n;
    return OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// Upper bound on the polls of any device-side wait.  A wait that runs out
// records ERR_SPIN in the kernel's error word and returns; nothing spins
// forever.
constexpr uint32_t kSpinLimit = 1u << 24;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_volatile_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.volatile.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Warp-aggregated atomicAdd of a per-lane value: one atomic per warp for the
// lanes that call it together.  Only the total is added (no per-lane offset).
__device__ __forceinline__ void warp_atomic_add_total(uint32_t* ctr, uint32_t val) {
  uint32_t active = __activemask();
  uint32_t total = __reduce_add_sync(active, val);
  if ((int)lane_id() == __ffs(active) - 1) atomicAdd(ctr, total);
}

__device__ __forceinline__ void warp_atomic_add_total64(unsigned long long* ctr, uint32_t val) {
  uint32_t active = __activemask();
  uint32_t total = __reduce_add_sync(active, val);
  if ((int)lane_id() == __ffs(active) - 1) atomicAdd(ctr, (unsigned long long)total);
}

// Block-aggregated counter add: every thread of the block calls it with its
// own value (block-uniform call site); thread 0 adds the block total with one
// atomic, and none when the total is 0.  s_tmp holds one entry per warp.
template <class T>
__device__ __forceinline__ void block_add_total(T* ctr, T val, T* s_tmp) {
#pragma unroll
  for (int o = 16; o; o >>= 1) val += __shfl_down_sync(0xffffffffu, val, o);
  const uint32_t warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane_id() == 0) s_tmp[warp] = val;
  __syncthreads();
  if (threadIdx.x == 0) {
    T t = 0;
    for (uint32_t i = 0; i < nw; i++) t += s_tmp[i];
    if (t) atomicAdd(ctr, t);
  }
}

// Warp-aggregated increment by 1 (the common case): cheaper than the
// general version.
__device__ __forceinline__ uint32_t warp_atomic_inc(uint32_t* ctr) {
  uint32_t active = __activemask();
  int leader = __ffs(active) - 1;
  uint32_t n = __popc(active);
  uint32_t base = 0;
  if ((int)lane_id() == leader) base = atomicAdd(ctr, n);
  base = __shfl_sync(active, base, leader);
  return base + __popc(active & lanemask_lt());
}

// Block-level append buffer: items pushed by any thread of a block are staged
// in shared memory and written out with ONE global atomic per flush, instead
// of one atomic per warp on a counter every block shares.
template <int CAP>
struct BlockAppend {
  uint32_t n;     // staged items
  uint32_t base;  // global offset of the flush in progress
  uint32_t buf[CAP];
};

template <int CAP>
__device__ __forceinline__ void ba_init(BlockAppend<CAP>& q) {
  if (threadIdx.x == 0) q.n = 0;
  __syncthreads();
}

// Any thread, any divergence; the caller keeps n + pushes <= CAP.
template <int CAP>
__device__ __forceinline__ void ba_push(BlockAppend<CAP>& q, uint32_t x) {
  q.buf[warp_atomic_inc(&q.n)] = x;
}

// Staged count, uniform over the block (call from block-uniform code).
template <int CAP>
__device__ __forceinline__ uint32_t ba_size(BlockAppend<CAP>& q) {
  __syncthreads();
  const uint32_t n = q.n;
  __syncthreads();
  return n;
}

// Every thread of the block calls it: appends the staged items to out[] at
// an offset reserved from *count, then empties the buffer.
template <int CAP>
__device__ __forceinline__ void ba_flush(BlockAppend<CAP>& q, uint32_t* out, uint32_t* count) {
  __syncthreads();
  const uint32_t n = q.n;
  if (threadIdx.x == 0 && n) q.base = atomicAdd(count, n);
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) out[q.base + k] = q.buf[k];
  __syncthreads();
  if (threadIdx.x == 0) q.n = 0;
  __syncthreads();
}

inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace ogb
