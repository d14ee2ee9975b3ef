// graph.cu -- CSR build on the device (both directions) and runtime helpers.
//
// Reference: graphCSRPreProcessingStep (00_graph_bench/src/structures/
// graphCSR.c:164-248) sorts the edge list, maps it to CSR
// (mapVerticesWithInOutDegree, vertex.c:204-325), makes the inverse list as
// a src/dst-swapped copy of the SORTED forward list (readEdgeListsMem,
// edgeList.c:597-745), sorts that copy with the same sort type and maps it.
// Here the swap costs nothing: the inverse sort reads the forward dst array
// as its key and the forward src array as its payload.
#include "graph.cuh"

#include <stdarg.h>
#include <mutex>
#include <unordered_map>

namespace ogb {

// ---------------------------------------------------------------- runtime --
static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

cudaStream_t lib_stream() {
  static std::mutex mu;
  static std::unordered_map<int, cudaStream_t> streams;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  streams[dev] = s;
  return s;
}

int sm_count() {
  static std::mutex mu;
  static std::unordered_map<int, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  if (n <= 0) n = 148;
  cache[dev] = n;
  return n;
}

DevGraph::~DevGraph() {
  dd_work_free(this);
  range_work_free(this);
  bfs_work_free(bfs);
  pr_work_free(pr);
  ms_work_free(ms);
  ppr_work_free(ppr);
}

// ------------------------------------------------------------- CSR kernels --

// Run starts and run ends of the sorted key array: edges_idx[s] = first
// index of s's run, end[s] = one past its last index (vertex.c:272-288).
// Keys >= V are reported through *err and skipped.
__global__ void __launch_bounds__(256) csr_boundary_kernel(const uint32_t* __restrict__ key, uint32_t E,
                                                           uint32_t V, uint32_t* __restrict__ edges_idx,
                                                           uint32_t* __restrict__ run_end,
                                                           uint32_t* __restrict__ err) {
  // four consecutive keys per thread (one 16-byte load; keys come from
  // cudaMalloc, so 16-byte aligned) plus the two neighbours of the group
  const uint32_t nq = E / 4;
  const uint4* kq = reinterpret_cast<const uint4*>(key);
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    const uint4 v = __ldg(kq + q);
    const uint32_t i0 = q * 4;
    const uint32_t k[6] = {i0 ? __ldg(key + i0 - 1) : 0xFFFFFFFFu, v.x, v.y, v.z, v.w,
                           i0 + 4 < E ? __ldg(key + i0 + 4) : 0xFFFFFFFFu};
#pragma unroll
    for (int j = 1; j <= 4; j++) {
      const uint32_t s = k[j];
      if (s >= V) {
        atomicExch(err, (uint32_t)ERR_RANGE);
        continue;
      }
      if (k[j - 1] != s) edges_idx[s] = i0 + j - 1;
      if (k[j + 1] != s) run_end[s] = i0 + j;
    }
  }
  // the last E % 4 keys
  for (uint32_t i = nq * 4 + blockIdx.x * blockDim.x + threadIdx.x; i < E; i += gridDim.x * blockDim.x) {
    const uint32_t s = key[i];
    if (s >= V) {
      atomicExch(err, (uint32_t)ERR_RANGE);
      continue;
    }
    if (i == 0 || key[i - 1] != s) edges_idx[s] = i;
    if (i + 1 == E || key[i + 1] != s) run_end[s] = i + 1;
  }
}

// out_degree = run_end - edges_idx (0 - 0 for vertices without edges),
// mirrored into the other direction's in_degree; rows packed.
__global__ void __launch_bounds__(256) csr_degree_kernel(uint32_t V, const uint32_t* __restrict__ edges_idx,
                                                         uint32_t* __restrict__ out_degree,
                                                         uint32_t* __restrict__ other_in_degree,
                                                         uint2* __restrict__ rows) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const uint32_t idx = edges_idx[v];
    const uint32_t d = out_degree[v] - idx;
    out_degree[v] = d;
    other_in_degree[v] = d;
    rows[v] = make_uint2(idx, d);
  }
}

__global__ void __launch_bounds__(256) csr_pack_kernel(uint32_t V, const uint32_t* __restrict__ edges_idx,
                                                       const uint32_t* __restrict__ out_degree,
                                                       uint2* __restrict__ rows) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    rows[v] = make_uint2(edges_idx[v], out_degree[v]);
}

static int reserve_csr(DevCSR& c, uint32_t V, uint32_t E, bool weighted) {
  OGB_TRY(c.src.alloc((size_t)E * 4));
  OGB_TRY(c.dst.alloc((size_t)E * 4));
  if (weighted) OGB_TRY(c.w.alloc((size_t)E * 4));
  OGB_TRY(c.out_degree.alloc((size_t)V * 4));
  OGB_TRY(c.in_degree.alloc((size_t)V * 4));
  OGB_TRY(c.edges_idx.alloc((size_t)V * 4));
  OGB_TRY(c.rows.alloc((size_t)V * 8));
  return OK;
}

int csr_map(DevCSR& c, DevCSR& other, uint32_t V, uint32_t E, uint32_t* d_err, cudaStream_t s) {
  if (V == 0) return OK;
  OGB_CUDA(cudaMemsetAsync(c.edges_idx.p, 0, (size_t)V * 4, s));
  OGB_CUDA(cudaMemsetAsync(c.out_degree.p, 0, (size_t)V * 4, s));
  const int grid = sm_count() * 8;
  if (E) {
    csr_boundary_kernel<<<grid, 256, 0, s>>>(c.d_src(), E, V, c.d_edges_idx(), c.d_out_degree(), d_err);
    OGB_CUDA(cudaGetLastError());
  }
  csr_degree_kernel<<<grid, 256, 0, s>>>(V, c.d_edges_idx(), c.d_out_degree(), other.d_in_degree(), c.d_rows());
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int csr_pack_rows(DevCSR& c, uint32_t V, cudaStream_t s) {
  if (V == 0) return OK;
  csr_pack_kernel<<<sm_count() * 8, 256, 0, s>>>(V, c.d_edges_idx(), c.d_out_degree(), c.d_rows());
  OGB_CUDA(cudaGetLastError());
  return OK;
}

int graph_build(DevGraph& g, const uint32_t* in_src, const uint32_t* in_dst, const float* in_w,
                uint32_t E, uint32_t V, uint32_t sort_type, cudaStream_t s) {
  if (V > (1u << 30)) return fail(ERR_RANGE, "graph_build: V=%u exceeds 2^30 (ids carry mask bits above)", V);
  const bool weighted = in_w != nullptr;
  g.V = V;
  g.E = E;
  g.weighted = weighted;
  g.sort_type = sort_type;
  g.build_id++;
  OGB_TRY(reserve_csr(g.fwd, V, E, weighted));
  OGB_TRY(reserve_csr(g.inv, V, E, weighted));
  OGB_TRY(g.err.alloc(16));
  OGB_CUDA(cudaMemsetAsync(g.err.p, 0, 16, s));
  const bool lex = (sort_type == 1 || sort_type == 3);

  // forward: sort by src (or by (src, dst))
  KV in{const_cast<uint32_t*>(in_src), const_cast<uint32_t*>(in_dst),
        reinterpret_cast<uint32_t*>(const_cast<float*>(in_w))};
  KV fwd{g.fwd.d_src(), g.fwd.d_dst(), weighted ? reinterpret_cast<uint32_t*>(g.fwd.d_w()) : nullptr};
  // ids are below V (a larger one fails the build in csr_map), so the sort
  // needs only the bits of V - 1
  uint32_t bits = 1;
  while (bits < 32 && (V - 1) >> bits) bits++;
  if (E) OGB_TRY(lex ? sort_pairs_lex(in, fwd, E, g.sort_ws, s, bits) : sort_pairs(in, fwd, E, g.sort_ws, s, bits));
  OGB_TRY(csr_map(g.fwd, g.inv, V, E, g.err.as<uint32_t>(), s));

  // inverse: the sorted forward list with src/dst swapped, sorted again
  KV inv_in{g.fwd.d_dst(), g.fwd.d_src(), fwd.v1};
  KV inv{g.inv.d_src(), g.inv.d_dst(), weighted ? reinterpret_cast<uint32_t*>(g.inv.d_w()) : nullptr};
  if (E)
    OGB_TRY(lex ? sort_pairs_lex(inv_in, inv, E, g.sort_ws, s, bits) : sort_pairs(inv_in, inv, E, g.sort_ws, s, bits));
  OGB_TRY(csr_map(g.inv, g.fwd, V, E, g.err.as<uint32_t>(), s));
  return OK;
}

int graph_check(DevGraph& g, cudaStream_t s) {
  OGB_TRY(sort_check(g.sort_ws, s));
  if (!g.err.p) return OK;
  uint32_t e = 0;
  OGB_CUDA(cudaMemcpyAsync(&e, g.err.p, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  if (e) return fail((int)e, "CSR build: a vertex id is >= V");
  return OK;
}

}  // namespace ogb
