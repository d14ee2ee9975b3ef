// abi.cu -- the OpenGraph C API over the device hot path (drop-in layer).
//
// Compiled twice: OGB200_WEIGHTED=0 -> libogb200.so, =1 -> libogb200_w.so.
// Host structs keep the reference layouts (ogb200.h); sorting, CSR mapping,
// BFS and PageRank run on the GPU.  A GraphCSR made by graphCSRPreProcessingStep
// keeps its device copy in a side table keyed by the GraphCSR pointer, so the
// algorithms do not upload it again; graphCSRFree drops it.  A GraphCSR built
// elsewhere (for example by the reference's own CPU code) is uploaded on its
// first use.
//
// Observable behaviour follows the reference: progress tables on stdout in the
// reference's format, err(1)-style exits on I/O errors, NULL for unsupported
// variants.  CUDA failures print the CUDA error and exit(1).
#include <err.h>
#include <fcntl.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <emmintrin.h>
#include <omp.h>
#include <unistd.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ogb200.h"
#include "../../include/ogb200_device.h"
#include "graph.cuh"

using namespace ogb;

// ------------------------------------------------------------------ misc ----

static int g_quiet = -1;

static bool quiet() {
  if (g_quiet < 0) {
    const char* e = getenv("OGB200_QUIET");
    g_quiet = (e && *e && *e != '0') ? 1 : 0;
  }
  return g_quiet == 1;
}

static void say(const char* fmt, ...) {
  if (quiet()) return;
  va_list ap;
  va_start(ap, fmt);
  vprintf(fmt, ap);
  va_end(ap);
}

static void print_msg_time(const char* msg, double t) {
  say(" -----------------------------------------------------\n");
  say("| %-51s | \n", msg);
  say(" -----------------------------------------------------\n");
  say("| %-51f | \n", t);
  say(" -----------------------------------------------------\n");
}

static double now_s() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + tv.tv_usec / 1e6;
}

// Allocation as the reference's my_malloc (128-byte aligned, free()-able).
static void* host_alloc(size_t bytes) {
  void* p = nullptr;
  if (posix_memalign(&p, 128, bytes ? bytes : 128) != 0 || !p) {
    fprintf(stderr, "Error, aligned_alloc!\n");
    exit(EXIT_FAILURE);
  }
  return p;
}

// Result arrays recycled between calls.  freeBFSStats / freePageRankStats
// hand their arrays back here and the next stats allocation of the same size
// takes them, so a call writes into pages that are already mapped instead of
// first-touching (page-faulting) fresh memory -- at V = 4M that is 12k faults
// per BFS call.  The arrays are ordinary posix_memalign memory: a caller
// that releases them with free() simply never returns them.  At most
// kPoolBytes stay parked; the rest is freed.
namespace {
struct HostPool {
  static constexpr size_t kPoolBytes = size_t(1) << 30;
  std::mutex mu;
  std::vector<std::pair<size_t, void*>> parked;
  size_t bytes = 0;
  ~HostPool() {
    for (auto& e : parked) free(e.second);
  }
};
HostPool& host_pool() {
  static HostPool p;
  return p;
}
}  // namespace

static void* pool_alloc(size_t n) {
  HostPool& P = host_pool();
  {
    std::lock_guard<std::mutex> lk(P.mu);
    for (size_t i = P.parked.size(); i-- > 0;) {
      if (P.parked[i].first == n) {
        void* p = P.parked[i].second;
        P.parked.erase(P.parked.begin() + (long)i);
        P.bytes -= n;
        return p;
      }
    }
  }
  return host_alloc(n);
}

static void pool_free(void* p, size_t n) {
  if (!p) return;
  HostPool& P = host_pool();
  std::lock_guard<std::mutex> lk(P.mu);
  if (P.bytes + n <= HostPool::kPoolBytes) {
    P.parked.emplace_back(n, p);
    P.bytes += n;
  } else {
    free(p);
  }
}

[[noreturn]] static void die_status(const char* where, int st) {
  fprintf(stderr, "ogb200: %s failed (status %d): %s\n", where, st, ogb::last_error());
  exit(1);
}

#define OGB_MUST(call)                     \
  do {                                     \
    int _st = (call);                      \
    if (_st != ::ogb::OK) die_status(#call, _st); \
  } while (0)

// A CUDA runtime call at the OpenGraph boundary: print and exit on failure.
#define OGB_CUDA_MUST(call)                                                                  \
  do {                                                                                       \
    cudaError_t _e = (call);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      fprintf(stderr, "ogb200: %s failed: %s\n", #call, cudaGetErrorString(_e));              \
      exit(1);                                                                               \
    }                                                                                        \
  } while (0)

// Host <-> device copies of malloc'd (pageable) arrays run through pinned
// bounce buffers: kBufs chunks in flight on the DMA engine while OpenMP
// threads move the previous chunk between the bounce buffer and the array.
namespace {
struct Bounce {
  static constexpr size_t kChunk = 8u << 20;
  static constexpr int kBufs = 4;
  void* h[kBufs] = {};
  cudaEvent_t ev[kBufs] = {};
  std::mutex mu;
  int init() {
    if (h[0]) return OK;
    for (int i = 0; i < kBufs; i++) {
      OGB_CUDA(cudaMallocHost(&h[i], kChunk));
      OGB_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    }
    return OK;
  }
};
Bounce& bounce() {
  static Bounce b;
  return b;
}

int host_threads() {
  static const int n = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
  return n;
}

void par_memcpy(void* dst, const void* src, size_t n) {
  const size_t kBlock = 1u << 20;
  if (n < (2u << 20)) {
    memcpy(dst, src, n);
    return;
  }
  const long nb = (long)((n + kBlock - 1) / kBlock);
#pragma omp parallel for num_threads(host_threads()) schedule(static)
  for (long b = 0; b < nb; b++) {
    const size_t lo = (size_t)b * kBlock;
    memcpy((char*)dst + lo, (const char*)src + lo, std::min(kBlock, n - lo));
  }
}
}  // namespace

static int h2d(void* d, const void* h, size_t n, cudaStream_t s) {
  if (!n) return OK;
  Bounce& b = bounce();
  std::lock_guard<std::mutex> lk(b.mu);
  OGB_TRY(b.init());
  size_t off = 0;
  int i = 0;
  while (off < n) {
    const size_t len = std::min(Bounce::kChunk, n - off);
    OGB_CUDA(cudaEventSynchronize(b.ev[i]));  // buffer i free again
    par_memcpy(b.h[i], (const char*)h + off, len);
    OGB_CUDA(cudaMemcpyAsync((char*)d + off, b.h[i], len, cudaMemcpyHostToDevice, s));
    OGB_CUDA(cudaEventRecord(b.ev[i], s));
    off += len;
    i = (i + 1) % Bounce::kBufs;
  }
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

static int d2h(void* h, const void* d, size_t n, cudaStream_t s) {
  if (!n) return OK;
  Bounce& b = bounce();
  std::lock_guard<std::mutex> lk(b.mu);
  OGB_TRY(b.init());
  const size_t nchunks = (n + Bounce::kChunk - 1) / Bounce::kChunk;
  size_t issued = 0;
  // keep up to kBufs chunks queued on the copy engine, drain in order
  for (size_t k = 0; k < nchunks; k++) {
    while (issued < nchunks && issued < k + Bounce::kBufs) {
      const size_t off = issued * Bounce::kChunk;
      const int i = (int)(issued % Bounce::kBufs);
      OGB_CUDA(cudaMemcpyAsync(b.h[i], (const char*)d + off, std::min(Bounce::kChunk, n - off),
                               cudaMemcpyDeviceToHost, s));
      OGB_CUDA(cudaEventRecord(b.ev[i], s));
      issued++;
    }
    const int i = (int)(k % Bounce::kBufs);
    const size_t off = k * Bounce::kChunk;
    OGB_CUDA(cudaEventSynchronize(b.ev[i]));
    par_memcpy((char*)h + off, b.h[i], std::min(Bounce::kChunk, n - off));
  }
  return OK;
}

// Run fn(lo, hi) over [0, n) on the OpenMP host threads (as the reference's
// own parallel loops).
template <class F>
static void host_par_for(size_t n, F&& fn) {
  if (n < (1u << 16)) {
    fn((size_t)0, n);
    return;
  }
  const long nb = 256;
  const size_t chunk = (n + nb - 1) / nb;
#pragma omp parallel for num_threads(host_threads()) schedule(static)
  for (long b = 0; b < nb; b++) {
    const size_t lo = (size_t)b * chunk, hi = std::min(n, lo + chunk);
    if (lo < hi) fn(lo, hi);
  }
}

// ---------------------------------------------------------- device mirror ---

struct ogb_graph {
  DevGraph g;
  DevBuf d_parents, d_distances, d_ranks;  // result arrays of the drop-in calls
  DevBuf d_depth8;                         // BFS depths as bytes, for the host copy
};

namespace {
struct MirrorEntry {
  ogb_graph* dg;
  const void* fwd_dst;   // host pointers the copy was made from
  const void* inv_dst;
  uint32_t V, E;
};
std::mutex g_mirror_mu;
std::unordered_map<const GraphCSR*, MirrorEntry> g_mirrors;

int upload_graph(const GraphCSR* h, ogb_graph* dg, cudaStream_t s) {
  DevGraph& g = dg->g;
  const uint32_t V = h->num_vertices, E = h->num_edges;
  if (!h->vertices || !h->sorted_edges_array || !h->inverse_vertices || !h->inverse_sorted_edges_array)
    return fail(ERR_ARG, "GraphCSR without both directions");
  g.V = V;
  g.E = E;
  g.weighted = false;
  g.build_id++;
  for (int dir = 0; dir < 2; dir++) {
    DevCSR& c = dir ? g.inv : g.fwd;
    const Vertex* hv = dir ? h->inverse_vertices : h->vertices;
    const EdgeList* he = dir ? h->inverse_sorted_edges_array : h->sorted_edges_array;
    OGB_TRY(c.dst.alloc((size_t)E * 4 + 4));
    OGB_TRY(c.out_degree.alloc((size_t)V * 4 + 4));
    OGB_TRY(c.in_degree.alloc((size_t)V * 4 + 4));
    OGB_TRY(c.edges_idx.alloc((size_t)V * 4 + 4));
    OGB_TRY(c.rows.alloc((size_t)V * 8 + 8));
    OGB_TRY(h2d(c.dst.p, he->edges_array_dest, (size_t)E * 4, s));
    OGB_TRY(h2d(c.out_degree.p, hv->out_degree, (size_t)V * 4, s));
    OGB_TRY(h2d(c.in_degree.p, hv->in_degree, (size_t)V * 4, s));
    OGB_TRY(h2d(c.edges_idx.p, hv->edges_idx, (size_t)V * 4, s));
    OGB_TRY(csr_pack_rows(c, V, s));
#if OGB200_WEIGHTED
    // the WEIGHTED layout carries edge weights (SPMV reads them)
    if (he->edges_array_weight) {
      OGB_TRY(c.w.alloc((size_t)E * 4 + 4));
      OGB_TRY(h2d(c.w.p, he->edges_array_weight, (size_t)E * 4, s));
    }
#endif
  }
#if OGB200_WEIGHTED
  g.weighted = h->sorted_edges_array->edges_array_weight && h->inverse_sorted_edges_array->edges_array_weight;
#endif
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}
}  // namespace

static ogb_graph* mirror_of(const GraphCSR* h, int* status) {
  std::lock_guard<std::mutex> lk(g_mirror_mu);
  auto it = g_mirrors.find(h);
  if (it != g_mirrors.end()) {
    const MirrorEntry& m = it->second;
    if (m.V == h->num_vertices && m.E == h->num_edges && m.fwd_dst == h->sorted_edges_array->edges_array_dest &&
        m.inv_dst == h->inverse_sorted_edges_array->edges_array_dest) {
      *status = OK;
      return m.dg;
    }
    delete m.dg;
    g_mirrors.erase(it);
  }
  ogb_graph* dg = new ogb_graph();
  int st = upload_graph(h, dg, lib_stream());
  if (st != OK) {
    delete dg;
    *status = st;
    return nullptr;
  }
  g_mirrors[h] = {dg, h->sorted_edges_array->edges_array_dest, h->inverse_sorted_edges_array->edges_array_dest,
                  h->num_vertices, h->num_edges};
  *status = OK;
  return dg;
}

static void mirror_set(const GraphCSR* h, ogb_graph* dg) {
  std::lock_guard<std::mutex> lk(g_mirror_mu);
  auto it = g_mirrors.find(h);
  if (it != g_mirrors.end()) {
    if (it->second.dg != dg) delete it->second.dg;
    g_mirrors.erase(it);
  }
  g_mirrors[h] = {dg, h->sorted_edges_array->edges_array_dest, h->inverse_sorted_edges_array->edges_array_dest,
                  h->num_vertices, h->num_edges};
}

static void mirror_drop(const GraphCSR* h) {
  std::lock_guard<std::mutex> lk(g_mirror_mu);
  auto it = g_mirrors.find(h);
  if (it != g_mirrors.end()) {
    delete it->second.dg;
    g_mirrors.erase(it);
  }
}

// ------------------------------------------------------------ RNG (MT) -----
// Mersenne Twister MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998)
// with the 1999 "sgenrand" seeding by the linear congruential map
// x -> 69069 x + 1 that the reference uses (mt19937.c:54-67), so that root
// draws and generated weights match it bit for bit.

extern "C" void initializeMersenneState(mt19937state* m, unsigned long seed) {
  unsigned long x = seed;
  for (int i = 0; i < 624; i++) {
    unsigned long hi = x & 0xffff0000UL;
    x = 69069UL * x + 1UL;
    unsigned long lo = (x & 0xffff0000UL) >> 16;
    x = 69069UL * x + 1UL;
    m->mt[i] = hi | lo;
  }
  m->mti = 624;
}

extern "C" unsigned long generateRandInt(mt19937state* m) {
  const unsigned long upper = 0x80000000UL, lower = 0x7fffffffUL, twist = 0x9908b0dfUL;
  if (m->mti >= 624) {
    for (int k = 0; k < 624; k++) {
      const unsigned long y = (m->mt[k] & upper) | (m->mt[(k + 1) % 624] & lower);
      m->mt[k] = m->mt[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1UL) ? twist : 0UL);
    }
    m->mti = 0;
  }
  unsigned long y = m->mt[m->mti++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680UL;
  y ^= (y << 15) & 0xefc60000UL;
  y ^= y >> 18;
  return y;
}

extern "C" float generateRandFloat(mt19937state* m) {
  return ((float)generateRandInt(m)) * 2.3283064370807974e-10;
}

// ------------------------------------------------------------ edge lists ---

extern "C" struct EdgeList* newEdgeList(uint32_t num_edges) {
  EdgeList* e = (EdgeList*)host_alloc(sizeof(EdgeList));
  e->edges_array_src = (uint32_t*)host_alloc((size_t)num_edges * 4);
  e->edges_array_dest = (uint32_t*)host_alloc((size_t)num_edges * 4);
  memset(e->edges_array_src, 0, (size_t)num_edges * 4);
  memset(e->edges_array_dest, 0, (size_t)num_edges * 4);
#if OGB200_WEIGHTED
  e->edges_array_weight = (float*)host_alloc((size_t)num_edges * 4);
  memset(e->edges_array_weight, 0, (size_t)num_edges * 4);
  e->max_weight = 0;
#endif
  e->mask_array = nullptr;
  e->label_array = nullptr;
  e->inverse_label_array = nullptr;
  e->num_edges = num_edges;
  e->num_vertices = 0;
  e->avg_degree = 0;
  return e;
}

extern "C" void freeEdgeList(struct EdgeList* e) {
  if (!e) return;
  free(e->edges_array_src);
  free(e->edges_array_dest);
  free(e->mask_array);
  free(e->label_array);
  free(e->inverse_label_array);
#if OGB200_WEIGHTED
  free(e->edges_array_weight);
#endif
  free(e);
}

static void alloc_labels(EdgeList* e, uint32_t V) {
  e->mask_array = (uint32_t*)host_alloc((size_t)V * 4);
  e->label_array = (uint32_t*)host_alloc((size_t)V * 4);
  e->inverse_label_array = (uint32_t*)host_alloc((size_t)V * 4);
  for (uint32_t i = 0; i < V; i++) {
    e->mask_array[i] = 0;
    e->label_array[i] = i;
    e->inverse_label_array[i] = i;
  }
}

// readEdgeListsbin (edgeList.c:336-594): records of 8 bytes, or 12 when
// weighted (the weight is read in the WEIGHTED layout and skipped in the
// other).  The WEIGHTED layout always reads 12-byte records
// (edgeList.c:383-393) and, when `weighted` is 0, ignores the file's weight
// and draws one from MT19937 seeded 27491095 in edge order.  symmetric
// appends the reversed copy.
extern "C" struct EdgeList* readEdgeListsbin(const char* fname, uint8_t inverse, uint32_t symmetric,
                                             uint32_t weighted) {
  int fd = open(fname, O_RDONLY);
  if (fd == -1) err(1, "open: %s", fname);
  struct stat fs;
  if (fstat(fd, &fs) == -1) err(1, "stat: %s", fname);
  const size_t rec = (OGB200_WEIGHTED || weighted) ? 12 : 8;
  const uint32_t num_edges = (uint32_t)((uint64_t)fs.st_size / rec);
  const uint32_t total = symmetric ? num_edges * 2 : num_edges;
  EdgeList* e = newEdgeList(total);
  const uint32_t* buf = nullptr;
  if (fs.st_size > 0) {
    void* addr = mmap(nullptr, fs.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (addr == MAP_FAILED) {
      close(fd);
      err(1, "mmap: %s", fname);
    }
    buf = (const uint32_t*)addr;
  }
  const uint32_t stride = (uint32_t)(rec / 4);
#if OGB200_WEIGHTED
  mt19937state* mt = nullptr;
  if (!weighted) {
    mt = (mt19937state*)host_alloc(sizeof(mt19937state));
    initializeMersenneState(mt, 27491095);
  }
  float max_weight = 0;
#endif
  // parse in parallel (no weight draws), V = max id + 1
  const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<uint32_t> vmax(nt, 0);
  std::vector<std::thread> th;
  const uint32_t chunk = (num_edges + nt - 1) / std::max(1u, nt);
  for (unsigned t = 0; t < nt; t++) {
    th.emplace_back([&, t] {
      const uint64_t lo = (uint64_t)t * chunk, hi = std::min<uint64_t>(num_edges, lo + chunk);
      uint32_t m = 0;
      for (uint64_t i = lo; i < hi; i++) {
        uint32_t s = buf[stride * i + 0], d = buf[stride * i + 1];
        if (inverse) std::swap(s, d);
        e->edges_array_src[i] = s;
        e->edges_array_dest[i] = d;
        if (symmetric) {
          e->edges_array_src[i + num_edges] = d;
          e->edges_array_dest[i + num_edges] = s;
        }
        m = std::max(m, std::max(s, d));
#if OGB200_WEIGHTED
        if (weighted) {
          float wt;
          memcpy(&wt, &buf[stride * i + 2], 4);
          e->edges_array_weight[i] = wt;
          if (symmetric) e->edges_array_weight[i + num_edges] = wt;
        }
#endif
      }
      vmax[t] = m;
    });
  }
  for (auto& x : th) x.join();
  uint32_t num_vertices = 0;
  for (uint32_t m : vmax) num_vertices = std::max(num_vertices, m);
#if OGB200_WEIGHTED
  for (uint32_t i = 0; i < num_edges; i++) {
    if (!weighted) {
      e->edges_array_weight[i] = generateRandFloat(mt);
      if (symmetric) e->edges_array_weight[i + num_edges] = e->edges_array_weight[i];
    }
    max_weight = std::max(max_weight, e->edges_array_weight[i]);
  }
  e->max_weight = max_weight;
  free(mt);
#endif
  e->num_vertices = num_vertices + 1;
  e->avg_degree = e->num_edges / e->num_vertices;
  alloc_labels(e, e->num_vertices);
  if (buf) munmap((void*)buf, fs.st_size);
  close(fd);
  return e;
}

// readEdgeListsMem (edgeList.c:597-745): copy of the list, src/dst swapped
// when inverse; label arrays copied when present.
extern "C" struct EdgeList* readEdgeListsMem(struct EdgeList* m, uint8_t inverse, uint32_t symmetric,
                                             uint32_t weighted) {
  (void)symmetric;
  (void)weighted;
  const uint32_t E = m->num_edges, V = m->num_vertices;
  EdgeList* e = newEdgeList(E);
  auto copy_arr = [&](uint32_t* src) -> uint32_t* {
    if (!src) return nullptr;
    uint32_t* d = (uint32_t*)host_alloc((size_t)V * 4);
    memcpy(d, src, (size_t)V * 4);
    return d;
  };
  e->mask_array = copy_arr(m->mask_array);
  e->label_array = copy_arr(m->label_array);
  e->inverse_label_array = copy_arr(m->inverse_label_array);
  par_memcpy(inverse ? e->edges_array_src : e->edges_array_dest, m->edges_array_dest, (size_t)E * 4);
  par_memcpy(inverse ? e->edges_array_dest : e->edges_array_src, m->edges_array_src, (size_t)E * 4);
#if OGB200_WEIGHTED
  par_memcpy(e->edges_array_weight, m->edges_array_weight, (size_t)E * 4);
  e->max_weight = m->max_weight;
#endif
  e->num_vertices = V;
  if (V) e->avg_degree = E / V;
  return e;
}

// ---------------------------------------------------------------- sorting ---

// Sort the arrays of a host edge list on the device (in place).
// lex: by (src, dst); by_dst: by dst only.
static int sort_host_list(EdgeList* e, bool lex, bool by_dst) {
  const uint32_t E = e->num_edges;
  if (E == 0) return OK;
  cudaStream_t s = lib_stream();
  DevBuf in_s, in_d, in_w, out_s, out_d, out_w;
  SortWorkspace ws;
  const bool w =
#if OGB200_WEIGHTED
      e->edges_array_weight != nullptr;
#else
      false;
#endif
  OGB_TRY(in_s.alloc((size_t)E * 4));
  OGB_TRY(in_d.alloc((size_t)E * 4));
  OGB_TRY(out_s.alloc((size_t)E * 4));
  OGB_TRY(out_d.alloc((size_t)E * 4));
  if (w) {
    OGB_TRY(in_w.alloc((size_t)E * 4));
    OGB_TRY(out_w.alloc((size_t)E * 4));
  }
  OGB_TRY(h2d(in_s.p, e->edges_array_src, (size_t)E * 4, s));
  OGB_TRY(h2d(in_d.p, e->edges_array_dest, (size_t)E * 4, s));
#if OGB200_WEIGHTED
  if (w) OGB_TRY(h2d(in_w.p, e->edges_array_weight, (size_t)E * 4, s));
#endif
  KV in{in_s.as<uint32_t>(), in_d.as<uint32_t>(), w ? in_w.as<uint32_t>() : nullptr};
  KV out{out_s.as<uint32_t>(), out_d.as<uint32_t>(), w ? out_w.as<uint32_t>() : nullptr};
  if (by_dst) {
    KV in2{in.v0, in.k, in.v1}, out2{out.v0, out.k, out.v1};
    OGB_TRY(sort_pairs(in2, out2, E, ws, s));
  } else if (lex) {
    OGB_TRY(sort_pairs_lex(in, out, E, ws, s));
  } else {
    OGB_TRY(sort_pairs(in, out, E, ws, s));
  }
  OGB_TRY(sort_check(ws, s));
  OGB_TRY(d2h(e->edges_array_src, out_s.p, (size_t)E * 4, s));
  OGB_TRY(d2h(e->edges_array_dest, out_d.p, (size_t)E * 4, s));
#if OGB200_WEIGHTED
  if (w) OGB_TRY(d2h(e->edges_array_weight, out_w.p, (size_t)E * 4, s));
#endif
  return OK;
}

extern "C" struct EdgeList* radixSortEdgesBySource(struct EdgeList* e) {
  OGB_MUST(sort_host_list(e, false, false));
  return e;
}
extern "C" struct EdgeList* radixSortEdgesBySourceAndDestination(struct EdgeList* e) {
  OGB_MUST(sort_host_list(e, true, false));
  return e;
}
extern "C" struct EdgeList* countSortEdgesBySource(struct EdgeList* e) {
  OGB_MUST(sort_host_list(e, false, false));
  return e;
}
extern "C" struct EdgeList* countSortEdgesByDestination(struct EdgeList* e) {
  OGB_MUST(sort_host_list(e, false, true));
  return e;
}
extern "C" struct EdgeList* countSortEdgesBySourceAndDestination(struct EdgeList* e) {
  OGB_MUST(sort_host_list(e, true, false));
  return e;
}

// sortRunAlgorithms (sortRun.c:26-63).
extern "C" struct EdgeList* sortRunAlgorithms(struct EdgeList* e, uint32_t sort) {
  const double t0 = now_s();
  const char* msg;
  switch (sort) {
    case 1:
      e = radixSortEdgesBySourceAndDestination(e);
      msg = "Radix Sort Edges By Source/Dest (Seconds)";
      break;
    case 2:
      e = countSortEdgesBySource(e);
      msg = "Count Sort Edges By Source (Seconds)";
      break;
    case 3:
      e = countSortEdgesBySourceAndDestination(e);
      msg = "Count Sort Edges By Source/Dest (Seconds)";
      break;
    default:
      e = radixSortEdgesBySource(e);
      msg = "Radix Sort Edges By Source (Seconds)";
      break;
  }
  print_msg_time(msg, now_s() - t0);
  return e;
}

// removeDulpicatesSelfLoopEdges (edgeList.c:138-211) on the device: drop
// self loops, then drop every edge equal to the last kept one.  In the
// WEIGHTED layout the reference passes kept weights through a uint32
// temporary, i.e. truncates them to integers; that is reproduced.
int dedup_device(const uint32_t* s, const uint32_t* d, const uint32_t* w, uint32_t E, uint32_t* os, uint32_t* od,
                 uint32_t* ow, int truncate_weights, uint32_t* out_count, cudaStream_t st);

extern "C" struct EdgeList* removeDulpicatesSelfLoopEdges(struct EdgeList* e) {
  const uint32_t E = e->num_edges;
  cudaStream_t s = lib_stream();
  DevBuf a_s, a_d, a_w, b_s, b_d, b_w;
  const bool w =
#if OGB200_WEIGHTED
      e->edges_array_weight != nullptr;
#else
      false;
#endif
  OGB_MUST(a_s.alloc((size_t)E * 4 + 4));
  OGB_MUST(a_d.alloc((size_t)E * 4 + 4));
  OGB_MUST(b_s.alloc((size_t)E * 4 + 4));
  OGB_MUST(b_d.alloc((size_t)E * 4 + 4));
  if (w) {
    OGB_MUST(a_w.alloc((size_t)E * 4 + 4));
    OGB_MUST(b_w.alloc((size_t)E * 4 + 4));
  }
  OGB_MUST(h2d(a_s.p, e->edges_array_src, (size_t)E * 4, s));
  OGB_MUST(h2d(a_d.p, e->edges_array_dest, (size_t)E * 4, s));
#if OGB200_WEIGHTED
  if (w) OGB_MUST(h2d(a_w.p, e->edges_array_weight, (size_t)E * 4, s));
#endif
  uint32_t kept = 0;
  OGB_MUST(dedup_device(a_s.as<uint32_t>(), a_d.as<uint32_t>(), w ? a_w.as<uint32_t>() : nullptr, E,
                        b_s.as<uint32_t>(), b_d.as<uint32_t>(), w ? b_w.as<uint32_t>() : nullptr, 1, &kept, s));
  EdgeList* t = newEdgeList(E);
  OGB_MUST(d2h(t->edges_array_src, b_s.p, (size_t)kept * 4, s));
  OGB_MUST(d2h(t->edges_array_dest, b_d.p, (size_t)kept * 4, s));
#if OGB200_WEIGHTED
  if (w) OGB_MUST(d2h(t->edges_array_weight, b_w.p, (size_t)kept * 4, s));
  t->max_weight = e->max_weight;
#endif
  t->num_edges = kept;
  t->num_vertices = e->num_vertices;
  t->avg_degree = t->num_vertices ? t->num_edges / t->num_vertices : 0;
  const uint32_t V = e->num_vertices;
  t->mask_array = (uint32_t*)host_alloc((size_t)V * 4);
  t->label_array = (uint32_t*)host_alloc((size_t)V * 4);
  t->inverse_label_array = (uint32_t*)host_alloc((size_t)V * 4);
  memcpy(t->mask_array, e->mask_array, (size_t)V * 4);
  memcpy(t->label_array, e->label_array, (size_t)V * 4);
  memcpy(t->inverse_label_array, e->inverse_label_array, (size_t)V * 4);
  freeEdgeList(e);
  return t;
}

// -------------------------------------------------------------------- CSR ---

extern "C" struct Vertex* newVertexArray(uint32_t V) {
  Vertex* v = (Vertex*)host_alloc(sizeof(Vertex));
  v->out_degree = (uint32_t*)host_alloc((size_t)V * 4);
  v->in_degree = (uint32_t*)host_alloc((size_t)V * 4);
  v->edges_idx = (uint32_t*)host_alloc((size_t)V * 4);
  memset(v->out_degree, 0, (size_t)V * 4);
  memset(v->in_degree, 0, (size_t)V * 4);
  memset(v->edges_idx, 0, (size_t)V * 4);
  return v;
}

extern "C" void freeVertexArray(struct Vertex* v) {
  if (!v) return;
  free(v->edges_idx);
  free(v->out_degree);
  free(v->in_degree);
  free(v);
}

extern "C" struct GraphCSR* graphCSRNew(uint32_t V, uint32_t E, uint8_t inverse) {
  GraphCSR* g = (GraphCSR*)host_alloc(sizeof(GraphCSR));
  g->num_vertices = V;
  g->num_edges = E;
  g->avg_degree = V ? E / V : 0;
  g->sorted_edges_array = nullptr;
  g->inverse_sorted_edges_array = nullptr;
#if OGB200_WEIGHTED
  g->max_weight = 0;
#endif
  g->vertices = newVertexArray(V);
  g->inverse_vertices = inverse ? newVertexArray(V) : nullptr;
  return g;
}

// mapVerticesWithInOutDegree (vertex.c:204-325) on the device for one host
// direction: out_degree and edges_idx of that direction, in_degree of the
// other (when it exists).
extern "C" struct GraphCSR* mapVerticesWithInOutDegree(struct GraphCSR* graph, uint8_t inverse) {
  EdgeList* e = inverse ? graph->inverse_sorted_edges_array : graph->sorted_edges_array;
  Vertex* hv = inverse ? graph->inverse_vertices : graph->vertices;
  Vertex* other = inverse ? graph->vertices : graph->inverse_vertices;
  const uint32_t V = graph->num_vertices, E = graph->num_edges;
  cudaStream_t s = lib_stream();
  DevCSR c, o;
  DevBuf err;
  OGB_MUST(c.src.alloc((size_t)E * 4 + 4));
  OGB_MUST(c.out_degree.alloc((size_t)V * 4 + 4));
  OGB_MUST(c.edges_idx.alloc((size_t)V * 4 + 4));
  OGB_MUST(c.rows.alloc((size_t)V * 8 + 8));
  OGB_MUST(o.in_degree.alloc((size_t)V * 4 + 4));
  OGB_MUST(err.alloc(16));
  OGB_MUST(h2d(c.src.p, e->edges_array_src, (size_t)E * 4, s));
  if (cudaMemsetAsync(err.p, 0, 16, s) != cudaSuccess) die_status("memset", ERR_CUDA);
  OGB_MUST(csr_map(c, o, V, E, err.as<uint32_t>(), s));
  uint32_t h_err = 0;
  OGB_MUST(d2h(&h_err, err.p, 4, s));
  if (h_err) {
    fprintf(stderr, "ogb200: mapVerticesWithInOutDegree: a source id is >= num_vertices (%u)\n", V);
    exit(1);
  }
  OGB_MUST(d2h(hv->out_degree, c.out_degree.p, (size_t)V * 4, s));
  OGB_MUST(d2h(hv->edges_idx, c.edges_idx.p, (size_t)V * 4, s));
  if (other) OGB_MUST(d2h(other->in_degree, o.in_degree.p, (size_t)V * 4, s));
  return graph;
}

extern "C" struct GraphCSR* graphCSRAssignEdgeList(struct GraphCSR* graphCSR, struct EdgeList* edgeList,
                                                   uint8_t inverse) {
  if (inverse)
    graphCSR->inverse_sorted_edges_array = edgeList;
  else
    graphCSR->sorted_edges_array = edgeList;
#if OGB200_WEIGHTED
  graphCSR->max_weight = edgeList->max_weight;
#endif
  return mapVerticesWithInOutDegree(graphCSR, inverse);
}

static void print_max_degree(const Vertex* v, uint32_t V, bool in) {
  uint32_t best = 0, idx = 0;
  for (uint32_t i = 0; i < V; i++) {
    best = std::max(best, v->out_degree[i]);
    if (v->out_degree[i] == best) idx = i;
  }
  say(" -----------------------------------------------------\n");
  if (!in) {
    say("| %-15s | %-15s | %-15s | \n", "Node", "*max_out_degree", "in_degree");
    say(" -----------------------------------------------------\n");
    say("| %-15u | %-15u | %-15u | \n", idx, V ? v->out_degree[idx] : 0, V ? v->in_degree[idx] : 0);
  } else {
    say("| %-15s | %-15s | %-15s | \n", "Node", "out_degree", "*max_in_degree");
    say(" -----------------------------------------------------\n");
    say("| %-15u | %-15u | %-15u | \n", idx, V ? v->in_degree[idx] : 0, V ? v->out_degree[idx] : 0);
  }
  say(" -----------------------------------------------------\n");
}

// graphCSRPrint (graphCSR.c:66-104).
extern "C" void graphCSRPrint(struct GraphCSR* g) {
  if (quiet()) return;
  say(" -----------------------------------------------------\n");
  say("| %-51s | \n", "GraphCSR Properties");
  say(" -----------------------------------------------------\n");
#if OGB200_WEIGHTED
  say("| %-51s | \n", "WEIGHTED");
  say("| %-51s | \n", "MAX WEIGHT");
  say("| %-51f | \n", g->max_weight);
#else
  say("| %-51s | \n", "UN-WEIGHTED");
#endif
  say("| %-51s | \n", "DIRECTED");
  say(" -----------------------------------------------------\n");
  say("| %-51s | \n", "Average Degree (D)");
  say("| %-51u | \n", g->avg_degree);
  say(" -----------------------------------------------------\n");
  say("| %-51s | \n", "Number of Vertices (V)");
  say("| %-51u | \n", g->num_vertices);
  say(" -----------------------------------------------------\n");
  say("| %-51s | \n", "Number of Edges (E)");
  say("| %-51u | \n", g->num_edges);
  say(" -----------------------------------------------------\n");
  print_max_degree(g->vertices, g->num_vertices, false);
  if (g->inverse_vertices) print_max_degree(g->inverse_vertices, g->num_vertices, true);
}

// Reorder/mask stages of the reference (reorder.c) are outside this
// library; in a link with the reference objects their definitions are used.
extern "C" struct EdgeList* reorderGraphProcess(struct EdgeList*, struct Arguments*) __attribute__((weak));
extern "C" struct EdgeList* maskGraphProcess(struct EdgeList*, struct Arguments*) __attribute__((weak));

// Download the device CSR into freshly allocated host structs.
static int download_graph(DevGraph& g, GraphCSR* h, EdgeList* fwd_list, EdgeList* inv_list, cudaStream_t s) {
  const uint32_t V = g.V, E = g.E;
  for (int dir = 0; dir < 2; dir++) {
    DevCSR& c = dir ? g.inv : g.fwd;
    EdgeList* e = dir ? inv_list : fwd_list;
    Vertex* v = dir ? h->inverse_vertices : h->vertices;
    OGB_TRY(d2h(e->edges_array_src, c.src.p, (size_t)E * 4, s));
    OGB_TRY(d2h(e->edges_array_dest, c.dst.p, (size_t)E * 4, s));
#if OGB200_WEIGHTED
    if (g.weighted) OGB_TRY(d2h(e->edges_array_weight, c.w.p, (size_t)E * 4, s));
#endif
    OGB_TRY(d2h(v->out_degree, c.out_degree.p, (size_t)V * 4, s));
    OGB_TRY(d2h(v->in_degree, c.in_degree.p, (size_t)V * 4, s));
    OGB_TRY(d2h(v->edges_idx, c.edges_idx.p, (size_t)V * 4, s));
  }
  return OK;
}

// graphCSRPreProcessingStep (graphCSR.c:164-248): read, sort, [dedup],
// [reorder/mask through the reference], CSR both directions.  The whole
// build runs on the device from one upload; the host struct receives the
// results, and the device copy stays for the algorithms.
extern "C" struct GraphCSR* graphCSRPreProcessingStep(struct Arguments* arguments) {
  double t0 = now_s();
  EdgeList* edges = readEdgeListsbin(arguments->fnameb, 0, arguments->symmetric, arguments->weighted);
  print_msg_time("Read Edge List From File (Seconds)", now_s() - t0);

  const bool host_stages = arguments->lmode || arguments->lmode_l2 || arguments->lmode_l3 || arguments->mmode;
  if (host_stages) {
    // Relabelling stages need the reference's reorder code on host lists.
    if (!reorderGraphProcess || !maskGraphProcess) {
      fprintf(stderr, "ogb200: reorder/mask modes (-l/-L/-O/-M) need the reference's reorder.c in the link\n");
      exit(1);
    }
    edges = sortRunAlgorithms(edges, arguments->sort);
    if (arguments->dflag) {
      t0 = now_s();
      edges = removeDulpicatesSelfLoopEdges(edges);
      print_msg_time("Removing duplicate edges (Seconds)", now_s() - t0);
    }
    uint32_t modes[3] = {arguments->lmode, arguments->lmode_l2, arguments->lmode_l3};
    for (int i = 0; i < 3; i++) {
      arguments->lmode = modes[i];
      if (arguments->lmode) {
        edges = reorderGraphProcess(edges, arguments);
        edges = sortRunAlgorithms(edges, arguments->sort);
      }
    }
    if (arguments->mmode) edges = maskGraphProcess(edges, arguments);
  }

  cudaStream_t s = lib_stream();
  ogb_graph* dg = new ogb_graph();
  DevGraph& g = dg->g;
  uint32_t E = edges->num_edges;
  const uint32_t V = edges->num_vertices;
#if OGB200_WEIGHTED
  const bool w = edges->edges_array_weight != nullptr;
#else
  const bool w = false;
#endif
  OGB_MUST(g.input_src.alloc((size_t)E * 4 + 4));
  OGB_MUST(g.input_dst.alloc((size_t)E * 4 + 4));
  if (w) OGB_MUST(g.input_w.alloc((size_t)E * 4 + 4));
  OGB_MUST(h2d(g.input_src.p, edges->edges_array_src, (size_t)E * 4, s));
  OGB_MUST(h2d(g.input_dst.p, edges->edges_array_dest, (size_t)E * 4, s));
#if OGB200_WEIGHTED
  if (w) OGB_MUST(h2d(g.input_w.p, edges->edges_array_weight, (size_t)E * 4, s));
#endif
  const float* in_w = w ? g.input_w.as<float>() : nullptr;

  if (!host_stages && arguments->dflag) {
    // sort, dedup on the device, then the CSR build re-sorts (a no-op order)
    t0 = now_s();
    KV in{g.input_src.as<uint32_t>(), g.input_dst.as<uint32_t>(), w ? g.input_w.as<uint32_t>() : nullptr};
    DevBuf ss, sd, sw;
    OGB_MUST(ss.alloc((size_t)E * 4 + 4));
    OGB_MUST(sd.alloc((size_t)E * 4 + 4));
    if (w) OGB_MUST(sw.alloc((size_t)E * 4 + 4));
    KV out{ss.as<uint32_t>(), sd.as<uint32_t>(), w ? sw.as<uint32_t>() : nullptr};
    const bool lex = arguments->sort == 1 || arguments->sort == 3;
    OGB_MUST(lex ? sort_pairs_lex(in, out, E, g.sort_ws, s) : sort_pairs(in, out, E, g.sort_ws, s));
    OGB_MUST(sort_check(g.sort_ws, s));
    print_msg_time("Radix Sort Edges By Source (Seconds)", now_s() - t0);
    t0 = now_s();
    uint32_t kept = 0;
    OGB_MUST(dedup_device(out.k, out.v0, out.v1, E, in.k, in.v0, in.v1, 1, &kept, s));
    print_msg_time("Removing duplicate edges (Seconds)", now_s() - t0);
    E = kept;
    // host list mirrors the deduplicated sorted list
    edges->num_edges = E;
    edges->avg_degree = V ? E / V : 0;
  }

  t0 = now_s();
  OGB_MUST(graph_build(g, g.input_src.as<uint32_t>(), g.input_dst.as<uint32_t>(), in_w, E, V, arguments->sort, s));
  OGB_MUST(graph_check(g, s));
  const double t_build = now_s() - t0;
  g.input_src.release();
  g.input_dst.release();
  g.input_w.release();

  GraphCSR* h = graphCSRNew(V, E, 1);
  EdgeList* inv = newEdgeList(E);
  inv->num_vertices = V;
  inv->avg_degree = V ? E / V : 0;
  auto copy_arr = [&](uint32_t* src) -> uint32_t* {
    if (!src) return nullptr;
    uint32_t* d = (uint32_t*)host_alloc((size_t)V * 4);
    memcpy(d, src, (size_t)V * 4);
    return d;
  };
  inv->mask_array = copy_arr(edges->mask_array);
  inv->label_array = copy_arr(edges->label_array);
  inv->inverse_label_array = copy_arr(edges->inverse_label_array);
#if OGB200_WEIGHTED
  inv->max_weight = edges->max_weight;
  h->max_weight = edges->max_weight;
  if (!w) {
    free(inv->edges_array_weight);
    inv->edges_array_weight = nullptr;
  }
#endif
  t0 = now_s();
  OGB_MUST(download_graph(g, h, edges, inv, s));
  h->sorted_edges_array = edges;
  h->inverse_sorted_edges_array = inv;
  print_msg_time("Radix Sort + CSR both directions on GPU (Seconds)", t_build);
  print_msg_time("Copy GraphCSR to host (Seconds)", now_s() - t0);
  // the device copy no longer needs the sorted src arrays
  mirror_set(h, dg);
  graphCSRPrint(h);
  return h;
}

// graphCSRVertexLabelRemappingDualOrder (graphCSR.c:337-377): each edge
// list's inverse-label array maps its vertex ids to the other list's.
extern "C" void graphCSRVertexLabelRemappingDualOrder(struct GraphCSR* graphCSR) {
  const uint32_t V = graphCSR->num_vertices;
  EdgeList* el = graphCSR->sorted_edges_array;
  EdgeList* iel = graphCSR->inverse_sorted_edges_array ? graphCSR->inverse_sorted_edges_array : el;
  const uint32_t *lab_el = el->label_array, *lab_iel = iel->label_array;
  uint32_t *inv_el = el->inverse_label_array, *inv_iel = iel->inverse_label_array;
  if (!lab_el || !lab_iel || !inv_el || !inv_iel) return;  // lists without labels: nothing to map
  for (uint32_t v = 0; v < V; v++) inv_el[lab_el[v]] = lab_iel[v];
  if (graphCSR->inverse_sorted_edges_array)
    for (uint32_t v = 0; v < V; v++) inv_iel[lab_iel[v]] = lab_el[v];
}

// graphCSRPreProcessingStepDualOrder (graphCSR.c:250-335): without
// reordering the same graph as graphCSRPreProcessingStep, then the label
// remapping.  The reordering stages give the two directions different
// vertex orders, which the DualOrder searches here do not provide.
extern "C" struct GraphCSR* graphCSRPreProcessingStepDualOrder(struct Arguments* arguments) {
  if (arguments->lmode || arguments->lmode_l2 || arguments->lmode_l3 || arguments->mmode) {
    fprintf(stderr, "ogb200: DualOrder preprocessing with reordering (-l/-L/-O/-M) is not provided\n");
    exit(1);
  }
  GraphCSR* g = graphCSRPreProcessingStep(arguments);
  graphCSRVertexLabelRemappingDualOrder(g);
  return g;
}

// ---- .csr binary file (graphCSR.c:380-558) ----------------------------------
// Layout, native (little-endian) order: u32 num_edges, u32 num_vertices,
// [f32 max_weight in the WEIGHTED layout]; then per vertex the forward
// out_degree, in_degree, edges_idx and, when the graph has an inverse CSR,
// the inverse's three; then per edge the forward src, dst[, weight] and the
// inverse's src, dst[, weight].  The reference moves it one value per
// fread/fwrite; here host threads encode / decode whole chunks.

namespace {
constexpr uint32_t kCsrW = OGB200_WEIGHTED ? 1u : 0u;  // weight words per edge record
constexpr size_t kCsrChunk = size_t(1) << 20;           // records per chunk

inline uint32_t fbits(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  return u;
}
inline float bitsf(uint32_t u) {
  float x;
  memcpy(&x, &u, 4);
  return x;
}
}  // namespace

// writeToBinFileGraphCSR (graphCSR.c:380-437): the file is fname + ".csr".
extern "C" void writeToBinFileGraphCSR(const char* fname, struct GraphCSR* g) {
  std::string path = std::string(fname) + ".csr";
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) err(1, "open: %s", path.c_str());
  const uint32_t V = g->num_vertices, E = g->num_edges;
  const bool inv = g->inverse_vertices != nullptr;
  uint32_t head[3] = {E, V, 0};
#if OGB200_WEIGHTED
  head[2] = fbits(g->max_weight);
#endif
  fwrite(head, 4, 2 + kCsrW, f);
  const size_t vw = inv ? 6 : 3, ew = (2 + kCsrW) * (inv ? 2 : 1);
  std::vector<uint32_t> buf(kCsrChunk * std::max(vw, ew));
  const Vertex *fv = g->vertices, *iv = g->inverse_vertices;
  for (size_t v0 = 0; v0 < V; v0 += kCsrChunk) {
    const size_t n = std::min<size_t>(kCsrChunk, V - v0);
    host_par_for(n, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++) {
        uint32_t* r = &buf[i * vw];
        const size_t v = v0 + i;
        r[0] = fv->out_degree[v];
        r[1] = fv->in_degree[v];
        r[2] = fv->edges_idx[v];
        if (inv) {
          r[3] = iv->out_degree[v];
          r[4] = iv->in_degree[v];
          r[5] = iv->edges_idx[v];
        }
      }
    });
    fwrite(buf.data(), 4 * vw, n, f);
  }
  const EdgeList *fe = g->sorted_edges_array, *ie = g->inverse_sorted_edges_array;
  for (size_t e0 = 0; e0 < E; e0 += kCsrChunk) {
    const size_t n = std::min<size_t>(kCsrChunk, E - e0);
    host_par_for(n, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; i++) {
        uint32_t* r = &buf[i * ew];
        const size_t e = e0 + i;
        size_t k = 0;
        r[k++] = fe->edges_array_src[e];
        r[k++] = fe->edges_array_dest[e];
#if OGB200_WEIGHTED
        r[k++] = fbits(fe->edges_array_weight[e]);
#endif
        if (inv) {
          r[k++] = ie->edges_array_src[e];
          r[k++] = ie->edges_array_dest[e];
#if OGB200_WEIGHTED
          r[k++] = fbits(ie->edges_array_weight[e]);
#endif
        }
      }
    });
    fwrite(buf.data(), 4 * ew, n, f);
  }
  fclose(f);
}

namespace {
// Decode the edge records [e0, e0 + n) into the host lists and, when stage is
// given, the dst (and weight) words of both directions into the pinned
// stage laid out as [fwd dst | inv dst | fwd w | inv w] of n words each.
void csr_decode_edges(const uint32_t* rec, size_t ew, bool inv, size_t e0, size_t n, EdgeList* fe, EdgeList* ie,
                      uint32_t* stage) {
  host_par_for(n, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; i++) {
      const uint32_t* r = rec + (e0 + i) * ew;
      const size_t e = e0 + i;
      size_t k = 0;
      fe->edges_array_src[e] = r[k++];
      fe->edges_array_dest[e] = r[k++];
#if OGB200_WEIGHTED
      fe->edges_array_weight[e] = bitsf(r[k++]);
#endif
      if (inv) {
        ie->edges_array_src[e] = r[k++];
        ie->edges_array_dest[e] = r[k++];
#if OGB200_WEIGHTED
        ie->edges_array_weight[e] = bitsf(r[k++]);
#endif
      }
      if (stage) {
        stage[i] = fe->edges_array_dest[e];
        if (inv) stage[n + i] = ie->edges_array_dest[e];
#if OGB200_WEIGHTED
        stage[2 * n + i] = fbits(fe->edges_array_weight[e]);
        if (inv) stage[3 * n + i] = fbits(ie->edges_array_weight[e]);
#endif
      }
    }
  });
}
}  // namespace

// readFromBinFileGraphCSR (graphCSR.c:439-558).  The file is mapped and
// decoded by host threads; when a GPU is present the device copy the
// algorithms use is built on the way: the edge section is decoded chunk by
// chunk into pinned double buffers whose copies to the device run while the
// next chunk decodes.  The label arrays stay NULL, as in the reference.  A
// short file leaves the missing values at zero (the reference's fread does
// the same).
extern "C" struct GraphCSR* readFromBinFileGraphCSR(const char* fname) {
  const int fd = open(fname, O_RDONLY);
  if (fd < 0) err(1, "open: %s", fname);
  struct stat sb;
  if (fstat(fd, &sb) != 0) err(1, "open: %s", fname);
  const size_t bytes = (size_t)sb.st_size;
  const uint32_t* map = nullptr;
  if (bytes) {
    void* p = mmap(nullptr, bytes, PROT_READ, MAP_PRIVATE, fd, 0);
    if (p == MAP_FAILED) err(1, "open: %s", fname);
    map = static_cast<const uint32_t*>(p);
  }
  const size_t words = bytes / 4;
  const size_t hw = 2 + kCsrW;
  const uint32_t E = words > 0 ? map[0] : 0, V = words > 1 ? map[1] : 0;
  GraphCSR* h = graphCSRNew(V, E, 1);
  EdgeList* fe = newEdgeList(E);
  EdgeList* ie = newEdgeList(E);
  fe->num_vertices = ie->num_vertices = V;
#if OGB200_WEIGHTED
  const float mw = words > 2 ? bitsf(map[2]) : 0.0f;
  h->max_weight = fe->max_weight = ie->max_weight = mw;
#endif
  h->sorted_edges_array = fe;
  h->inverse_sorted_edges_array = ie;
  const bool inv = true;  // graphCSRNew(.., 1): the reference reads both directions
  const size_t vw = 6, ew = (2 + kCsrW) * 2;
  // vertices (a short file leaves zeros)
  const size_t vavail = words > hw ? std::min<size_t>(V, (words - hw) / vw) : 0;
  const uint32_t* vrec = map ? map + hw : nullptr;
  host_par_for(vavail, [&](size_t lo, size_t hi) {
    for (size_t v = lo; v < hi; v++) {
      const uint32_t* r = vrec + v * vw;
      h->vertices->out_degree[v] = r[0];
      h->vertices->in_degree[v] = r[1];
      h->vertices->edges_idx[v] = r[2];
      h->inverse_vertices->out_degree[v] = r[3];
      h->inverse_vertices->in_degree[v] = r[4];
      h->inverse_vertices->edges_idx[v] = r[5];
    }
  });
  const size_t ebase = hw + (size_t)V * vw;
  const size_t eavail = words > ebase ? std::min<size_t>(E, (words - ebase) / ew) : 0;
  const uint32_t* erec = map ? map + ebase : nullptr;
  int ndev = 0;
  const bool gpu = cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0 && V > 0;
  if (!gpu) {
    cudaGetLastError();  // clear the no-device error
    for (size_t e0 = 0; e0 < eavail; e0 += kCsrChunk)
      csr_decode_edges(erec, ew, inv, e0, std::min(kCsrChunk, eavail - e0), fe, ie, nullptr);
  } else {
    cudaStream_t s = lib_stream();
    ogb_graph* dg = new ogb_graph();
    DevGraph& g = dg->g;
    g.V = V;
    g.E = E;
    g.weighted = kCsrW != 0;
    g.build_id++;
    for (int dir = 0; dir < 2; dir++) {
      DevCSR& c = dir ? g.inv : g.fwd;
      const Vertex* hv = dir ? h->inverse_vertices : h->vertices;
      OGB_MUST(c.dst.alloc((size_t)E * 4 + 4));
      if (kCsrW) OGB_MUST(c.w.alloc((size_t)E * 4 + 4));
      OGB_MUST(c.out_degree.alloc((size_t)V * 4 + 4));
      OGB_MUST(c.in_degree.alloc((size_t)V * 4 + 4));
      OGB_MUST(c.edges_idx.alloc((size_t)V * 4 + 4));
      OGB_MUST(c.rows.alloc((size_t)V * 8 + 8));
      OGB_MUST(h2d(c.out_degree.p, hv->out_degree, (size_t)V * 4, s));
      OGB_MUST(h2d(c.in_degree.p, hv->in_degree, (size_t)V * 4, s));
      OGB_MUST(h2d(c.edges_idx.p, hv->edges_idx, (size_t)V * 4, s));
      OGB_MUST(csr_pack_rows(c, V, s));
    }
    // the device arrays past the file's end stay as the host's: zeros
    if (eavail < E) {
      for (DevCSR* c : {&g.fwd, &g.inv}) {
        OGB_CUDA_MUST(cudaMemsetAsync(c->dst.as<uint32_t>() + eavail, 0, (size_t)(E - eavail) * 4, s));
        if (kCsrW) OGB_CUDA_MUST(cudaMemsetAsync(c->w.as<uint32_t>() + eavail, 0, (size_t)(E - eavail) * 4, s));
      }
    }
    const size_t per = 2 * (1 + kCsrW);  // staged words per edge
    uint32_t* stage[2] = {nullptr, nullptr};
    cudaEvent_t ev[2];
    for (int k = 0; k < 2; k++) {
      OGB_CUDA_MUST(cudaMallocHost(&stage[k], kCsrChunk * per * 4));
      OGB_CUDA_MUST(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
    }
    size_t chunk = 0;
    for (size_t e0 = 0; e0 < eavail; e0 += kCsrChunk, chunk++) {
      const int k = (int)(chunk & 1);
      const size_t n = std::min(kCsrChunk, eavail - e0);
      OGB_CUDA_MUST(cudaEventSynchronize(ev[k]));  // this buffer's previous copies are done
      csr_decode_edges(erec, ew, inv, e0, n, fe, ie, stage[k]);
      const size_t nb = n * 4;
      OGB_CUDA_MUST(cudaMemcpyAsync(g.fwd.dst.as<uint32_t>() + e0, stage[k], nb, cudaMemcpyHostToDevice, s));
      OGB_CUDA_MUST(cudaMemcpyAsync(g.inv.dst.as<uint32_t>() + e0, stage[k] + n, nb, cudaMemcpyHostToDevice, s));
      if (kCsrW) {
        OGB_CUDA_MUST(cudaMemcpyAsync(g.fwd.w.as<uint32_t>() + e0, stage[k] + 2 * n, nb, cudaMemcpyHostToDevice, s));
        OGB_CUDA_MUST(cudaMemcpyAsync(g.inv.w.as<uint32_t>() + e0, stage[k] + 3 * n, nb, cudaMemcpyHostToDevice, s));
      }
      OGB_CUDA_MUST(cudaEventRecord(ev[k], s));
    }
    OGB_CUDA_MUST(cudaStreamSynchronize(s));
    for (int k = 0; k < 2; k++) {
      cudaFreeHost(stage[k]);
      cudaEventDestroy(ev[k]);
    }
    mirror_set(h, dg);
  }
  if (map) munmap(const_cast<uint32_t*>(map), bytes);
  close(fd);
  graphCSRPrint(h);
  return h;
}

extern "C" void graphCSRFree(struct GraphCSR* g) {
  if (!g) return;
  mirror_drop(g);
  freeVertexArray(g->vertices);
  freeEdgeList(g->sorted_edges_array);
  freeVertexArray(g->inverse_vertices);
  freeEdgeList(g->inverse_sorted_edges_array);
  free(g);
}

// -------------------------------------------------------------------- BFS ---


// BFSStats with its four arrays allocated but not initialized.
static BFSStats* bfs_stats_alloc(uint32_t V) {
  BFSStats* st = (BFSStats*)host_alloc(sizeof(BFSStats));
  st->distances = (uint32_t*)pool_alloc((size_t)V * 4);
  st->distances_DualOrder = (uint32_t*)pool_alloc((size_t)V * 4);
  st->parents = (int*)pool_alloc((size_t)V * 4);
  st->parents_DualOrder = (int*)pool_alloc((size_t)V * 4);
  st->processed_nodes = 0;
  st->iteration = 0;
  st->num_vertices = V;
  st->time_total = 0.0;
  return st;
}

// newBFSStatsGraphCSR (BFS.c:42-78): distances 0, parents (and the DualOrder
// copy) -out_degree or -1; the reference's parallel loop, on host threads.
extern "C" struct BFSStats* newBFSStatsGraphCSR(struct GraphCSR* graph) {
  const uint32_t V = graph->num_vertices;
  BFSStats* st = bfs_stats_alloc(V);
  const uint32_t* od = graph->vertices->out_degree;
  host_par_for(V, [&](size_t lo, size_t hi) {
    for (size_t v = lo; v < hi; v++) {
      st->distances[v] = 0;
      const uint32_t d = od[v];
      st->parents[v] = d ? -(int)d : -1;
      st->parents_DualOrder[v] = st->parents[v];
    }
  });
  return st;
}

extern "C" void freeBFSStats(struct BFSStats* st) {
  if (!st) return;
  const size_t n = (size_t)st->num_vertices * 4;
  pool_free(st->distances, n);
  pool_free(st->parents, n);
  pool_free(st->distances_DualOrder, n);
  pool_free(st->parents_DualOrder, n);
  free(st);
}

static BfsResult g_last_bfs;  // level trace of the last drop-in BFS

// Wall-clock phases of the last drop-in BFS call, in seconds (see
// ogb_dropin_bfs_phases in ogb200_device.h).
static double g_bfs_phase[OGB_DROPIN_BFS_PHASES];

// 32 consecutive int32 values to 128-byte-aligned memory with non-temporal
// 16-byte stores: the result arrays are written whole and not read again by
// this call, so bypassing the cache saves the read-for-ownership of every
// line (half of the memory traffic of an ordinary store).
static inline void stream32(void* dst, const int32_t* src) {
  __m128i* d = reinterpret_cast<__m128i*>(dst);
  const __m128i* q = reinterpret_cast<const __m128i*>(src);
#pragma unroll
  for (int i = 0; i < 8; i++) _mm_stream_si128(d + i, _mm_loadu_si128(q + i));
}

// Pinned staging of BFS results (one per process, grows).
namespace {
struct ResultStage {
  static constexpr int kEv = 17;  // one for the depths, the rest for parent chunks
  std::mutex mu;
  unsigned char* h = nullptr;
  size_t bytes = 0;
  cudaEvent_t ev[kEv] = {};
  int reserve(size_t n) {
    if (!ev[0])
      for (auto& e : ev) OGB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (n <= bytes) return OK;
    if (h) cudaFreeHost(h);
    h = nullptr;
    bytes = 0;
    OGB_CUDA(cudaMallocHost(&h, n));
    bytes = n;
    return OK;
  }
};
ResultStage& result_stage() {
  static ResultStage p;
  return p;
}
}  // namespace

// The result of a search into the reference's host arrays.  The device
// arrays already hold the reference's values (parents: the tree, with the
// -out_degree / -1 sentinels of unreached vertices; depth 0 for those), so
// the host only copies.  Depths travel as one byte per vertex when the search
// has fewer than 255 levels (V bytes instead of 4V on the host link) and are
// widened by the host threads while the parents, copied whole in chunks, are
// still on the link; each chunk is copied out by all threads as it lands.
// The chunks halve in size (1/2, 1/4, 1/8, 1/8 of the vertices): every copy
// costs link time of its own (16 equal chunks took 0.10 ms more than one
// copy of 16.8 MB), and only the last chunk's copy-out is left after the
// link is done.
constexpr size_t kParentChunks = 4;  // <= ResultStage::kEv - 1
static int bfs_result_to_host(ogb_graph* dg, uint32_t V, uint32_t levels, int* parents, uint32_t* dist,
                              cudaStream_t s) {
  if (levels >= 255) {  // depths do not fit a byte: plain copies
    OGB_TRY(d2h(parents, dg->d_parents.p, (size_t)V * 4, s));
    OGB_TRY(d2h(dist, dg->d_distances.p, (size_t)V * 4, s));
    return OK;
  }
  const size_t d8_bytes = ((size_t)V + 3) / 4 * 4;
  OGB_TRY(dg->d_depth8.alloc(d8_bytes));
  OGB_TRY(bfs_depth_bytes(V, dg->d_distances.as<uint32_t>(), dg->d_depth8.as<uint8_t>(), s));
  ResultStage& rs = result_stage();
  std::lock_guard<std::mutex> lk(rs.mu);
  OGB_TRY(rs.reserve(d8_bytes + (size_t)V * 4));
  const unsigned char* h8 = rs.h;
  int32_t* hp = reinterpret_cast<int32_t*>(rs.h + d8_bytes);
  const int32_t* dp = dg->d_parents.as<int32_t>();
  OGB_CUDA(cudaMemcpyAsync(rs.h, dg->d_depth8.p, d8_bytes, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaEventRecord(rs.ev[0], s));
  // parent chunks of 1/2, 1/4, ... of the vertices, the last two equal: few
  // copies (each costs a few microseconds of link time), and the host's
  // copy-out of every chunk but the last hides under the next chunk's copy
  size_t cbeg[ResultStage::kEv], cend[ResultStage::kEv];
  size_t nchunks = 0;
  for (size_t lo = 0; lo < V && nchunks < kParentChunks;) {
    const size_t left = (size_t)V - lo;
    const size_t n = nchunks + 1 == kParentChunks ? left : std::max<size_t>(1, std::min(left, (left + 1) / 2));
    OGB_CUDA(cudaMemcpyAsync(hp + lo, dp + lo, n * 4, cudaMemcpyDeviceToHost, s));
    OGB_CUDA(cudaEventRecord(rs.ev[1 + nchunks], s));
    cbeg[nchunks] = lo;
    cend[nchunks] = lo + n;
    lo += n;
    nchunks++;
  }
  int failed = 0;
#pragma omp parallel num_threads(host_threads()) reduction(| : failed)
  {
    const size_t tid = (size_t)omp_get_thread_num(), nth = (size_t)omp_get_num_threads();
    if (cudaEventSynchronize(rs.ev[0]) != cudaSuccess) failed = 1;
    const size_t lo = (size_t)V * tid / nth, hi = (size_t)V * (tid + 1) / nth;
    for (size_t v = lo; v < hi; v++) dist[v] = h8[v];
    for (size_t c = 0; c < nchunks; c++) {
      if (cudaEventSynchronize(rs.ev[1 + c]) != cudaSuccess) failed = 1;
      const size_t clo = cbeg[c], cn = cend[c] - cbeg[c];
      const size_t a = clo + cn * tid / nth, b = clo + cn * (tid + 1) / nth;
      if (b > a) memcpy(parents + a, hp + a, (b - a) * 4);
    }
  }
  if (failed) return fail(ERR_CUDA, "bfs result copy: %s", cudaGetErrorString(cudaGetLastError()));
  return OK;
}

static struct BFSStats* bfs_dropin(struct Arguments* a, struct GraphCSR* graph, uint32_t mode, const char* title,
                                   bool bitmap_nf, bool want_trace = false) {
  const uint32_t V = graph->num_vertices;
  // The reference checks source > V (BFS.c:482); source == V would index
  // past the label array there, so it is rejected here too.
  if (a->source < 0 || (uint32_t)a->source >= V) {
    BFSStats* st0 = newBFSStatsGraphCSR(graph);
    say(" -----------------------------------------------------\n");
    say("| %-51s | \n", "ERROR!! CHECK SOURCE RANGE");
    say(" -----------------------------------------------------\n");
    return st0;
  }
  // parents, distances and the DualOrder parent copy (its initial sentinels,
  // BFS.c:64-73) are written whole from the device result.
  const double t_call = now_s();
  BFSStats* st = bfs_stats_alloc(V);
  const uint32_t* od = graph->vertices->out_degree;
  const uint32_t* labels = graph->sorted_edges_array ? graph->sorted_edges_array->label_array : nullptr;
  a->source = labels ? (int)labels[a->source] : a->source;
  say(" -----------------------------------------------------\n");
  say("| %-51s | \n", title);
  say(" -----------------------------------------------------\n");
  say("| %-51u | \n", (uint32_t)a->source);
  say(" -----------------------------------------------------\n");
  say("| %-15s | %-15s | %-15s | \n", "Iteration", "Nodes", "Time (Seconds)");
  say(" -----------------------------------------------------\n");
  int status = OK;
  ogb_graph* dg = mirror_of(graph, &status);
  if (!dg) die_status("device copy of GraphCSR", status);
  cudaStream_t s = lib_stream();
  // device result arrays live with the device copy (no per-call cudaMalloc)
  OGB_MUST(dg->d_parents.alloc((size_t)V * 4 + 4));
  OGB_MUST(dg->d_distances.alloc((size_t)V * 4 + 4));
  BfsResult& r = g_last_bfs;
  const double t0 = now_s();
  g_bfs_phase[1] = t0 - t_call;
  // The DualOrder parent copy keeps its initial sentinels (BFS.c:64-73): the
  // other host threads write them (streamed, 32 vertices at a time, ranges
  // split on 32-vertex boundaries) while thread 0 runs the device search.
  int run_status = OK;
  int* dual = st->parents_DualOrder;
  double t_search = 0.0, t_dual = 0.0;
#pragma omp parallel num_threads(host_threads())
  {
    const int tid = omp_get_thread_num(), nth = omp_get_num_threads();
    if (tid == 0) {
      // (the reference's stats need no reached-vertex count)
      run_status = bfs_run(dg->g, (uint32_t)a->source, mode, dg->d_parents.as<int32_t>(),
                           dg->d_distances.as<uint32_t>(), &r, want_trace || !quiet(), bitmap_nf, s, false);
      t_search = now_s() - t0;
    }
    if (tid > 0 || nth == 1) {
      const size_t parts = nth > 1 ? (size_t)(nth - 1) : 1, me = nth > 1 ? (size_t)(tid - 1) : 0;
      const size_t words = ((size_t)V + 31) / 32;
      const size_t lo = std::min<size_t>(V, words * me / parts * 32), hi = std::min<size_t>(V, words * (me + 1) / parts * 32);
      alignas(16) int32_t buf[32];
      size_t v = lo;
      for (; v + 32 <= hi; v += 32) {
        for (int i = 0; i < 32; i++) buf[i] = od[v + i] ? -(int)od[v + i] : -1;
        stream32(dual + v, buf);
      }
      for (; v < hi; v++) dual[v] = od[v] ? -(int)od[v] : -1;
      _mm_sfence();
      if (tid == 1 || nth == 1) t_dual = now_s() - t0;
    }
  }
  OGB_MUST(run_status);
  const double t_trav = now_s() - t0;
  g_bfs_phase[2] = t_search;
  g_bfs_phase[3] = t_dual;
  g_bfs_phase[4] = t_trav;
  const double t1 = now_s();
  OGB_MUST(bfs_result_to_host(dg, V, (uint32_t)r.nlevels, st->parents, st->distances, s));
  g_bfs_phase[5] = now_s() - t1;
  g_bfs_phase[0] = now_s() - t_call;
  st->processed_nodes = r.processed_nodes;
  st->iteration = r.iteration;
  st->time_total = t_trav;
  if (!quiet()) {
    say("| %s %-12u | %-15u | %-15f | \n", mode == BFS_PULL ? "BU" : "TD", 0u, 1u, 0.0);
    for (size_t i = 0; i < r.levels.size(); i++) {
      const BfsLevel& L = r.levels[i];
      say("| %s %-12u | %-15u | %-15f | \n", L.direction ? "BU" : "TD", (uint32_t)(i + 1), L.discovered,
          L.ms / 1000.0);
    }
    say(" -----------------------------------------------------\n");
    say("| %-15s | %-15u | %-15f | \n", "No OverHead", st->processed_nodes, r.ms / 1000.0);
    say(" -----------------------------------------------------\n");
    say(" -----------------------------------------------------\n");
    say("| %-15s | %-15u | %-15f | \n", "total", st->processed_nodes, st->time_total);
    say(" -----------------------------------------------------\n");
  }
  return st;
}

extern "C" struct BFSStats* breadthFirstSearchPullGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return bfs_dropin(a, g, BFS_PULL, "Starting BFS PULL/BU (SOURCE NODE)", false);
}
extern "C" struct BFSStats* breadthFirstSearchPushGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return bfs_dropin(a, g, BFS_PUSH, "Starting BFS PUSH/TD (SOURCE NODE)", false);
}
extern "C" struct BFSStats* breadthFirstSearchDirectionOptimizedGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return bfs_dropin(a, g, BFS_DO, "Starting BFS PUSH/PULL(SOURCE NODE)", false);
}
extern "C" struct BFSStats* breadthFirstSearchPushBitmapGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return bfs_dropin(a, g, BFS_PUSH, "Starting BFS PUSH/Bitmap (SOURCE NODE)", false);
}
extern "C" struct BFSStats* breadthFirstSearchPushDirectionOptimizedBitmapGraphCSR(struct Arguments* a,
                                                                                   struct GraphCSR* g) {
  return bfs_dropin(a, g, BFS_DO, "Starting BFS PUSH/PULL Bitmap (SOURCE NODE)", true);
}

// ---- DualOrder (BFS.c:1045-1562, graphCSR.c:250-335) ---------------------
//
// The DualOrder variants run top-down steps in the forward CSR's vertex
// order and bottom-up steps in the inverse CSR's, translating the frontier
// and the parent array between the two orders through the label maps when
// the direction changes (syncDualOrderParentArrays, BFS.c:182-211: the
// parents are copied into parents_DualOrder in the other order and the two
// pointers swapped, once entering and once leaving a bottom-up phase).
// Without reordering both orders are the identity (this library's
// preprocessing builds no other), and then the search is the plain one and
// the only trace of the translation is parents_DualOrder: after a
// direction-optimized search it holds the parent array as it stood when the
// last bottom-up phase ended (the sentinels if no bottom-up step ran); the
// pull-only and push-only variants never translate and leave it at the
// sentinels.  distances_DualOrder is never written, as in the reference.
// Graphs whose two orders differ (built by the reference's reordering) are
// not provided: message and NULL, which the reference's runner skips.

static bool labels_identity(const GraphCSR* g) {
  const uint32_t V = g->num_vertices;
  const uint32_t* arrs[4] = {g->sorted_edges_array ? g->sorted_edges_array->label_array : nullptr,
                             g->sorted_edges_array ? g->sorted_edges_array->inverse_label_array : nullptr,
                             g->inverse_sorted_edges_array ? g->inverse_sorted_edges_array->label_array : nullptr,
                             g->inverse_sorted_edges_array ? g->inverse_sorted_edges_array->inverse_label_array
                                                           : nullptr};
  int bad = 0;
  for (const uint32_t* a : arrs) {
    if (!a) continue;
    host_par_for(V, [&](size_t lo, size_t hi) {
      int b = 0;
      for (size_t v = lo; v < hi; v++) b |= a[v] != (uint32_t)v;
      if (b) __atomic_store_n(&bad, 1, __ATOMIC_RELAXED);
    });
  }
  return !bad;
}

static struct BFSStats* bfs_dropin_dual(struct Arguments* a, struct GraphCSR* graph, uint32_t mode,
                                        const char* title) {
  if (!labels_identity(graph)) {
    say(" -----------------------------------------------------\n");
    say("| %-51s | \n", "DualOrder BFS on reordered labels not provided");
    say(" -----------------------------------------------------\n");
    return nullptr;
  }
  BFSStats* st = bfs_dropin(a, graph, mode, title, false, mode == BFS_DO);
  if (mode != BFS_DO || (uint32_t)a->source >= graph->num_vertices) return st;
  // the step index of the last bottom-up step: its discoveries have depth
  // index + 1, and everything found up to then is in the snapshot
  const BfsResult& r = g_last_bfs;
  int last_bu = -1;
  for (size_t i = 0; i < r.levels.size(); i++)
    if (r.levels[i].direction) last_bu = (int)i;
  if (last_bu < 0) return st;
  const uint32_t dmax = (uint32_t)last_bu + 1;
  const int* par = st->parents;
  const uint32_t* dist = st->distances;
  int* dual = st->parents_DualOrder;
  host_par_for(graph->num_vertices, [&](size_t lo, size_t hi) {
    for (size_t v = lo; v < hi; v++)
      if (par[v] >= 0 && dist[v] <= dmax) dual[v] = par[v];
  });
  return st;
}

extern "C" struct BFSStats* breadthFirstSearchPullGraphCSRDualOrder(struct Arguments* a, struct GraphCSR* g) {
  return bfs_dropin_dual(a, g, BFS_PULL, "Starting BFS DualOrder PULL/BU (SOURCE NODE)");
}
extern "C" struct BFSStats* breadthFirstSearchPushGraphCSRDualOrder(struct Arguments* a, struct GraphCSR* g) {
  return bfs_dropin_dual(a, g, BFS_PUSH, "Starting BFS DualOrder PUSH/TD (SOURCE NODE)");
}
extern "C" struct BFSStats* breadthFirstSearchDirectionOptimizedGraphCSRDualOrder(struct Arguments* a,
                                                                                   struct GraphCSR* g) {
  return bfs_dropin_dual(a, g, BFS_DO, "Starting BFS DualOrder PUSH/PULL(SOURCE NODE)");
}
// breadthFirstSearchGraphCSRDualOrder (BFS.c:1045-1068).
extern "C" struct BFSStats* breadthFirstSearchGraphCSRDualOrder(struct Arguments* a, struct GraphCSR* g) {
  switch (a->pushpull) {
    case 0:
      return breadthFirstSearchPullGraphCSRDualOrder(a, g);
    case 1:
      return breadthFirstSearchPushGraphCSRDualOrder(a, g);
    default:
      return breadthFirstSearchDirectionOptimizedGraphCSRDualOrder(a, g);
  }
}

// breadthFirstSearchGraphCSR (BFS.c:238-268).
extern "C" struct BFSStats* breadthFirstSearchGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  switch (a->pushpull) {
    case 0:
      return breadthFirstSearchPullGraphCSR(a, g);
    case 1:
      return breadthFirstSearchPushGraphCSR(a, g);
    case 2:
      return breadthFirstSearchDirectionOptimizedGraphCSR(a, g);
    case 3:
      return breadthFirstSearchPushBitmapGraphCSR(a, g);
    case 4:
      return breadthFirstSearchPushDirectionOptimizedBitmapGraphCSR(a, g);
    default:
      return breadthFirstSearchDirectionOptimizedGraphCSR(a, g);
  }
}

// Single-level steps over host state (BFS.c:639-754).
int bfs_td_step_host(ogb::DevGraph& g, const uint32_t* q, uint32_t qsize, int32_t* parents, uint32_t* distances,
                     uint32_t* next_q, uint32_t* next_size, uint32_t* mf, cudaStream_t s);
int bfs_bu_step_host(ogb::DevGraph& g, const uint32_t* bm_cur, uint32_t* bm_next, int32_t* parents,
                     uint32_t* distances, uint32_t* nf, cudaStream_t s);

extern "C" uint32_t topDownStepGraphCSR(struct GraphCSR* graph, struct ArrayQueue* q, struct ArrayQueue** local,
                                        struct BFSStats* stats) {
  (void)local;
  int status = OK;
  ogb_graph* dg = mirror_of(graph, &status);
  if (!dg) die_status("device copy of GraphCSR", status);
  uint32_t next_size = 0, mf = 0;
  OGB_MUST(bfs_td_step_host(dg->g, q->queue + q->head, q->tail - q->head, stats->parents, stats->distances,
                            q->queue + q->tail_next, &next_size, &mf, lib_stream()));
  q->tail_next += next_size;
  return mf;
}

extern "C" uint32_t bottomUpStepGraphCSR(struct GraphCSR* graph, struct Bitmap* cur, struct Bitmap* next,
                                         struct BFSStats* stats) {
  int status = OK;
  ogb_graph* dg = mirror_of(graph, &status);
  if (!dg) die_status("device copy of GraphCSR", status);
  uint32_t nf = 0;
  OGB_MUST(bfs_bu_step_host(dg->g, cur->bitarray, next->bitarray, stats->parents, stats->distances, &nf,
                            lib_stream()));
  return nf;
}

// The DualOrder steps (BFS.c:1442-1562) are the plain steps' code.
extern "C" uint32_t topDownStepGraphCSRDualOrder(struct GraphCSR* graph, struct ArrayQueue* sharedFrontierQueue,
                                                 struct ArrayQueue** localFrontierQueues, struct BFSStats* stats) {
  return topDownStepGraphCSR(graph, sharedFrontierQueue, localFrontierQueues, stats);
}
extern "C" uint32_t bottomUpStepGraphCSRDualOrder(struct GraphCSR* graph, struct Bitmap* bitmapCurr,
                                                  struct Bitmap* bitmapNext, struct BFSStats* stats) {
  return bottomUpStepGraphCSR(graph, bitmapCurr, bitmapNext, stats);
}

// --------------------------------------------------------------- PageRank ---

extern "C" struct PageRankStats* newPageRankStatsGraphCSR(struct GraphCSR* graph) {
  const uint32_t V = graph->num_vertices;
  PageRankStats* st = (PageRankStats*)host_alloc(sizeof(PageRankStats));
  st->damp = 0.85f;
  st->base_pr = 1.0f - st->damp;
  st->iterations = 0;
  st->num_vertices = V;
  st->time_total = 0.0;
  st->error_total = 0.0;
  st->activeVertices = 0;
  st->realRanks = (uint32_t*)pool_alloc((size_t)V * 4);
  st->pageRanks = (float*)pool_alloc((size_t)V * 4);
  const float base = st->base_pr;
  host_par_for(V, [&](size_t lo, size_t hi) {
    for (size_t v = lo; v < hi; v++) {
      st->pageRanks[v] = base;
      st->realRanks[v] = (uint32_t)v;
    }
  });
  return st;
}

extern "C" void freePageRankStats(struct PageRankStats* st) {
  if (!st) return;
  pool_free(st->realRanks, (size_t)st->num_vertices * 4);
  pool_free(st->pageRanks, (size_t)st->num_vertices * 4);
  free(st);
}

static struct PageRankStats* pr_dropin(struct Arguments* a, struct GraphCSR* graph, uint32_t mode,
                                       const char* title) {
  PageRankStats* st = newPageRankStatsGraphCSR(graph);
  say(" -----------------------------------------------------\n");
  say("| %-51s | \n", title);
  say(" -----------------------------------------------------\n");
  say("| %-51.13lf | \n", a->epsilon);
  say(" -----------------------------------------------------\n");
  say("| %-10s | %-8s | %-15s | %-9s | \n", "Iteration", "Active", "Error", "Time (S)");
  say(" -----------------------------------------------------\n");
  int status = OK;
  ogb_graph* dg = mirror_of(graph, &status);
  if (!dg) die_status("device copy of GraphCSR", status);
  cudaStream_t s = lib_stream();
  const uint32_t V = graph->num_vertices;
  DevBuf d_pr;
  OGB_MUST(d_pr.alloc((size_t)V * 4 + 4));
  static PrResult r;
  const double t0 = now_s();
  if (mode == PR_PULL || mode == PR_PUSH)
    OGB_MUST(pagerank_run(dg->g, mode, a->iterations, a->epsilon, d_pr.as<float>(), nullptr, &r, s));
  else
    OGB_MUST(pagerank_dd_run(dg->g, mode, a->iterations, a->epsilon, d_pr.as<float>(), &r, s));
  OGB_MUST(d2h(st->pageRanks, d_pr.p, (size_t)V * 4, s));
  st->time_total = now_s() - t0;
  st->iterations = r.iterations;
  st->error_total = r.error_total;
  st->activeVertices = r.activeVertices;
  if (!quiet()) {
    const double per = r.executed ? (r.ms / 1000.0) / r.executed : 0.0;
    for (uint32_t i = 0; i < r.executed && i < 1024; i++)
      say("| %-10u | %-8u | %-15.13lf | %-9f | \n", i, r.active_hist[i], r.err_hist[i], per);
    double sum = 0.0;
    for (uint32_t v = 0; v < V; v++) sum += st->pageRanks[v];
    say(" -----------------------------------------------------\n");
    say("| %-10s | %-8s | %-15s | %-9s | \n", "Iterations", "PR Sum", "Error", "Time (S)");
    say(" -----------------------------------------------------\n");
    say("| %-10u | %-8lf | %-15.13lf | %-9f | \n", st->iterations, sum, st->error_total, st->time_total);
    say(" -----------------------------------------------------\n");
  }
  return st;
}

extern "C" struct PageRankStats* pageRankPullGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return pr_dropin(a, g, PR_PULL, "Starting Page Rank Pull (tolerance/epsilon)");
}
extern "C" struct PageRankStats* pageRankPushGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return pr_dropin(a, g, PR_PUSH, "Starting Page Rank Push (tolerance/epsilon)");
}
extern "C" struct PageRankStats* pageRankDataDrivenPullGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return pr_dropin(a, g, PR_DD_PULL, "Starting Page Rank Pull DD (tolerance/epsilon)");
}
extern "C" struct PageRankStats* pageRankDataDrivenPushGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return pr_dropin(a, g, PR_DD_PUSH, "Starting Page Rank Push DD (tolerance/epsilon)");
}
extern "C" struct PageRankStats* pageRankDataDrivenPullPushGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return pr_dropin(a, g, PR_DD_PULLPUSH, "Starting Page Rank Pull-Push DD (tolerance/epsilon)");
}

// pageRankGraphCSR (pageRank.c:871-936): pull, push and the data-driven
// variants (6 pull, 7 push, 8 pull-push) are provided; the fixed-point and
// quantized variants are not part of this library.
extern "C" struct PageRankStats* pageRankGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  switch (a->pushpull) {
    case 0:
      return pageRankPullGraphCSR(a, g);
    case 1:
      return pageRankPushGraphCSR(a, g);
    case 6:
      return pageRankDataDrivenPullGraphCSR(a, g);
    case 7:
      return pageRankDataDrivenPushGraphCSR(a, g);
    case 8:
      return pageRankDataDrivenPullPushGraphCSR(a, g);
    default:
      if (a->pushpull > 13) return pageRankPullGraphCSR(a, g);
      say(" -----------------------------------------------------\n");
      say("| %-51s | \n", "PR variant not provided by ogb200 (use 0, 1, 6, 7 or 8)");
      say(" -----------------------------------------------------\n");
      return nullptr;
  }
}

// radixSortEdgesByPageRank (reorder.c:165-221): labels stably sorted by the
// fixed-point rank key, in place; the same array is returned.
extern "C" uint32_t* radixSortEdgesByPageRank(float* pageRanks, uint32_t* labels, uint32_t num_vertices) {
  if (!num_vertices) return labels;
  cudaStream_t s = lib_stream();
  DevBuf d_r, d_l;
  OGB_MUST(d_r.alloc((size_t)num_vertices * 4));
  OGB_MUST(d_l.alloc((size_t)num_vertices * 4));
  OGB_MUST(h2d(d_r.p, pageRanks, (size_t)num_vertices * 4, s));
  OGB_MUST(h2d(d_l.p, labels, (size_t)num_vertices * 4, s));
  OGB_MUST(rank_sort(d_r.as<float>(), d_l.as<uint32_t>(), num_vertices, s));
  OGB_MUST(d2h(labels, d_l.p, (size_t)num_vertices * 4, s));
  return labels;
}

// ------------------------------------------------------------------- SPMV ---

// newSPMVStatsGraphCSR (SPMV.c:45-66): both vectors zeroed.
extern "C" struct SPMVStats* newSPMVStatsGraphCSR(struct GraphCSR* graph) {
  const uint32_t V = graph->num_vertices;
  SPMVStats* st = (SPMVStats*)host_alloc(sizeof(SPMVStats));
  st->iterations = 0;
  st->arguments = nullptr;
  st->num_vertices = V;
  st->time_total = 0.0;
  st->vector_output = (float*)host_alloc((size_t)V * 4);
  st->vector_input = (float*)host_alloc((size_t)V * 4);
  host_par_for(V, [&](size_t lo, size_t hi) {
    for (size_t v = lo; v < hi; v++) {
      st->vector_output[v] = 0.0f;
      st->vector_input[v] = 0.0f;
    }
  });
  return st;
}

// freeSPMVStats (SPMV.c:139-154).
extern "C" void freeSPMVStats(struct SPMVStats* st) {
  if (!st) return;
  free(st->vector_output);
  free(st->vector_input);
  free(st);
}

static struct SPMVStats* spmv_dropin(struct Arguments* a, struct GraphCSR* graph, uint32_t mode,
                                     const char* title) {
  SPMVStats* st = newSPMVStatsGraphCSR(graph);
  say(" -----------------------------------------------------\n");
  say("| %-51s | \n", title);
  say(" -----------------------------------------------------\n");
  say("| %-21s | %-27s | \n", "Iteration", "Time (S)");
  say(" -----------------------------------------------------\n");
  int status = OK;
  ogb_graph* dg = mirror_of(graph, &status);
  if (!dg) die_status("device copy of GraphCSR", status);
  cudaStream_t s = lib_stream();
  const uint32_t V = graph->num_vertices;
  DevBuf d_x, d_y;
  OGB_MUST(d_x.alloc((size_t)V * 4 + 4));
  OGB_MUST(d_y.alloc((size_t)V * 4 + 4));
  double ms = 0.0;
  OGB_MUST(spmv_run(dg->g, mode, a->iterations, d_x.as<float>(), d_y.as<float>(), &ms, s));
  OGB_MUST(d2h(st->vector_input, d_x.p, (size_t)V * 4, s));
  OGB_MUST(d2h(st->vector_output, d_y.p, (size_t)V * 4, s));
  st->iterations = a->iterations;
  st->time_total = ms / 1000.0;
  if (!quiet()) {
    double sum = 0.0;
    for (uint32_t v = 0; v < V; v++) sum += ((int)(st->vector_output[v] * 100 + .5) / 100.0);
    say(" -----------------------------------------------------\n");
    say("| %-15s | %-15s | %-15s | \n", "Iterations", "Sum", "Time (S)");
    say(" -----------------------------------------------------\n");
    say("| %-15u | %-15lf | %-15f | \n", st->iterations, sum, st->time_total);
    say(" -----------------------------------------------------\n");
  }
  return st;
}

extern "C" struct SPMVStats* SPMVPullGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return spmv_dropin(a, g, 0, "Starting SPMV-PULL");
}
extern "C" struct SPMVStats* SPMVPushGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  return spmv_dropin(a, g, 1, "Starting SPMV-PUSH");
}

// SPMVGraphCSR (SPMV.c:588-614): 0 pull, 1 push, other values pull; the
// fixed-point variants (2, 3) are not part of this library (message + NULL).
extern "C" struct SPMVStats* SPMVGraphCSR(struct Arguments* a, struct GraphCSR* g) {
  switch (a->pushpull) {
    case 0:
      return SPMVPullGraphCSR(a, g);
    case 1:
      return SPMVPushGraphCSR(a, g);
    case 2:
    case 3:
      say(" -----------------------------------------------------\n");
      say("| %-51s | \n", "SPMV variant not provided by ogb200 (use 0 or 1)");
      say(" -----------------------------------------------------\n");
      return nullptr;
    default:
      return SPMVPullGraphCSR(a, g);
  }
}

// ------------------------------------------------------------------ roots ---

// generateRandomRootGraphCSR (graphRun.c:537-556).
extern "C" uint32_t generateRandomRootGraphCSR(mt19937state* mt, struct GraphCSR* graph) {
  const uint32_t* labels = graph->sorted_edges_array ? graph->sorted_edges_array->label_array : nullptr;
  for (;;) {
    const uint32_t source = (uint32_t)generateRandInt(mt);
    if (source < graph->num_vertices) {
      const uint32_t t = labels ? labels[source] : source;
      if (graph->vertices->out_degree[t] > graph->avg_degree) return source;
    }
  }
}

// ------------------------------------------------------------- device API ---

extern "C" int ogb_dropin_bfs_phases(double* seconds, uint32_t n) {
  if (!seconds) return ogb::fail(ogb::ERR_ARG, "null output");
  for (uint32_t i = 0; i < n && i < OGB_DROPIN_BFS_PHASES; i++) seconds[i] = g_bfs_phase[i];
  return ogb::OK;
}

extern "C" const char* ogb_last_error(void) { return ogb::last_error(); }
extern "C" int ogb_weighted_layout(void) { return OGB200_WEIGHTED; }
extern "C" void ogb_set_quiet(int q) { g_quiet = q ? 1 : 0; }

extern "C" int ogb_graph_create(ogb_graph** g) {
  if (!g) return fail(ERR_ARG, "null");
  *g = new ogb_graph();
  return OK;
}

extern "C" void ogb_graph_destroy(ogb_graph* g) { delete g; }

// A null stream argument is the legacy default stream (as in the CUDA
// libraries), so the call waits for the caller's default-stream work.
static cudaStream_t as_stream(void* s) { return s ? (cudaStream_t)s : cudaStreamLegacy; }

extern "C" int ogb_graph_build(ogb_graph* g, const uint32_t* d_src, const uint32_t* d_dst, const float* d_w,
                               uint32_t E, uint32_t V, uint32_t sort_type, void* stream) {
  if (!g) return fail(ERR_ARG, "null graph");
  if (E && (!d_src || !d_dst)) return fail(ERR_ARG, "null edge arrays");
  cudaStream_t s = as_stream(stream);
  OGB_TRY(graph_build(g->g, d_src, d_dst, d_w, E, V, sort_type, s));
  return graph_check(g->g, s);
}

extern "C" int ogb_graph_view(ogb_graph* g, int inverse, ogb_csr_view* v) {
  if (!g || !v) return fail(ERR_ARG, "null");
  DevCSR& c = inverse ? g->g.inv : g->g.fwd;
  v->num_vertices = g->g.V;
  v->num_edges = g->g.E;
  v->src = c.d_src();
  v->dst = c.d_dst();
  v->weight = c.d_w();
  v->out_degree = c.d_out_degree();
  v->in_degree = c.d_in_degree();
  v->edges_idx = c.d_edges_idx();
  return OK;
}

extern "C" ogb_graph* ogb_graph_of(const void* graphCSR) {
  int st = OK;
  return mirror_of((const GraphCSR*)graphCSR, &st);
}

extern "C" int ogb_sort_edges(const uint32_t* d_src, const uint32_t* d_dst, const float* d_w, uint32_t E,
                              uint32_t sort_type, uint32_t* o_src, uint32_t* o_dst, float* o_w, void* stream) {
  cudaStream_t s = as_stream(stream);
  static SortWorkspace* ws = new SortWorkspace();
  KV in{const_cast<uint32_t*>(d_src), const_cast<uint32_t*>(d_dst), (uint32_t*)(d_w)};
  KV out{o_src, o_dst, (uint32_t*)o_w};
  if (d_w && !o_w) return fail(ERR_ARG, "weighted sort needs an output weight array");
  if (!d_w) out.v1 = nullptr;
  const bool lex = sort_type == 1 || sort_type == 3;
  OGB_TRY(lex ? sort_pairs_lex(in, out, E, *ws, s) : sort_pairs(in, out, E, *ws, s));
  return sort_check(*ws, s);
}

extern "C" int ogb_bfs(ogb_graph* g, uint32_t root, uint32_t mode, int32_t* d_parents, uint32_t* d_distances,
                       ogb_bfs_info* info, void* stream) {
  if (!g || !d_parents || !d_distances) return fail(ERR_ARG, "null");
  if (mode > 4) return fail(ERR_ARG, "bfs mode %u", mode);
  static thread_local BfsResult r;
  OGB_TRY(bfs_run(g->g, root, mode, d_parents, d_distances, &r, true, false, as_stream(stream)));
  if (info) {
    info->iteration = r.iteration;
    info->processed_nodes = r.processed_nodes;
    info->td_steps = r.td_steps;
    info->bu_steps = r.bu_steps;
    info->reached = r.reached;
    info->levels = (uint32_t)r.nlevels;
    info->reached_out_edges = r.reached_out_edges;
    info->edges_examined = r.edges_examined;
    info->ms = r.ms;
    info->launches = r.launches;
    info->pad = 0;
  }
  g->g.bfs_trace.swap(r.levels);
  g->g.bfs_feat.swap(r.feat);
  return OK;
}

extern "C" int ogb_bfs_features(ogb_graph* g, float* features, uint32_t max_levels, uint32_t* count) {
  if (!g || !features || !count) return fail(ERR_ARG, "ogb_bfs_features: null argument");
  const uint32_t n = std::min<uint32_t>(max_levels, (uint32_t)g->g.bfs_trace.size());
  memcpy(features, g->g.bfs_feat.data(), (size_t)n * 8 * sizeof(float));
  *count = n;
  return OK;
}

extern "C" int ogb_bfs_set_policy(const float* params) { return bfs_set_policy(params); }

extern "C" uint32_t ogb_mlp_nparams(uint32_t in, uint32_t hidden) { return (uint32_t)mlp_nparams_host((int)in, (int)hidden); }

extern "C" int ogb_mlp_grad(uint32_t in, uint32_t hidden, uint32_t loss, const float* d_X, const float* d_T,
                            uint32_t batch, const float* params, float* grad, float* loss_out, void* stream) {
  if (!d_X || !d_T || !params || !grad) return fail(ERR_ARG, "ogb_mlp_grad: null argument");
  return mlp_grad((int)in, (int)hidden, (int)loss, d_X, d_T, (int)batch, params, grad, loss_out, as_stream(stream));
}

extern "C" int ogb_mlp_train(uint32_t in, uint32_t hidden, uint32_t loss, const float* d_X, const float* d_T,
                             uint32_t n, uint32_t epochs, uint32_t batch, float lr, uint32_t seed, float* params,
                             float* loss_hist, void* stream) {
  if (!d_X || !d_T || !params) return fail(ERR_ARG, "ogb_mlp_train: null argument");
  return mlp_train((int)in, (int)hidden, (int)loss, d_X, d_T, (int)n, (int)epochs, (int)batch, lr, seed, params,
                   loss_hist, as_stream(stream));
}

extern "C" int ogb_mlp_infer(uint32_t in, uint32_t hidden, const float* params, const float* d_X, uint32_t n,
                             float* d_Y, void* stream) {
  if (!params || (n && (!d_X || !d_Y))) return fail(ERR_ARG, "ogb_mlp_infer: null argument");
  return mlp_infer((int)in, (int)hidden, params, d_X, (int)n, d_Y, as_stream(stream));
}

extern "C" int ogb_pagerank_warm_start(ogb_graph* g, uint32_t hidden, const float* params, float* d_init,
                                       void* stream) {
  if (!g || !params || !d_init) return fail(ERR_ARG, "ogb_pagerank_warm_start: null argument");
  return pr_warm_start(g->g, (int)hidden, params, d_init, as_stream(stream));
}

extern "C" int ogb_msbfs(ogb_graph* g, const uint32_t* roots, uint32_t nroots, uint16_t* d_depths,
                         ogb_msbfs_info* info, void* stream) {
  if (!g || !roots || !d_depths) return fail(ERR_ARG, "ogb_msbfs: null argument");
  MsResult r;
  OGB_TRY(msbfs_run(g->g, roots, nroots, d_depths, &r, as_stream(stream)));
  if (info) {
    info->levels = r.levels;
    info->push_levels = r.push_levels;
    info->pull_levels = r.pull_levels;
    info->launches = r.launches;
    info->reached_pairs = r.reached;
    info->edges_examined = r.edges_examined;
    info->ms = r.ms;
    info->init_ms = r.init_ms;
  }
  return OK;
}

extern "C" int ogb_ppr(ogb_graph* g, const uint32_t* seeds, uint32_t nseeds, uint32_t max_iterations,
                       double epsilon, float* d_ranks, ogb_ppr_info* info, void* stream) {
  if (!g || !seeds) return fail(ERR_ARG, "ogb_ppr: null argument");
  PprResult r;
  OGB_TRY(ppr_run(g->g, seeds, nseeds, max_iterations, epsilon, d_ranks, &r, as_stream(stream)));
  if (info) {
    info->executed = r.executed;
    info->converged = r.converged;
    info->launches = r.launches;
    info->pad = 0;
    info->ms = r.ms;
    for (int k = 0; k < 32; k++) info->err_last[k] = r.err_last[k];
  }
  return OK;
}

struct ogb_batch {
  GraphBatch* b = nullptr;
};

extern "C" ogb_batch* ogb_batch_create(uint32_t num_graphs, const uint32_t* num_vertices,
                                       const uint64_t* edge_offsets, const uint32_t* src, const uint32_t* dst,
                                       uint32_t sort_type) {
  if (!num_vertices || !edge_offsets || (!src && edge_offsets[num_graphs]) || (!dst && edge_offsets[num_graphs])) {
    fail(ERR_ARG, "ogb_batch_create: null argument");
    return nullptr;
  }
  GraphBatch* b = batch_new();
  if (batch_create(*b, num_graphs, num_vertices, edge_offsets, src, dst, sort_type, lib_stream()) != OK) {
    batch_free(b);
    return nullptr;
  }
  ogb_batch* h = new ogb_batch();
  h->b = b;
  return h;
}

extern "C" void ogb_batch_free(ogb_batch* b) {
  if (!b) return;
  batch_free(b->b);
  delete b;
}

extern "C" int ogb_batch_offsets(ogb_batch* b, uint32_t* vertex_offsets) {
  if (!b || !vertex_offsets) return fail(ERR_ARG, "ogb_batch_offsets: null argument");
  memcpy(vertex_offsets, batch_voff(b->b), (size_t)(batch_ngraphs(b->b) + 1) * 4);
  return OK;
}

extern "C" int ogb_batch_bfs(ogb_batch* b, const uint32_t* roots, int32_t* d_parents, uint32_t* d_distances,
                             ogb_batch_bfs_info* info, void* stream) {
  if (!b || !roots || !d_parents || !d_distances) return fail(ERR_ARG, "ogb_batch_bfs: null argument");
  BfsResult r;
  OGB_TRY(batch_bfs(*b->b, roots, d_parents, d_distances, &r, as_stream(stream)));
  if (info) {
    info->levels = (uint32_t)r.nlevels;
    info->td_steps = r.td_steps;
    info->bu_steps = r.bu_steps;
    info->reached = r.reached;
    info->ms = r.ms;
  }
  return OK;
}

extern "C" int ogb_batch_pagerank(ogb_batch* b, uint32_t max_iterations, double epsilon, float* d_ranks,
                                  ogb_batch_pr_graph* per_graph, ogb_batch_pr_info* info, void* stream) {
  if (!b || !d_ranks) return fail(ERR_ARG, "ogb_batch_pagerank: null argument");
  const uint32_t n = batch_ngraphs(b->b);
  std::vector<BatchPrGraph> pg(n);
  double ms = 0.0;
  uint32_t cap = 0;
  OGB_TRY(batch_pagerank(*b->b, max_iterations, epsilon, d_ranks, pg.data(), &ms, &cap, as_stream(stream)));
  if (per_graph)
    for (uint32_t i = 0; i < n; i++) {
      per_graph[i].iterations = pg[i].iterations;
      per_graph[i].executed = pg[i].executed;
      per_graph[i].activeVertices = pg[i].activeVertices;
      per_graph[i].converged = pg[i].converged;
      per_graph[i].error_total = pg[i].error_total;
    }
  if (info) {
    info->ms = ms;
    info->captured = cap;
    info->pad = 0;
  }
  return OK;
}

extern "C" int ogb_batch_autotune(ogb_batch* b, ogb_tune_info* info) {
  if (!b) return fail(ERR_ARG, "ogb_batch_autotune: null argument");
  TuneResult t;
  OGB_TRY(batch_autotune(*b->b, 5, &t, lib_stream()));
  if (info) {
    info->ncandidates = t.n;
    info->best = t.best;
    for (int i = 0; i < 16; i++) {
      info->warp_thr[i] = t.warp_thr[i];
      info->cta_thr[i] = t.cta_thr[i];
      info->ms[i] = t.ms[i];
    }
  }
  return OK;
}

extern "C" int ogb_bfs_trace(ogb_graph* g, ogb_bfs_level* levels, uint32_t max_levels, uint32_t* count) {
  if (!g) return fail(ERR_ARG, "null");
  const uint32_t n = std::min<uint32_t>(max_levels, (uint32_t)g->g.bfs_trace.size());
  for (uint32_t i = 0; i < n; i++) {
    const BfsLevel& L = g->g.bfs_trace[i];
    levels[i].direction = L.direction;
    levels[i].discovered = L.discovered;
    levels[i].frontier = L.frontier;
    levels[i].mf = L.mf;
    levels[i].mu = L.mu;
    levels[i].pad = 0;
    levels[i].edges = L.edges;
    levels[i].ms = L.ms;
    levels[i].pad2 = 0;
  }
  if (count) *count = n;
  return OK;
}

extern "C" int ogb_pagerank(ogb_graph* g, uint32_t mode, uint32_t max_iters, double eps, float* d_ranks,
                            const float* d_init, ogb_pr_info* info, void* stream) {
  if (!g || !d_ranks) return fail(ERR_ARG, "null");
  const bool dd = mode == PR_DD_PULL || mode == PR_DD_PUSH || mode == PR_DD_PULLPUSH;
  if (mode > 1 && !dd) return fail(ERR_ARG, "pagerank mode %u", mode);
  if (dd && d_init) return fail(ERR_ARG, "pagerank mode %u takes no start vector", mode);
  static thread_local PrResult r;
  if (dd)
    OGB_TRY(pagerank_dd_run(g->g, mode, max_iters, eps, d_ranks, &r, as_stream(stream)));
  else
    OGB_TRY(pagerank_run(g->g, mode, max_iters, eps, d_ranks, d_init, &r, as_stream(stream)));
  g->g.pr_last_executed = r.executed;
  memcpy(g->g.pr_err_hist, r.err_hist, sizeof(double) * std::min<uint32_t>(r.executed, 1024));
  memcpy(g->g.pr_active_hist, r.active_hist, sizeof(uint32_t) * std::min<uint32_t>(r.executed, 1024));
  if (info) {
    info->iterations = r.iterations;
    info->executed = r.executed;
    info->activeVertices = r.activeVertices;
    info->converged = r.converged;
    info->error_total = r.error_total;
    info->ms = r.ms;
    info->launches = r.launches;
    info->pad = 0;
  }
  return OK;
}

extern "C" int ogb_spmv(ogb_graph* g, uint32_t mode, uint32_t iterations, float* d_x, float* d_y, ogb_spmv_info* info,
                        void* stream) {
  if (!g || !d_x || !d_y) return fail(ERR_ARG, "null");
  double ms = 0.0;
  OGB_TRY(spmv_run(g->g, mode, iterations, d_x, d_y, &ms, as_stream(stream)));
  if (info) {
    info->iterations = iterations;
    info->weighted = g->g.weighted ? 1u : 0u;
    info->ms = ms;
  }
  return OK;
}

extern "C" int ogb_pagerank_range_init(ogb_graph* g, float* d_ranks, float* d_contrib, void* stream) {
  if (!g || !d_ranks || !d_contrib) return fail(ERR_ARG, "null");
  return pagerank_range_init(g->g, d_ranks, d_contrib, as_stream(stream));
}

extern "C" int ogb_pagerank_range_step(ogb_graph* g, uint32_t lo, uint32_t hi, const float* d_contrib,
                                       float* d_ranks, float* d_contrib_next, double epsilon, double* d_err,
                                       uint32_t* d_active, void* stream) {
  if (!g || !d_contrib || !d_ranks || !d_contrib_next || !d_err || !d_active) return fail(ERR_ARG, "null");
  return pagerank_range_step(g->g, lo, hi, d_contrib, d_ranks, d_contrib_next, epsilon, d_err, d_active,
                             as_stream(stream));
}

extern "C" int ogb_pagerank_range_step_peers(ogb_graph* g, uint32_t lo, uint32_t hi, const float* d_contrib,
                                             float* d_ranks, float* d_contrib_next, const uint64_t* d_peers,
                                             uint32_t npeers, double epsilon, double* d_err, uint32_t* d_active,
                                             void* stream) {
  if (!g || !d_contrib || !d_ranks || !d_contrib_next || !d_err || !d_active || (npeers && !d_peers))
    return fail(ERR_ARG, "null");
  return pagerank_range_step(g->g, lo, hi, d_contrib, d_ranks, d_contrib_next, epsilon, d_err, d_active,
                             as_stream(stream), reinterpret_cast<float* const*>(d_peers), npeers);
}

extern "C" int ogb_pagerank_range_finish(ogb_graph* g, float* d_ranks, void* stream) {
  if (!g || !d_ranks) return fail(ERR_ARG, "null");
  return pagerank_range_finish(g->g, d_ranks, as_stream(stream));
}

extern "C" int ogb_partition_edges(const uint32_t* d_src, const uint32_t* d_dst, const float* d_w, uint32_t E,
                                   const uint32_t* bounds, uint32_t nparts, uint32_t* d_out_src, uint32_t* d_out_dst,
                                   float* d_out_w, uint32_t* counts, void* stream) {
  return partition_edges(d_src, d_dst, d_w, E, bounds, nparts, d_out_src, d_out_dst, d_out_w, counts,
                         as_stream(stream));
}

extern "C" int ogb_bfs_range_init(ogb_graph* g, uint32_t lo, uint32_t hi, uint32_t root, int32_t* d_parents,
                                  uint32_t* d_dist, uint8_t* d_frontier, uint8_t* d_visited, int32_t* d_cand,
                                  uint64_t* d_counts, void* stream) {
  if (!g || !d_parents || !d_dist || !d_frontier || !d_visited || !d_cand || !d_counts) return fail(ERR_ARG, "null");
  return bfs_range_init(g->g, lo, hi, root, d_parents, d_dist, d_frontier, d_visited, d_cand,
                        reinterpret_cast<unsigned long long*>(d_counts), as_stream(stream));
}

extern "C" int ogb_bfs_range_expand(ogb_graph* g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                                    const uint8_t* d_frontier, const uint8_t* d_visited, uint8_t* d_next,
                                    int32_t* d_cand, int32_t* d_parents, uint32_t* d_dist, uint64_t* d_counts,
                                    void* stream) {
  if (!g || !d_frontier || !d_visited || !d_next || !d_cand || !d_parents || !d_dist || !d_counts)
    return fail(ERR_ARG, "null");
  return bfs_range_expand(g->g, lo, hi, direction, depth, d_frontier, d_visited, d_next, d_cand, d_parents, d_dist,
                          reinterpret_cast<unsigned long long*>(d_counts), as_stream(stream));
}

extern "C" int ogb_bfs_range_settle(ogb_graph* g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                                    int32_t* d_cand, uint8_t* d_next, uint8_t* d_visited, int32_t* d_parents,
                                    uint32_t* d_dist, uint64_t* d_counts, void* stream) {
  if (!g || !d_cand || !d_next || !d_visited || !d_parents || !d_dist || !d_counts) return fail(ERR_ARG, "null");
  return bfs_range_settle(g->g, lo, hi, direction, depth, d_cand, d_next, d_visited, d_parents, d_dist,
                          reinterpret_cast<unsigned long long*>(d_counts), as_stream(stream));
}

extern "C" int ogb_bfs_range_expand_peers(ogb_graph* g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                                          const uint8_t* d_frontier, const uint8_t* d_visited, uint8_t* d_next,
                                          const uint64_t* d_cand_peers, const uint32_t* d_bounds, uint32_t nparts,
                                          int32_t* d_parents, uint32_t* d_dist, uint64_t* d_counts, void* stream) {
  if (!g || !d_frontier || !d_visited || !d_next || !d_cand_peers || !d_bounds || !d_parents || !d_dist || !d_counts)
    return fail(ERR_ARG, "null");
  return bfs_range_expand_peers(g->g, lo, hi, direction, depth, d_frontier, d_visited, d_next,
                                reinterpret_cast<int32_t* const*>(d_cand_peers), d_bounds, nparts, d_parents, d_dist,
                                reinterpret_cast<unsigned long long*>(d_counts), as_stream(stream));
}

extern "C" int ogb_bfs_range_claim_peers(ogb_graph* g, uint32_t lo, uint32_t hi, uint32_t direction, uint32_t depth,
                                         int32_t* d_cand, uint8_t* d_next, const uint64_t* d_next_peers,
                                         uint32_t npeers, int32_t* d_parents, uint32_t* d_dist, uint64_t* d_counts,
                                         void* stream) {
  if (!g || !d_cand || !d_next || !d_next_peers || !d_parents || !d_dist || !d_counts) return fail(ERR_ARG, "null");
  return bfs_range_claim_peers(g->g, lo, hi, direction, depth, d_cand, d_next,
                               reinterpret_cast<uint8_t* const*>(d_next_peers), npeers, d_parents, d_dist,
                               reinterpret_cast<unsigned long long*>(d_counts), as_stream(stream));
}

extern "C" int ogb_sort_by_rank(const float* d_ranks, uint32_t* d_labels, uint32_t n, void* stream) {
  if (n && (!d_ranks || !d_labels)) return fail(ERR_ARG, "null");
  return rank_sort(d_ranks, d_labels, n, as_stream(stream));
}

extern "C" void ogb_pagerank_set_bins(uint32_t warp_thr, uint32_t cta_thr) { pagerank_set_bins(warp_thr, cta_thr); }

extern "C" void ogb_pagerank_get_bins(uint32_t* warp_thr, uint32_t* cta_thr, uint32_t* cta_threads,
                                      uint32_t* chunk_edges) {
  pagerank_get_bins(warp_thr, cta_thr, cta_threads, chunk_edges);
}

extern "C" int ogb_pagerank_history(ogb_graph* g, double* errors, uint32_t* active, uint32_t max_entries,
                                    uint32_t* count) {
  if (!g) return fail(ERR_ARG, "null");
  const uint32_t n = std::min<uint32_t>(max_entries, g->g.pr_last_executed);
  for (uint32_t i = 0; i < n; i++) {
    if (errors) errors[i] = g->g.pr_err_hist[i];
    if (active) active[i] = g->g.pr_active_hist[i];
  }
  if (count) *count = n;
  return OK;
}
