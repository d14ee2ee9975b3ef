// generate.cpp -- deterministic synthetic graph generators (host, threaded).
//
// Every random draw is a hash of (seed, edge index, draw index), so the
// output does not depend on the thread count and any slice can be
// regenerated on its own.  The reference reads these edges from .bin/.wbin
// files ({u32 src, u32 dst[, f32 w]} records, edgeList.c:336-594).
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "../../include/ogb200_device.h"

namespace {

inline uint64_t mix64(uint64_t z) {
  // SplitMix64 finalizer (Steele, Lea, Flood 2014).
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

inline uint64_t draw(uint64_t seed, uint64_t index, uint64_t k) {
  return mix64(mix64(seed ^ (k * 0xD1B54A32D192ED03ull)) ^ index);
}

inline double unit53(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

inline float weight_of(uint64_t seed, uint64_t i) {
  const double u = (double)(draw(seed ^ 0x5713ull, i, 0xFFFF) >> 40) * (1.0 / 16777216.0);
  return (float)(1.0 + 255.0 * u);  // [1, 256)
}

template <class F>
void parallel_for(uint64_t n, F&& f) {
  unsigned nt = std::max(1u, std::thread::hardware_concurrency());
  if (n < (1u << 16)) nt = 1;
  std::vector<std::thread> th;
  const uint64_t chunk = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; t++) {
    const uint64_t lo = t * chunk, hi = std::min<uint64_t>(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([=, &f] { f(lo, hi); });
  }
  for (auto& x : th) x.join();
}

// Seeded Fisher-Yates permutation of [0, n).
std::vector<uint32_t> permutation(uint32_t n, uint64_t seed) {
  std::vector<uint32_t> p(n);
  for (uint32_t i = 0; i < n; i++) p[i] = i;
  uint64_t state = mix64(seed ^ 0xA5A5A5A5ull);
  for (uint32_t i = n; i > 1; i--) {
    state = mix64(state);
    const uint32_t j = (uint32_t)(((unsigned __int128)state * i) >> 64);
    std::swap(p[i - 1], p[j]);
  }
  return p;
}

}  // namespace

extern "C" int ogb_generate_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b, double c,
                                 int permute, uint32_t* src, uint32_t* dst, float* w) {
  if (scale == 0 || scale > 30 || !src || !dst) return OGB_ERR_ARG;
  const uint64_t V = 1ull << scale;
  const uint64_t E = V * edge_factor;
  if (E > 0xFFFFFFFFull) return OGB_ERR_ARG;
  const double ab = a + b, abc = a + b + c;
  std::vector<uint32_t> perm;
  if (permute) perm = permutation((uint32_t)V, seed);
  parallel_for(E, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; i++) {
      uint32_t u = 0, v = 0;
      for (uint32_t l = 0; l < scale; l++) {
        const double r = unit53(draw(seed, i, l));
        const uint32_t bu = r >= ab ? 1u : 0u;                       // quadrants c, d
        const uint32_t bv = (r >= a && r < ab) || r >= abc ? 1u : 0u;  // quadrants b, d
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      if (permute) {
        u = perm[u];
        v = perm[v];
      }
      src[i] = u;
      dst[i] = v;
      if (w) w[i] = weight_of(seed, i);
    }
  });
  return OGB_OK;
}

extern "C" int ogb_generate_uniform(uint32_t num_vertices, uint64_t num_edges, uint64_t seed, uint32_t* src,
                                    uint32_t* dst, float* w) {
  if (!num_vertices || !src || !dst || num_edges > 0xFFFFFFFFull) return OGB_ERR_ARG;
  parallel_for(num_edges, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t i = lo; i < hi; i++) {
      src[i] = (uint32_t)(((unsigned __int128)draw(seed, i, 0) * num_vertices) >> 64);
      dst[i] = (uint32_t)(((unsigned __int128)draw(seed, i, 1) * num_vertices) >> 64);
      if (w) w[i] = weight_of(seed, i);
    }
  });
  return OGB_OK;
}

// side x side grid, vertex id r*side + c; each vertex points to its up to 4
// axis neighbours, and with probability p to its diagonal neighbour
// (r+1, c+1) and back.  Diagonal shortcuts shorten paths only locally, so the
// diameter stays of order side.
extern "C" int ogb_generate_grid(uint32_t side, double p, uint64_t seed, uint32_t* src, uint32_t* dst, float* w,
                                 uint64_t* num_edges) {
  if (side < 2 || !num_edges || (uint64_t)side * side > 0xFFFFFFFFull) return OGB_ERR_ARG;
  const bool always = p >= 1.0;
  const uint64_t thresh = always ? ~0ull : (uint64_t)(p * 18446744073709551616.0);
  uint64_t k = 0;
  for (uint32_t r = 0; r < side; r++) {
    for (uint32_t c = 0; c < side; c++) {
      const uint32_t v = r * side + c;
      auto emit = [&](uint32_t x, uint32_t y) {
        if (src) {
          src[k] = x;
          dst[k] = y;
          if (w) w[k] = weight_of(seed, k);
        }
        k++;
      };
      if (r > 0) emit(v, v - side);
      if (r + 1 < side) emit(v, v + side);
      if (c > 0) emit(v, v - 1);
      if (c + 1 < side) emit(v, v + 1);
      if (r + 1 < side && c + 1 < side && p > 0 && (always || draw(seed, v, 7) < thresh)) {
        emit(v, v + side + 1);
        emit(v + side + 1, v);
      }
    }
  }
  *num_edges = k;
  return OGB_OK;
}

extern "C" int ogb_write_edge_file(const char* path, const uint32_t* src, const uint32_t* dst, const float* w,
                                   uint64_t num_edges) {
  FILE* f = fopen(path, "wb");
  if (!f) return OGB_ERR_ARG;
  const size_t rec = w ? 12 : 8;
  const uint64_t chunk = 1u << 20;
  std::vector<uint32_t> buf(chunk * (rec / 4));
  for (uint64_t i = 0; i < num_edges; i += chunk) {
    const uint64_t n = std::min<uint64_t>(chunk, num_edges - i);
    for (uint64_t j = 0; j < n; j++) {
      uint32_t* r = &buf[j * (rec / 4)];
      r[0] = src[i + j];
      r[1] = dst[i + j];
      if (w) memcpy(&r[2], &w[i + j], 4);
    }
    if (fwrite(buf.data(), rec, n, f) != n) {
      fclose(f);
      return OGB_ERR_ARG;
    }
  }
  fclose(f);
  return OGB_OK;
}
