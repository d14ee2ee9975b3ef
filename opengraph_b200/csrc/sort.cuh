// sort.cuh -- stable LSD radix sort of (key, payload[, payload]) u32 arrays.
#pragma once
#include "common.cuh"

namespace ogb {

// One array set of an edge list on the device: key array and up to two
// payload arrays (dst and the weight bits, or src and the weight bits).
struct KV {
  uint32_t* k = nullptr;
  uint32_t* v0 = nullptr;
  uint32_t* v1 = nullptr;  // may be null (unweighted)
};

struct SortWorkspace {
  DevBuf hist;       // passes*256 u32 counts, then passes*256 exclusive bases
  DevBuf status;     // look-back words: passes * tiles * 256 u64
  DevBuf counters;   // per-pass tile counters + error word
  DevBuf tmp_k, tmp_v0, tmp_v1;  // one ping-pong array set
  int reserve(uint64_t n, bool weighted, int max_passes);
};

// Stable sort of `in` by key into `out`, moving the payloads along.  Every
// key must be below 2^key_bits (32: any key); the digits are ceil(key_bits /
// 8) groups of nearly equal width from bit 0 up, and digit groups in which
// every key has the same value are skipped.  `in` is not modified unless it
// aliases `out`.  Runs on `stream`; one small device->host read (the digit
// histograms) happens inside.
int sort_pairs(const KV& in, const KV& out, uint64_t n, SortWorkspace& ws, cudaStream_t stream,
               uint32_t key_bits = 32);

// Lexicographic (primary, secondary) stable sort: `in.k` is the primary key
// and `in.v0` the secondary key (both below 2^key_bits); payload v1 follows.
int sort_pairs_lex(const KV& in, const KV& out, uint64_t n, SortWorkspace& ws, cudaStream_t stream,
                   uint32_t key_bits = 32);

}  // namespace ogb
