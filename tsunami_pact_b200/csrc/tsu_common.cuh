// tsu_common.cuh -- shared types of the sm_100a WFA kernels.
//
// Conventions of the reference kernel (wfa_gpu.cu:214-215,643-645): pattern
// vertical (v), text horizontal (h), diagonal k = h - v, offset = h; the
// alignment ends on diagonal n - m at offset n.  Scores run in units of
// g = gcd(x, o, e): all reachable scores are multiples of g, so the steps in
// between are null and skipping them changes no wavefront.
#pragma once

#include <climits>
#include <cstdint>

namespace tsu {

constexpr int32_t kNull = INT32_MIN / 2;  // int32 offset null (reference: INT16_MIN/2, common.h:6)
constexpr int16_t kNull16 = -16384;       // int16 ring null (any negative value is out of bounds)

enum : int32_t { kPairOk = 0, kPairScratch = 1, kPairArena = 2, kPairInternal = 3 };
// backtrace word: bits 31..4 pre-extension M offset, 1..0 M source, 2 I ext, 3 D ext
enum : uint32_t { kSrcMis = 0, kSrcIns = 1, kSrcDel = 2, kIExt = 4, kDExt = 8 };
enum : uint32_t { kOpM = 0, kOpI = 1, kOpD = 2, kOpX = 8 };
// align kernel variants
enum : int { kModeShared = 0, kModeGlobal = 1 };

struct SeqView {
  int64_t n;  // pairs
  const uint8_t* pat;
  const int64_t* pat_off;
  const int32_t* pat_len;
  const uint8_t* txt;
  const int64_t* txt_off;
  const int32_t* txt_len;
};

struct PackView {
  uint64_t* words;      // packed 2-bit words, 32 bases per word, + 1 zero word per sequence
  const int64_t* woff;  // [2n]: pattern i at i, text i at n + i
  uint8_t* nonacgt;     // [2n]: 1 if the sequence holds a byte outside ACGT
};

struct AlignArgs {
  SeqView seq;
  PackView pk;
  const int32_t* order;  // pairs of this launch (nullptr: 0..n_order-1)
  int64_t n_order;
  int x, go, ge, g;      // reduced mismatch, open+extend, extend; gcd
  int rm, re;            // ring depths: rm = max(x, go) + 1, re = ge + 1
  int ring_w;            // diagonals per ring slot
  int seq_cap;           // shared-memory sequence words (uint32) per warp
  int32_t* ring_global;  // per-warp rings (global mode)
  int64_t ring_stride;   // int32 per warp in ring_global
  uint32_t* hist;        // per-warp backtrace words
  int64_t hist_cap;
  int2* table;           // per-warp step table: (lo, base) per score
  int32_t table_cap;
  int32_t* score;        // [n] (pair index)
  int32_t* status;       // [n]
  uint32_t* arena;       // CIGAR runs
  unsigned long long* arena_cursor;
  int64_t arena_cap;
  int64_t* cig_pos;      // [n]
  int32_t* cig_len;      // [n]
  unsigned int* queue;   // work-queue head
  int32_t* retry;        // [n] pairs to re-run with more scratch / arena
  unsigned int* retry_count;
  unsigned long long* work;  // [2]: wavefront cells computed, score steps
};

__host__ __device__ inline int ring_slots(int rm, int re) { return rm + 2 * re; }

// Shared memory per group of gw warps, in bytes: slot limits (lo, hi, alo
// per slot), warp partials [2][gw][8] (gw > 1), 4 broadcast words, then in
// shared mode an int16 ring of ring_slots * ring_w and seq_cap sequence
// words.
__host__ __device__ inline int group_smem_bytes(int rm, int re, int ring_w, int mode, int seq_cap, int gw) {
  const int ns = ring_slots(rm, re);
  int b = 3 * ns * 4 + (gw > 1 ? 16 * gw * 4 : 0) + 16;
  if (mode == kModeShared) {
    b += ((ns * ring_w * 2 + 15) & ~15) + seq_cap * 4;
  }
  return (b + 15) & ~15;
}

__device__ __forceinline__ bool in_bounds(int32_t off, int k, int m, int n) {
  return (uint32_t)off <= (uint32_t)n && (uint32_t)(off - k) <= (uint32_t)m;
}

// Reduced-unit upper bound of the optimal score: all mismatches plus the
// length difference as one gap, or one gap per sequence.
__device__ __forceinline__ int64_t score_bound(int m, int n, int x, int go, int ge) {
  const int mn = m < n ? m : n;
  const int d = m > n ? m - n : n - m;
  const int64_t a = (int64_t)x * mn + (d ? (int64_t)(go - ge) + (int64_t)ge * d : 0);
  const int64_t b = (m ? (int64_t)(go - ge) + (int64_t)ge * m : 0) + (n ? (int64_t)(go - ge) + (int64_t)ge * n : 0);
  return a < b ? a : b;
}

}  // namespace tsu
