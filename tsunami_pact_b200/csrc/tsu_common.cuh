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
// dual gap-affine backtrace word: bits 31..8 pre-extension M offset, 2..0 M
// source (kSrcMis, kSrcIns, kSrcDel, kSrcIns2, kSrcDel2), then one extension
// bit per gap component
enum : uint32_t { kSrcIns2 = 3, kSrcDel2 = 4, kI1Ext2 = 8, kD1Ext2 = 16, kI2Ext2 = 32, kD2Ext2 = 64 };
constexpr int kDualMaxLen = (1 << 24) - 2;  // offsets of the dual backtrace word
enum : uint32_t { kOpM = 0, kOpI = 1, kOpD = 2, kOpX = 8 };
// align kernel variants: ring mode; penalty model (gap-affine; dual
// gap-affine; gap-linear, which edit and indel distance are cases of)
enum : int { kModeShared = 0, kModeGlobal = 1 };
enum : int { kModelAffine = 0, kModelDual = 1, kModelLinear = 2 };
// added to a model: the low-memory (checkpointed history) variant of its
// CIGAR kernels
enum : int { kLowMemFlag = 8 };

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

// Penalties in score units g = gcd of all penalties, and the depths of the
// wavefront ring: rm M slots (the scores s - x, s - o - e, s - o2 - e2 back),
// re slots of I1 and of D1 (s - e back) and, for dual gap-affine, re2 slots
// of I2 and of D2.  go = o + e (a gap of length L costs go + ge (L - 1)).
// One piece: go2 = ge2 = re2 = 0.  Gap-linear (a gap costs ge per base): go =
// ge and no I/D components (re = re2 = 0).
struct Pen {
  int x = 0, go = 0, ge = 0, go2 = 0, ge2 = 0;
  int rm = 0, re = 0, re2 = 0;
  __host__ __device__ bool dual() const { return re2 > 0; }
  __host__ __device__ bool linear() const { return re == 0; }
  __host__ __device__ int model() const { return linear() ? kModelLinear : (dual() ? kModelDual : kModelAffine); }
  __host__ __device__ int slots() const { return rm + 2 * re + 2 * re2; }
  // cheapest and dearest single-base edit (a one-base gap costs
  // min(go, go2)), smallest extension
  __host__ __device__ int min_pen() const {
    const int a = x < go ? x : go;
    return dual() && go2 < a ? go2 : a;
  }
  __host__ __device__ int max_pen() const {
    const int g1 = dual() && go2 < go ? go2 : go;
    return x > g1 ? x : g1;
  }
  // deepest M source: max(x, go, go2) scores back
  __host__ __device__ int ring_depth() const {
    const int a = x > go ? x : go;
    return dual() && go2 > a ? go2 : a;
  }
  __host__ __device__ int min_ge() const { return dual() && ge2 < ge ? ge2 : ge; }
  // cost of one gap of length L >= 1
  __host__ __device__ int64_t gap(int64_t L) const {
    const int64_t a = (int64_t)go + (int64_t)ge * (L - 1);
    if (!dual()) return a;
    const int64_t b = (int64_t)go2 + (int64_t)ge2 * (L - 1);
    return a < b ? a : b;
  }
};

inline int gcd_int(int a, int b) {
  while (b) {
    const int t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// Reduce raw penalties (mismatch, open, extend; open2 / ext2 < 0: one piece)
// to score units; *g receives the unit.
inline Pen reduce_penalties(int mismatch, int open, int ext, int open2, int ext2, int* g) {
  const bool dual = open2 >= 0 && ext2 > 0;
  int u = gcd_int(gcd_int(mismatch, open), ext);
  if (dual) u = gcd_int(gcd_int(u, open2), ext2);
  Pen p;
  p.x = mismatch / u;
  p.go = (open + ext) / u;
  p.ge = ext / u;
  if (dual) {
    p.go2 = (open2 + ext2) / u;
    p.ge2 = ext2 / u;
  }
  p.re = p.ge + 1;
  p.re2 = dual ? p.ge2 + 1 : 0;
  p.rm = p.ring_depth() + 1;
  if (g) *g = u;
  return p;
}

// Gap-linear penalties (mismatch, per-base gap) in score units.
inline Pen reduce_linear(int mismatch, int ext, int* g) {
  const int u = gcd_int(mismatch, ext);
  Pen p;
  p.x = mismatch / u;
  p.go = p.ge = ext / u;
  p.re = p.re2 = 0;
  p.rm = p.ring_depth() + 1;
  if (g) *g = u;
  return p;
}

struct AlignArgs {
  SeqView seq;
  PackView pk;
  const int32_t* order;  // pairs of this launch (nullptr: 0..n_order-1)
  int64_t n_order;
  Pen pen;               // reduced penalties and ring depths
  int g;                 // score unit
  int ring_w;            // diagonals per ring slot
  int seq_cap;           // shared-memory sequence words (uint32) per group (global mode: 0 = not staged)
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
  unsigned long long* work;  // [3]: wavefront cells computed, score steps, bases matched by extend steps
  // free ends (all 0: end-to-end): starts (v, 0), v <= ef_pb, and (0, h),
  // h <= ef_tb, cost nothing, and so do ends (m, h), h >= n - ef_te, and
  // (v, n), v >= m - ef_pe
  int32_t ef_pb, ef_pe, ef_tb, ef_te;
  // low-memory mode (ckpt_k > 0): checkpoints every ckpt_k scores, ckpt_cap
  // of ckpt_bytes each per group (ckpt_stride bytes apart); the history then
  // holds one segment of ckpt_k scores
  uint8_t* ckpt;
  int64_t ckpt_stride;
  int32_t ckpt_bytes, ckpt_cap, ckpt_k;
};

// Bytes of one low-memory checkpoint: limits (3 ints per slot), then the
// ring's values (ring_w per slot) in the ring's element type.
__host__ __device__ inline int64_t ckpt_bytes_for(const Pen& p, int ring_w, int mode) {
  const int64_t b = 12 * (int64_t)p.slots() + (int64_t)p.slots() * ring_w * (mode == kModeShared ? 2 : 4);
  return (b + 15) & ~(int64_t)15;
}

// Warp partials per warp and step parity: 7 (one piece) or 11 values.
__host__ __device__ inline int partial_words(const Pen& p) { return p.dual() ? 16 : 8; }

// Shared memory per group of gw warps, in bytes: slot limits (lo, hi, alo
// per slot), warp partials [2][gw][partial_words] (gw > 1), 4 broadcast
// words, then in shared mode an int16 ring of slots * ring_w and seq_cap
// sequence words; in global mode with seq_cap > 0, at the next 16-byte
// boundary, 16 reserved bytes and seq_cap sequence words.
__host__ __device__ inline int group_smem_bytes(const Pen& p, int ring_w, int mode, int seq_cap, int gw) {
  const int ns = p.slots();
  int b = 3 * ns * 4 + (gw > 1 ? 2 * partial_words(p) * gw * 4 : 0) + 16;
  if (mode == kModeShared) {
    b += ((ns * ring_w * 2 + 15) & ~15) + seq_cap * 4;
  } else if (seq_cap > 0) {
    b = ((b + 15) & ~15) + 16 + seq_cap * 4;
  }
  return (b + 15) & ~15;
}

// Packed 64-bit words allocated per sequence of len bases: ceil(len / 32)
// data words and a zero padding word (read by the unaligned window loads),
// rounded up to an even count so that every sequence starts on a 16-byte
// boundary (what a bulk copy needs).
__host__ __device__ __forceinline__ int64_t packed_words(int64_t len) { return ((len + 31) / 32 + 2) & ~(int64_t)1; }

__device__ __forceinline__ bool in_bounds(int32_t off, int k, int m, int n) {
  return (uint32_t)off <= (uint32_t)n && (uint32_t)(off - k) <= (uint32_t)m;
}
// The same test without a short-circuit, for select-based code.
__device__ __forceinline__ bool in_bounds_sel(int32_t off, int k, int m, int n) {
  return ((uint32_t)off <= (uint32_t)n) & ((uint32_t)(off - k) <= (uint32_t)m);
}

// Reduced-unit upper bound of the optimal score: all mismatches plus the
// length difference as one gap, or one gap per sequence.
__host__ __device__ __forceinline__ int64_t score_bound(int m, int n, const Pen& p) {
  const int mn = m < n ? m : n;
  const int d = m > n ? m - n : n - m;
  const int64_t a = (int64_t)p.x * mn + (d ? p.gap(d) : 0);
  const int64_t b = (m ? p.gap(m) : 0) + (n ? p.gap(n) : 0);
  return a < b ? a : b;
}

}  // namespace tsu
