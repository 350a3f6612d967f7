// tsu_kernels.cuh -- sm_100a kernels of the gap-affine WFA engine.
//
// Path (reference wfa_gpu.cu:191-752 re-designed):
//   pack_kernel     ASCII -> 2-bit codes, 32 bases per uint64 word
//                   (the reference compares raw bytes, wfa_gpu.cu:735).
//   align_kernel    persistent: each warp pulls pairs from a device work
//                   queue and runs score steps s = 0, 1, ... (in units of
//                   gcd(x, o, e)).  One fused pass per step computes the
//                   I/D/M wavefronts of score s (wfa_gpu.cu:610-631), extends
//                   M along its diagonal with XOR + find-first-set on 2-bit
//                   words (replaces count_chars, wfa_gpu.cu:724-752), trims
//                   the ends with warp min/max reductions
//                   (wfa_gpu.cu:636-719), detects the end point
//                   (wfa_gpu.cu:288-338) and, when a CIGAR is wanted,
//                   streams one 32-bit backtrace word per (score, diagonal)
//                   to HBM.  The wavefront ring of the last max(x, o+e)+1
//                   scores lives in shared memory (global memory when a pair
//                   is too wide for the shared-memory slots).
//                   After the end is reached, lane 0 walks the backtrace
//                   words and writes run-length CIGAR runs into an arena.
//   compact_kernel  gathers per-pair CIGAR runs into pair order.
//
// Backtrace word: bits 31..4 = pre-extension M offset P, bits 1..0 = M
// source (0 mismatch, 1 insertion, 2 deletion), bit 2 = I from I (gap
// extension) rather than M (open), bit 3 = D from D rather than M.  Ties are
// resolved in the order of the piggyback codes the reference copies from
// WFA2-lib (common.h:67-77): mismatch > D_ext > D_open > I_ext > I_open.
#pragma once

#include <cstdint>
#include <climits>

namespace tsu {

constexpr int32_t kNull = INT32_MIN / 2;  // offset null (reference: INT16_MIN/2, common.h:6)

enum : int32_t { kPairOk = 0, kPairScratch = 1, kPairArena = 2, kPairInternal = 3 };
enum : uint32_t { kSrcMis = 0, kSrcIns = 1, kSrcDel = 2, kIExt = 4, kDExt = 8 };
enum : uint32_t { kOpM = 0, kOpI = 1, kOpD = 2, kOpX = 8 };

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
  uint64_t* words;        // packed 2-bit words
  const int64_t* woff;    // [2n]: pattern i at i, text i at n + i
  uint8_t* nonacgt;       // [2n]: 1 if the sequence holds a byte outside ACGT
};

struct AlignArgs {
  SeqView seq;
  PackView pk;
  const int32_t* order;  // pairs of this launch (nullptr: 0..n_order-1)
  int64_t n_order;
  int x, go, ge, g;      // reduced mismatch, open+extend, extend; gcd
  int rm, re;            // ring depths: rm = max(x, go) + 1, re = ge + 1
  int ring_w;            // diagonals per ring slot
  int smem_ring;         // 1: ring in shared memory, 0: ring_global
  int32_t* ring_global;  // per-warp rings when !smem_ring
  int64_t ring_stride;   // int32 per warp in ring_global
  uint32_t* hist;        // per-warp backtrace words
  int64_t hist_cap;
  int2* table;           // per-warp step table: (lo, base) per score
  int32_t table_cap;
  int want_cigar;
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
// Shared memory per warp, in int32 units: 3 metadata arrays + ring (opt.)
__host__ __device__ inline int warp_smem_ints(int rm, int re, int ring_w, int smem_ring) {
  int ns = ring_slots(rm, re);
  int v = 3 * ns + (smem_ring ? ns * ring_w : 0);
  return (v + 3) & ~3;
}

// ---------------------------------------------------------------------------
// Packing.  One warp per sequence; lane l of iteration j looks at byte
// 32*j + l, so each warp load instruction touches 32 consecutive bytes.  The
// 2-bit code of a base is (c >> 1) & 3 (A=0, C=1, T=2, G=3), a bijection on
// "ACGT"; any other byte marks the sequence for the byte-compare path.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t spread32(uint32_t v) {
  uint64_t x = v;
  x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
  x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
  x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

__global__ void pack_kernel(SeqView sv, PackView pk) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t nseq = 2 * sv.n;
  for (int64_t j = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); j < nseq; j += warps) {
    const bool is_pat = j < sv.n;
    const int64_t i = is_pat ? j : j - sv.n;
    const uint8_t* src = is_pat ? sv.pat + sv.pat_off[i] : sv.txt + sv.txt_off[i];
    const int len = is_pat ? sv.pat_len[i] : sv.txt_len[i];
    uint64_t* dst = pk.words + pk.woff[j];
    const int nw = (len + 31) >> 5;
    unsigned bad = 0;
    for (int w = 0; w < nw; ++w) {
      const int p = (w << 5) + lane;
      uint32_t c = 0x41;  // 'A' beyond the end (masked by lengths later)
      if (p < len) c = src[p];
      const uint32_t code = (c >> 1) & 3u;
      const bool ok = (c == 0x41u) | (c == 0x43u) | (c == 0x47u) | (c == 0x54u);
      bad |= __ballot_sync(0xffffffffu, !ok);
      const uint32_t b0 = __ballot_sync(0xffffffffu, code & 1u);
      const uint32_t b1 = __ballot_sync(0xffffffffu, (code >> 1) & 1u);
      if (lane == 0) dst[w] = spread32(b0) | (spread32(b1) << 1);
    }
    if (lane == 0) {
      dst[nw] = 0;  // padding word read by the unaligned window loads
      pk.nonacgt[j] = bad ? 1 : 0;
    }
  }
}

// ---------------------------------------------------------------------------
// Extension (longest common prefix along a diagonal).
// ---------------------------------------------------------------------------
// 32 bases starting at base `pos` of a packed sequence: two aligned words
// and a funnel shift.  pos < len is guaranteed by the caller, so the second
// word is at most the padding word.
__device__ __forceinline__ uint64_t win2(const uint64_t* __restrict__ w, int pos) {
  const int wi = pos >> 5;
  const int sh = (pos & 31) << 1;
  const uint64_t lo = __ldg(w + wi);
  const uint64_t hi = __ldg(w + wi + 1);
  return (lo >> sh) | ((hi << 1) << (63 - sh));
}

__device__ __forceinline__ int lcp2(const uint64_t* __restrict__ pw, int v, const uint64_t* __restrict__ tw, int h,
                                    int rem) {
  int l = 0;
  while (l < rem) {
    const uint64_t d = win2(pw, v + l) ^ win2(tw, h + l);
    if (d) {
      l += (__ffsll((long long)d) - 1) >> 1;
      break;
    }
    l += 32;
  }
  return l < rem ? l : rem;
}

// Byte path for pairs with bytes outside ACGT: bounded byte loads, 8 per
// window (no reads outside the caller's sequences).
__device__ __forceinline__ uint64_t win8(const uint8_t* __restrict__ s, int len, int pos) {
  uint64_t r = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int p = pos + i;
    const uint64_t c = p < len ? (uint64_t)s[p] : 0ull;
    r |= c << (8 * i);
  }
  return r;
}

__device__ __forceinline__ int lcp8(const uint8_t* __restrict__ p, int m, int v, const uint8_t* __restrict__ t, int n,
                                    int h, int rem) {
  int l = 0;
  while (l < rem) {
    const uint64_t d = win8(p, m, v + l) ^ win8(t, n, h + l);
    if (d) {
      l += (__ffsll((long long)d) - 1) >> 3;
      break;
    }
    l += 8;
  }
  return l < rem ? l : rem;
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

// ---------------------------------------------------------------------------
// Backtrace (lane 0).  Walks the per-(score, diagonal) words from the end
// point and writes run-length runs backwards ending at out_end.  Restates
// the WFA2 wavefront backtrace the reference's check relies on
// (wfa_gpu.cu:164): in M, first the matches down to the pre-extension
// offset, then one operation chosen by the stored source bits.
// Returns the number of runs, or -1 on an internal inconsistency.
// ---------------------------------------------------------------------------
struct RunWriter {
  uint32_t* end;
  int cnt, cap;
  uint32_t op;
  int64_t len;
  __device__ __forceinline__ void put(uint32_t o, int64_t l) {
    if (l <= 0) return;
    if (o == op) {
      len += l;
      return;
    }
    flush();
    op = o;
    len = l;
  }
  __device__ __forceinline__ void flush() {
    if (len > 0) {
      if (cnt < cap) end[-1 - cnt] = ((uint32_t)len << 4) | op;
      ++cnt;
    }
    len = 0;
  }
};

__device__ int backtrace_walk(const uint32_t* __restrict__ hist, int64_t hist_used, const int2* __restrict__ table,
                              int s_end, int m, int n, int x, int go, int ge, uint32_t* out_end, int cap) {
  RunWriter w{out_end, 0, cap, 0xffffffffu, 0};
  enum { M = 0, I = 1, D = 2 };
  int state = M, s = s_end, k = n - m;
  int32_t off = n;
  int v = off - k, h = off;
  int guard = 4 * (m + n) + 8;
  while (v > 0 && h > 0 && s > 0) {
    if (--guard < 0) return -1;
    const int2 te = table[s];
    const int64_t hidx = (int64_t)te.y + (k - te.x);
    if (k < te.x || hidx >= hist_used) return -1;  // never on a valid path
    const uint32_t word = hist[hidx];
    if (state == M) {
      const int32_t p = (int32_t)(word >> 4);
      if (p > off) return -1;
      w.put(kOpM, off - p);
      off = p;
      v = off - k;
      h = off;
      if (v <= 0 || h <= 0) break;
      const uint32_t src = word & 3u;
      if (src == kSrcMis) {
        w.put(kOpX, 1);
        s -= x;
        --off;
      } else if (src == kSrcIns) {
        w.put(kOpI, 1);
        if (word & kIExt) {
          s -= ge;
          state = I;
        } else {
          s -= go;
        }
        --k;
        --off;
      } else {
        w.put(kOpD, 1);
        if (word & kDExt) {
          s -= ge;
          state = D;
        } else {
          s -= go;
        }
        ++k;
      }
    } else if (state == I) {
      w.put(kOpI, 1);
      if (word & kIExt) {
        s -= ge;
      } else {
        s -= go;
        state = M;
      }
      --k;
      --off;
    } else {
      w.put(kOpD, 1);
      if (word & kDExt) {
        s -= ge;
      } else {
        s -= go;
        state = M;
      }
      ++k;
    }
    v = off - k;
    h = off;
    if (s < 0) return -1;
  }
  if (v > 0 && h > 0) {
    const int nm = v < h ? v : h;
    w.put(kOpM, nm);
    v -= nm;
    h -= nm;
  }
  w.put(kOpD, v);
  w.put(kOpI, h);
  w.flush();
  return w.cnt <= cap ? w.cnt : -1;
}

// ---------------------------------------------------------------------------
// The aligner.  kCigar selects whether backtrace words are written.
// ---------------------------------------------------------------------------
template <bool kCigar>
__global__ void __launch_bounds__(128) align_kernel(AlignArgs a) {
  extern __shared__ int4 smem_raw[];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int64_t gwarp = (int64_t)blockIdx.x * wpb + wib;
  const int ns = ring_slots(a.rm, a.re);
  int* wsm = reinterpret_cast<int*>(smem_raw) + (size_t)wib * warp_smem_ints(a.rm, a.re, a.ring_w, a.smem_ring);
  int* s_lo = wsm;
  int* s_hi = wsm + ns;
  int* s_alo = wsm + 2 * ns;
  int32_t* ring = a.smem_ring ? (int32_t*)(wsm + 3 * ns) : (a.ring_global + gwarp * a.ring_stride);
  uint32_t* hist = a.hist + gwarp * a.hist_cap;
  int2* table = a.table + gwarp * (int64_t)a.table_cap;
  const int W = a.ring_w;

  for (;;) {
    unsigned qi = 0;
    if (lane == 0) qi = atomicAdd(a.queue, 1u);
    qi = __shfl_sync(FULL, qi, 0);
    if ((int64_t)qi >= a.n_order) break;
    const int64_t pair = a.order ? a.order[qi] : (int64_t)qi;
    const int m = a.seq.pat_len[pair];
    const int n = a.seq.txt_len[pair];
    const bool bytemode = a.pk.nonacgt[pair] | a.pk.nonacgt[a.seq.n + pair];
    const uint64_t* pw = a.pk.words + a.pk.woff[pair];
    const uint64_t* tw = a.pk.words + a.pk.woff[a.seq.n + pair];
    const uint8_t* pb = a.seq.pat + a.seq.pat_off[pair];
    const uint8_t* tb = a.seq.txt + a.seq.txt_off[pair];
    const int k_end = n - m;
    const int64_t s_max = score_bound(m, n, a.x, a.go, a.ge);

    for (int i = lane; i < ns; i += 32) {
      s_lo[i] = 1;
      s_hi[i] = 0;
      s_alo[i] = 0;
    }
    __syncwarp();

    int32_t st = kPairOk;
    int s_end = -1;
    int64_t hbase = 0;
    // ---- score 0: M[0] = {k = 0: offset 0}, extended (wfa_gpu.cu:239-242)
    {
      int32_t o0 = 0;
      if (lane == 0) {
        const int rem = m < n ? m : n;
        o0 = bytemode ? lcp8(pb, m, 0, tb, n, 0, rem) : lcp2(pw, 0, tw, 0, rem);
        ring[0 * W + 0] = o0;
        s_lo[0] = 0;
        s_hi[0] = 0;
        s_alo[0] = 0;
        if (kCigar) {
          table[0] = make_int2(0, 0);
          hist[0] = 0u;
        }
      }
      o0 = __shfl_sync(FULL, o0, 0);
      hbase = 1;
      if (k_end == 0 && o0 >= n) s_end = 0;
      __syncwarp();
    }

    int s = 0;
    int slm = 0, sli = 0;  // s mod rm, s mod re
    unsigned long long n_cells = 1, n_steps = 1;
    while (s_end < 0) {
      ++s;
      if (++slm == a.rm) slm = 0;
      if (++sli == a.re) sli = 0;
      if (s > s_max) {  // the end is reachable at s_max: inconsistency
        st = kPairInternal;
        break;
      }
      // source slots
      const int sm = s - a.x, so = s - a.go, se = s - a.ge;
      int q;
      q = slm - a.x;
      if (q < 0) q += a.rm;
      const int slot_mm = q;
      q = slm - a.go;
      if (q < 0) q += a.rm;
      const int slot_mo = q;
      q = sli - a.ge;
      if (q < 0) q += a.re;
      const int slot_ie = a.rm + q;
      const int slot_de = a.rm + a.re + q;
      const int lo_mm = sm >= 0 ? s_lo[slot_mm] : 1, hi_mm = sm >= 0 ? s_hi[slot_mm] : 0;
      const int lo_mo = so >= 0 ? s_lo[slot_mo] : 1, hi_mo = so >= 0 ? s_hi[slot_mo] : 0;
      const int lo_ie = se >= 0 ? s_lo[slot_ie] : 1, hi_ie = se >= 0 ? s_hi[slot_ie] : 0;
      const int lo_de = se >= 0 ? s_lo[slot_de] : 1, hi_de = se >= 0 ? s_hi[slot_de] : 0;
      const bool nmm = lo_mm > hi_mm, nmo = lo_mo > hi_mo, nie = lo_ie > hi_ie, nde = lo_de > hi_de;
      const int out_m = slm, out_i = a.rm + sli, out_d = a.rm + a.re + sli;
      if (nmm && nmo && nie && nde) {  // null step (wfa_gpu.cu:417-422)
        __syncwarp();
        if (lane == 0) {
          s_lo[out_m] = 1; s_hi[out_m] = 0;
          s_lo[out_i] = 1; s_hi[out_i] = 0;
          s_lo[out_d] = 1; s_hi[out_d] = 0;
        }
        __syncwarp();
        continue;
      }
      int lo = INT_MAX, hi = INT_MIN;  // wfa_gpu.cu:429-439
      if (!nmm) { lo = lo_mm; hi = hi_mm; }
      if (!nmo) { lo = min(lo, lo_mo - 1); hi = max(hi, hi_mo + 1); }
      if (!nie) { lo = min(lo, lo_ie + 1); hi = max(hi, hi_ie + 1); }
      if (!nde) { lo = min(lo, lo_de - 1); hi = max(hi, hi_de - 1); }
      const int width = hi - lo + 1;
      const bool i_present = !nmo || !nie;
      const bool d_present = !nmo || !nde;
      if (width > W || (kCigar && (s >= a.table_cap || hbase + width > a.hist_cap))) {
        st = kPairScratch;
        break;
      }
      const int32_t* rmm = ring + slot_mm * W;
      const int32_t* rmo = ring + slot_mo * W;
      const int32_t* rie = ring + slot_ie * W;
      const int32_t* rde = ring + slot_de * W;
      const int alo_mm = s_alo[slot_mm], alo_mo = s_alo[slot_mo];
      const int alo_ie = s_alo[slot_ie], alo_de = s_alo[slot_de];
      int32_t* wm = ring + out_m * W;
      int32_t* wi = ring + out_i * W;
      int32_t* wd = ring + out_d * W;
      uint32_t* hrow = hist + hbase;
      int mn_m = INT_MAX, mx_m = INT_MIN, mn_i = INT_MAX, mx_i = INT_MIN, mn_d = INT_MAX, mx_d = INT_MIN;
      bool found = false;
      for (int k = lo + lane; k <= hi; k += 32) {
        const int32_t ins_o = (k - 1 >= lo_mo && k - 1 <= hi_mo) ? rmo[k - 1 - alo_mo] : kNull;
        const int32_t ins_e = (k - 1 >= lo_ie && k - 1 <= hi_ie) ? rie[k - 1 - alo_ie] : kNull;
        const int32_t del_o = (k + 1 >= lo_mo && k + 1 <= hi_mo) ? rmo[k + 1 - alo_mo] : kNull;
        const int32_t del_e = (k + 1 >= lo_de && k + 1 <= hi_de) ? rde[k + 1 - alo_de] : kNull;
        const int32_t mis = ((k >= lo_mm && k <= hi_mm) ? rmm[k - alo_mm] : kNull) + 1;
        const int32_t ins = max(ins_o, ins_e) + 1;
        const int32_t del = max(del_o, del_e);
        int32_t p = ins;
        uint32_t src = kSrcIns;
        if (del >= p) { p = del; src = kSrcDel; }
        if (mis >= p) { p = mis; src = kSrcMis; }
        uint32_t bits = src;
        if (ins_e >= ins_o) bits |= kIExt;
        if (del_e >= del_o) bits |= kDExt;
        int32_t om = kNull;
        if (in_bounds(p, k, m, n)) {
          const int vv = p - k;
          const int rem = min(m - vv, n - p);
          const int l = bytemode ? lcp8(pb, m, vv, tb, n, p, rem) : lcp2(pw, vv, tw, p, rem);
          om = p + l;
          mn_m = min(mn_m, k);
          mx_m = max(mx_m, k);
          if (k == k_end && om >= n) found = true;
        }
        wm[k - lo] = om;
        if (i_present) {
          wi[k - lo] = ins;
          if (in_bounds(ins, k, m, n)) { mn_i = min(mn_i, k); mx_i = max(mx_i, k); }
        }
        if (d_present) {
          wd[k - lo] = del;
          if (in_bounds(del, k, m, n)) { mn_d = min(mn_d, k); mx_d = max(mx_d, k); }
        }
        if (kCigar) hrow[k - lo] = ((uint32_t)p << 4) | bits;
      }
      mn_m = __reduce_min_sync(FULL, mn_m);
      mx_m = __reduce_max_sync(FULL, mx_m);
      mn_i = __reduce_min_sync(FULL, mn_i);
      mx_i = __reduce_max_sync(FULL, mx_i);
      mn_d = __reduce_min_sync(FULL, mn_d);
      mx_d = __reduce_max_sync(FULL, mx_d);
      const bool any_found = __any_sync(FULL, found);
      if (lane == 0) {
        // trimmed limits (wfa_gpu.cu:636-719); empty => null
        s_lo[out_m] = mn_m; s_hi[out_m] = mx_m; s_alo[out_m] = lo;
        if (i_present) { s_lo[out_i] = mn_i; s_hi[out_i] = mx_i; } else { s_lo[out_i] = 1; s_hi[out_i] = 0; }
        s_alo[out_i] = lo;
        if (d_present) { s_lo[out_d] = mn_d; s_hi[out_d] = mx_d; } else { s_lo[out_d] = 1; s_hi[out_d] = 0; }
        s_alo[out_d] = lo;
        if (kCigar) table[s] = make_int2(lo, (int)hbase);
      }
      hbase += width;
      n_cells += (unsigned long long)width;
      ++n_steps;
      __syncwarp();
      if (any_found) s_end = s;
    }
    if (lane == 0 && a.work) {
      atomicAdd(a.work, n_cells);
      atomicAdd(a.work + 1, n_steps);
    }

    if (st == kPairOk) {
      if (lane == 0) a.score[pair] = s_end * a.g;
      if (kCigar) {
        // reserve the run bound 2*s/min_pen + 1 in the arena, then walk
        const int min_pen = min(a.x, a.go);
        const int64_t bound = 2 * (int64_t)s_end / min_pen + 1;
        int32_t len = 0;
        int64_t pos = 0;
        if (lane == 0) {
          const unsigned long long at = atomicAdd(a.arena_cursor, (unsigned long long)bound);
          if ((int64_t)(at + bound) > a.arena_cap) {
            st = kPairArena;
          } else {
            const int r =
                backtrace_walk(hist, hbase, table, s_end, m, n, a.x, a.go, a.ge, a.arena + at + bound, (int)bound);
            if (r < 0) {
              st = kPairInternal;
            } else {
              len = r;
              pos = (int64_t)(at + bound) - r;
            }
          }
          a.cig_pos[pair] = pos;
          a.cig_len[pair] = len;
        }
        st = __shfl_sync(FULL, st, 0);
      }
    }
    if (lane == 0) {
      a.status[pair] = st;
      if (st == kPairScratch || st == kPairArena) {
        const unsigned r = atomicAdd(a.retry_count, 1u);
        a.retry[r] = (int32_t)pair;
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Compaction: pair i's runs arena[cig_pos[i] ..) -> out[out_off[i] ..).
// One warp per pair, grid-stride.
// ---------------------------------------------------------------------------
__global__ void compact_kernel(int64_t n, const uint32_t* __restrict__ arena, const int64_t* __restrict__ cig_pos,
                               const int32_t* __restrict__ cig_len, const int64_t* __restrict__ out_off,
                               uint32_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int64_t src = cig_pos[i];
    const int64_t dst = out_off[i];
    // length from the status-masked scan: a pair that failed in this call
    // contributes 0 even if cig_len holds a stale value
    const int64_t len = out_off[i + 1] - dst;
    for (int64_t j = lane; j < len; j += 32) out[dst + j] = arena[src + j];
  }
}

// words per sequence: ceil(len/32) data words + 1 padding word
__global__ void word_count_kernel(int64_t n, const int32_t* __restrict__ pat_len, const int32_t* __restrict__ txt_len,
                                  int64_t* __restrict__ words) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < 2 * n; j += (int64_t)gridDim.x * blockDim.x) {
    const int len = j < n ? pat_len[j] : txt_len[j - n];
    words[j] = ((int64_t)len + 31) / 32 + 1;
  }
}

// cigar_len as int64 for the scan (negative/failed pairs count 0)
__global__ void cig_len64_kernel(int64_t n, const int32_t* __restrict__ len, const int32_t* __restrict__ status,
                                 int64_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = status[i] == kPairOk ? (int64_t)len[i] : 0;
}

}  // namespace tsu
