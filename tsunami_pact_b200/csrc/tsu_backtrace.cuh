// tsu_backtrace.cuh -- CIGAR backtrace from the per-(score, diagonal) words.
//
// The reference computes no CIGAR (its backtrace types are declared but
// unused, common.h:17-31,48-49,67-77); its check takes CIGARs from WFA2-lib
// (wfa_gpu.cu:164).  This walk restates the WFA2 wavefront backtrace: in M,
// first the matches down to the pre-extension offset, then one operation
// chosen by the source bits stored at compute time, whose tie order is the
// piggyback order of the reference's bt_type_t codes (mismatch 9 > D_ext 6 >
// D_open 5 > I_ext 2 > I_open 1).  Runs are written backwards, one uint32 per
// run ((len << 4) | op), ending at out_end.
#pragma once

#include "tsu_common.cuh"

namespace tsu {

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

// A walk in progress: the position (s, k, offset), the component being
// walked (0 = M; the one-piece walk uses 1 = I, 2 = D, the dual walk the
// M-source codes of its word), and the runs written so far.  The walk runs
// in pieces when the history is recomputed segment by segment (low-memory
// mode): walk_*_run stops once the score falls to s_min or below.
struct Walk {
  RunWriter w;
  uint32_t state;
  int s, k;
  int32_t off;
  int v, h;
  int guard;
};

// The walk starts on the end diagonal k_end (n - m end-to-end; with free
// ends the diagonal the kernel found), at offset min(n, m + k_end): the text
// or the pattern is consumed there, and the rest of the other is the free
// trailing gap, written first.
static __device__ __forceinline__ void walk_begin(Walk& wk, int s_end, int k_end, int m, int n, uint32_t* out_end,
                                                  int cap) {
  wk.w = RunWriter{out_end, 0, cap, 0xffffffffu, 0};
  wk.state = 0;
  wk.s = s_end;
  wk.k = k_end;
  wk.off = min(n, m + k_end);
  wk.v = wk.off - wk.k;
  wk.h = wk.off;
  wk.guard = 4 * (m + n) + 8;
  wk.w.put(kOpD, m - wk.v);
  wk.w.put(kOpI, n - wk.h);
}

// Whether the walk reached the start (nothing left but matches and the free
// leading gap).
static __device__ __forceinline__ bool walk_done(const Walk& wk) { return !(wk.v > 0 && wk.h > 0 && wk.s > 0); }

// The leading matches and free leading gap; the number of runs, or -1.
static __device__ __forceinline__ int walk_finish(Walk& wk) {
  if (wk.v > 0 && wk.h > 0) {
    const int nm = wk.v < wk.h ? wk.v : wk.h;
    wk.w.put(kOpM, nm);
    wk.v -= nm;
    wk.h -= nm;
  }
  wk.w.put(kOpD, wk.v);
  wk.w.put(kOpI, wk.h);
  wk.w.flush();
  return wk.w.cnt <= wk.w.cap ? wk.w.cnt : -1;
}

// One-piece (and gap-linear) walk down to score s_min.  0, or -1 on an
// inconsistency (a word outside the history, a predecessor beyond the
// current offset, a negative score).
static __device__ int walk_run(Walk& wk, const uint32_t* __restrict__ hist, int64_t hist_used,
                               const int2* __restrict__ table, int s_min, int x, int go, int ge) {
  enum { M = 0, I = 1, D = 2 };
  uint32_t state = wk.state;
  int s = wk.s, k = wk.k, v = wk.v, h = wk.h, guard = wk.guard;
  int32_t off = wk.off;
  RunWriter& w = wk.w;
  int rc = 0;
  while (v > 0 && h > 0 && s > s_min) {
    if (--guard < 0) { rc = -1; break; }
    const int2 te = table[s];
    const int64_t hidx = (int64_t)te.y + (k - te.x);
    if (k < te.x || hidx >= hist_used) { rc = -1; break; }  // never on a valid path
    const uint32_t word = hist[hidx];
    if (state == M) {
      const int32_t p = (int32_t)(word >> 4);
      if (p > off) { rc = -1; break; }
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
    if (s < 0) { rc = -1; break; }
  }
  wk.state = state;
  wk.s = s;
  wk.k = k;
  wk.off = off;
  wk.v = v;
  wk.h = h;
  wk.guard = guard;
  return rc;
}

// Dual gap-affine walk over words of the kModelDual kernel: five states (M,
// I1, D1, I2, D2); in M the 3-bit source picks the component, whose
// extension bit (kI1Ext2 ... kD2Ext2) then says open (back to M,
// s - o_j - e_j) or extend (stay, s - e_j).  Same conventions as walk_run.
static __device__ int walk_run_dual(Walk& wk, const uint32_t* __restrict__ hist, int64_t hist_used,
                                    const int2* __restrict__ table, int s_min, const Pen& pen) {
  uint32_t state = wk.state;  // M-source code of the component being walked (kSrcMis for M)
  int s = wk.s, k = wk.k, v = wk.v, h = wk.h, guard = wk.guard;
  int32_t off = wk.off;
  RunWriter& w = wk.w;
  int rc = 0;
  while (v > 0 && h > 0 && s > s_min) {
    if (--guard < 0) { rc = -1; break; }
    const int2 te = table[s];
    const int64_t hidx = (int64_t)te.y + (k - te.x);
    if (k < te.x || hidx >= hist_used) { rc = -1; break; }  // never on a valid path
    const uint32_t word = hist[hidx];
    uint32_t comp = state;
    if (state == kSrcMis) {
      const int32_t p = (int32_t)(word >> 8);
      if (p > off) { rc = -1; break; }
      w.put(kOpM, off - p);
      off = p;
      v = off - k;
      h = off;
      if (v <= 0 || h <= 0) break;
      comp = word & 7u;
      if (comp == kSrcMis) {
        w.put(kOpX, 1);
        s -= pen.x;
        --off;
        v = off - k;
        h = off;
        if (s < 0) { rc = -1; break; }
        continue;
      }
    }
    bool ext, ins;
    int go, ge;
    switch (comp) {
      case kSrcIns: ext = word & kI1Ext2; ins = true; go = pen.go; ge = pen.ge; break;
      case kSrcDel: ext = word & kD1Ext2; ins = false; go = pen.go; ge = pen.ge; break;
      case kSrcIns2: ext = word & kI2Ext2; ins = true; go = pen.go2; ge = pen.ge2; break;
      case kSrcDel2: ext = word & kD2Ext2; ins = false; go = pen.go2; ge = pen.ge2; break;
      default: ext = ins = false; go = ge = 0; rc = -1; break;
    }
    if (rc) break;
    if (ins) {
      w.put(kOpI, 1);
      --k;
      --off;
    } else {
      w.put(kOpD, 1);
      ++k;
    }
    if (ext) {
      s -= ge;
      state = comp;
    } else {
      s -= go;
      state = kSrcMis;
    }
    v = off - k;
    h = off;
    if (s < 0) { rc = -1; break; }
  }
  wk.state = state;
  wk.s = s;
  wk.k = k;
  wk.off = off;
  wk.v = v;
  wk.h = h;
  wk.guard = guard;
  return rc;
}

// The whole walk at once (history of every score in memory).  Returns the
// number of runs (written backwards, ending at out_end), or -1.
static __device__ int backtrace_walk(const uint32_t* __restrict__ hist, int64_t hist_used, const int2* __restrict__ table,
                                     int s_end, int k_end, int m, int n, int x, int go, int ge, uint32_t* out_end,
                                     int cap) {
  Walk wk;
  walk_begin(wk, s_end, k_end, m, n, out_end, cap);
  if (walk_run(wk, hist, hist_used, table, 0, x, go, ge)) return -1;
  return walk_finish(wk);
}

static __device__ int backtrace_walk_dual(const uint32_t* __restrict__ hist, int64_t hist_used,
                                          const int2* __restrict__ table, int s_end, int k_end, int m, int n,
                                          const Pen& pen, uint32_t* out_end, int cap) {
  Walk wk;
  walk_begin(wk, s_end, k_end, m, n, out_end, cap);
  if (walk_run_dual(wk, hist, hist_used, table, 0, pen)) return -1;
  return walk_finish(wk);
}

}  // namespace tsu
