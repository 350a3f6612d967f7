// tsu_plan.h -- pass geometry of the align kernel (host only, no CUDA).
//
// Shared by the engine (tsu_engine.cu), the no-allocation entry point
// (tsu_noalloc.cu) and the CPU warp emulation used by the tests, so all run
// the kernel with the same group size, ring width, staging size and scratch
// capacities.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "tsu_common.cuh"
#include "tsu_tuning.h"
#include "tsu_tuning_dual.h"

namespace tsu {

// A rung of the pass ladder: ring mode and warps per pair.
struct PassChoice {
  int mode, gw;
};

struct PassGeom {
  int mode = kModeShared;
  int gw = 1;              // warps per pair
  int cta_threads = 128;   // threads per block
  int groups_per_cta = 4;  // pairs in flight per block
  int min_blocks = 6;      // blocks per SM the kernel is compiled for
  int ring_w = 0;          // diagonals per ring slot
  int seq_cap = 0;         // staged sequence words per group (shared mode)
  int64_t hist_cap = 0;    // backtrace words per group
  int table_cap = 0;       // step-table entries per group
  int group_smem = 0;      // dynamic shared memory per group (bytes)
  int64_t ring_ints = 0;   // global ring int32 per group (global mode)
  int ckpt_k = 0;          // low-memory mode: checkpoint interval (0: off)
  int ckpt_cap = 0;        // checkpoints per group
  int64_t ckpt_bytes = 0;  // bytes per checkpoint
};

constexpr int kSharedW1 = 384;         // shared-mode ring width for one warp per pair (diagonals)
constexpr int kSharedSeqWords1 = 544;  // staging area for one warp per pair (uint32 words)
constexpr int kSharedSeqWordsN = 4096; // staging area for a group of warps
constexpr int kSharedMaxLen = 32000;   // int16 ring limit
// widest int16 ring: a negative (invalid) I value grows by one per diagonal
// of the ring's width and must stay negative (the kernel's store clamp)
constexpr int kSharedMaxW = 16368;
constexpr int kSmemPerSM = 228 * 1024; // B200 shared memory per SM (bytes)

// Reduced-unit score expected at edit rate `hint` for a pair of length L.
inline int64_t hint_score(const Pen& pen, int64_t L, double hint) {
  return (int64_t)(hint * (double)L * (double)pen.max_pen()) + 16;
}

inline int cta_threads_for(int gw) { return gw <= 4 ? 128 : 32 * gw; }
inline int min_blocks_for(int mode, int gw) {
  return mode == kModeShared ? (gw == 1 ? 7 : (gw <= 4 ? 6 : (gw == 8 ? 3 : 1))) : (gw <= 4 ? 4 : (gw == 8 ? 2 : 1));
}

// Ring width a shared-mode group of gw warps can hold with seq_cap staged
// words, at the block count the kernel is compiled for.
inline int shared_ring_width(const Pen& pen, int gw, int seq_cap, int smem_optin) {
  const int ns = pen.slots();
  const int blocks = min_blocks_for(kModeShared, gw);
  const int per_cta = std::min(smem_optin, kSmemPerSM / blocks - 1024);
  const int gpc = cta_threads_for(gw) / (32 * gw);
  const int per_group = per_cta / gpc;
  const int fixed = group_smem_bytes(pen, 0, kModeShared, seq_cap, gw) + 16;
  const int w = std::min((per_group - fixed) / (2 * ns), kSharedMaxW);
  return std::max(0, w & ~15);
}

// Shared ring width of a group of gw warps.  One warp per pair has a fixed
// width (kSharedW1), unless penalties with a very deep ring leave four such
// groups unable to fit one block; then the width one block can hold (below
// 64 diagonals the pass takes the global ring).
inline int shared_cap(const Pen& pen, int gw, int seq_cap, int smem_optin) {
  if (gw != 1) return shared_ring_width(pen, gw, seq_cap, smem_optin);
  const int gpc = cta_threads_for(1) / 32;
  if (gpc * group_smem_bytes(pen, kSharedW1, kModeShared, seq_cap, 1) <= smem_optin) return kSharedW1;
  const int w = (smem_optin / gpc - group_smem_bytes(pen, 0, kModeShared, seq_cap, 1) - 16) / (2 * pen.slots());
  return std::max(0, w & ~15);
}

// mode/gw: the configuration of this pass.  Shared mode needs lengths within
// the int16 ring; otherwise the pass falls back to the global ring.
// low_mem (CIGAR passes): 0 off; > 0 checkpoint every low_mem scores; < 0
// an interval chosen here.
inline PassGeom plan_geometry(const Pen& pen, int32_t max_m, int32_t max_n, int mode, int gw, double hint,
                              bool want_cigar, int smem_optin, int low_mem = 0) {
  PassGeom p;
  const bool lowmem = want_cigar && low_mem != 0;
  const int ns = pen.slots();
  const int ge = pen.min_ge();
  const int64_t maxlen = std::max(max_m, max_n);
  const int64_t s_hint = hint_score(pen, maxlen, hint);
  const int64_t full_w = (int64_t)max_m + max_n + 3;
  const int64_t width_hint = std::min<int64_t>(full_w, 2 * s_hint / ge + 3);
  p.gw = gw;
  p.cta_threads = cta_threads_for(gw);
  p.groups_per_cta = p.cta_threads / (32 * gw);
  p.mode = (mode == kModeShared && maxlen <= kSharedMaxLen) ? kModeShared : kModeGlobal;
  if (p.mode == kModeShared) {
    const int64_t seqw = 2 * packed_words(max_m) + 2 * packed_words(max_n);
    p.seq_cap = (int)std::min<int64_t>(seqw, gw == 1 ? kSharedSeqWords1 : kSharedSeqWordsN);
    const int cap = shared_cap(pen, gw, p.seq_cap, smem_optin);
    p.ring_w = (int)std::max<int64_t>(16, (std::min<int64_t>(full_w, cap) + 15) & ~15);
    if (cap < 64) p.mode = kModeGlobal;
  }
  if (p.mode == kModeGlobal) {
    p.ring_w = (int)full_w;
    // the pair's packed words staged in shared memory when
    // they fit beside the group's limits at the block count the kernel is
    // compiled for (0: read from global memory; always for 32-warp groups)
    const int64_t seqw = 2 * packed_words(max_m) + 2 * packed_words(max_n);
    const int per_cta = std::min(smem_optin, kSmemPerSM / min_blocks_for(kModeGlobal, gw) - 1024);
    const int gpc = cta_threads_for(gw) / (32 * gw);
    const int64_t room = per_cta / gpc - group_smem_bytes(pen, 0, kModeGlobal, 0, gw) - 48;
    p.seq_cap = (gw < 32 && seqw * 4 <= room) ? (int)seqw : 0;
  }
  p.min_blocks = min_blocks_for(p.mode, gw);
  p.group_smem = group_smem_bytes(pen, p.ring_w, p.mode, p.seq_cap, gw);
  // Backtrace words up to score s: sum_j (2j/ge + 1) ~= s^2/ge + 2s.
  p.table_cap = want_cigar ? (int)std::min<int64_t>(s_hint + 1, INT32_MAX / 2) : 0;
  if (want_cigar) {
    const int64_t sq = s_hint * s_hint / ge + 2 * s_hint + 64;
    p.hist_cap = std::min<int64_t>(std::min<int64_t>(sq, (s_hint + 1) * width_hint), INT32_MAX - 64);
  }
  p.ring_ints = p.mode == kModeShared ? 0 : (int64_t)ns * p.ring_w;
  if (lowmem) {
    // The checkpoints of a pair (s_hint / K + 2 of ckpt_bytes) plus one
    // segment of history (K + 1 rows of at most width_hint words): K near
    // sqrt(s_hint * ckpt_bytes / (4 width_hint)) balances the two.  K is at
    // least the ring depth, so a backtrace step crosses one segment at most.
    p.ckpt_bytes = ckpt_bytes_for(pen, p.ring_w, p.mode);
    int64_t K = low_mem;
    if (K < 0) {
      const double k = std::sqrt((double)s_hint * (double)p.ckpt_bytes / (4.0 * (double)std::max<int64_t>(width_hint, 1)));
      K = (int64_t)k;
    }
    K = std::max<int64_t>(std::min<int64_t>(K, std::max<int64_t>(s_hint, 1)), pen.rm);
    p.ckpt_k = (int)K;
    p.ckpt_cap = (int)std::min<int64_t>(s_hint / K + 2, INT32_MAX / 2);
    p.hist_cap = std::min<int64_t>(p.hist_cap, (K + 1) * width_hint + 64);
  }
  return p;
}

// Retry ladder: the configuration of the pass after `prev` for n_pairs pairs
// of at most max_m x max_n that outgrew it.  The smallest group whose shared
// ring holds the widest possible wavefront (m + n + 3 diagonals, so it cannot
// overflow), else the largest shared group, then the global ring with
// global_gw (16) warps per pair (the pairs that reach it are the longest and
// most divergent ones; their count in flight is bounded by memory, not by
// warps).
inline PassChoice next_pass(PassChoice prev, const Pen& pen, int32_t max_m, int32_t max_n, int smem_optin,
                            int global_gw = 16) {
  const int64_t need_w = (int64_t)max_m + max_n + 3;
  if (prev.mode == kModeShared && std::max(max_m, max_n) <= kSharedMaxLen) {
    const int64_t seqw =
        std::min<int64_t>(2 * packed_words(max_m) + 2 * packed_words(max_n), kSharedSeqWordsN);
    static const int kGW[] = {2, 4, 8, 16};
    for (int gw : kGW) {
      if (gw <= prev.gw) continue;
      if (shared_ring_width(pen, gw, (int)seqw, smem_optin) >= need_w) return {kModeShared, gw};
    }
    if (prev.gw < 16) return {kModeShared, 16};
  }
  return {kModeGlobal, global_gw};
}

// The first rung at or above pc whose ring holds the wavefront width the
// hint predicts for pairs of at most max_m x max_n (2 s_hint / e + 3
// diagonals, at most m + n + 3): pc itself, a larger shared group, or the
// global ring with 8 or more warps.  Used when the hint is a per-pair
// estimate, so a pair that is bound to outgrow the shared ring does not
// start there; a wavefront wider than 16,384 diagonals gets 32 warps.
inline PassChoice fit_start(PassChoice pc, const Pen& pen, int32_t max_m, int32_t max_n, double hint,
                            int smem_optin) {
  const int64_t maxlen = std::max(max_m, max_n);
  const int64_t w =
      std::min<int64_t>((int64_t)max_m + max_n + 3, 2 * hint_score(pen, maxlen, hint) / pen.min_ge() + 3);
  if (pc.mode != kModeShared) return {kModeGlobal, w > 16384 ? 32 : pc.gw};
  if (maxlen > kSharedMaxLen) return {kModeGlobal, w > 16384 ? 32 : std::max(8, pc.gw)};
  const int64_t seqw = 2 * packed_words(max_m) + 2 * packed_words(max_n);
  static const int kGW[] = {1, 2, 4, 8, 16};
  for (int gw : kGW) {
    if (gw < pc.gw) continue;
    if (seqw > (gw == 1 ? kSharedSeqWords1 : kSharedSeqWordsN)) continue;
    const int cap = shared_cap(pen, gw, (int)seqw, smem_optin);
    if (cap >= w && cap >= 64) return {kModeShared, gw};
  }
  // wavefronts wider than 16,384 diagonals: 32 warps (one 1024-thread block)
  return {kModeGlobal, w > 16384 ? 32 : std::max(8, pc.gw)};
}

// Length bands of the batched scheduler: max(m, n) < 1024, < 2048, < 4096,
// < 8192, < 16384, >= 16384.  Each band starts its ladder at the rung the
// autotuner measured fastest for it (tsu_tuning.h; the dual gap-affine
// kernels, with their deeper and wider rings: tsu_tuning_dual.h).
constexpr int kBands = 6;
inline int length_band(int32_t L) {
  if (L < 1024) return 0;
  if (L < 2048) return 1;
  if (L < 4096) return 2;
  if (L < 8192) return 3;
  if (L < 16384) return 4;
  return 5;
}
// The starting rung of each band in a table (a context's copy of the
// compiled one), adjusted for lengths beyond the int16 shared ring.
inline PassChoice band_start_in(const PassChoice* table, int band, int32_t maxlen) {
  PassChoice r = table[band < 0 ? 0 : (band >= kBands ? kBands - 1 : band)];
  if (r.mode == kModeShared && maxlen > kSharedMaxLen) r = {kModeGlobal, r.gw >= 8 ? r.gw : 8};
  return r;
}
inline const PassChoice* band_start_table(bool dual = false) {
  static const PassChoice kStart[kBands] = TSU_BAND_START;
  static const PassChoice kStartDual[kBands] = TSU_BAND_START_DUAL;
  return dual ? kStartDual : kStart;
}

// Edit-rate hint of the next retry pass.  Shared-ring passes keep the hint
// (they fail on ring width, staging or history); from the second global pass
// on it grows 4x up to kHintCeiling, at which the step table and the history
// cover the score bound of every pair (s_max <= max_pen * maxlen < s_hint,
// max_pen the dearest single-base edit), so a pass there can fail only on
// memory.
constexpr double kHintCeiling = 2.0;
inline double next_hint(double hint, bool grow) { return grow ? std::min(hint * 4.0, kHintCeiling) : hint; }

// CIGAR arena runs for a batch: 2*s/(cheapest edit) + 1 per pair at the hint.
inline int64_t arena_runs(const Pen& pen, int64_t n, int32_t max_m, int32_t max_n, double hint) {
  const int64_t maxlen = std::max(max_m, max_n);
  const int64_t per_pair = 2 * hint_score(pen, maxlen, hint) / pen.min_pen() + 1;
  return std::max<int64_t>(n * std::min<int64_t>(per_pair, (int64_t)max_m + max_n + 1), 1024);
}

}  // namespace tsu
