// tsu_plan.h -- pass geometry of the align kernel (host only, no CUDA).
//
// Shared by the engine (tsu_engine.cu) and the CPU warp emulation used by the
// tests, so both run the kernel with the same ring width, staging size and
// scratch capacities.
#pragma once

#include <algorithm>
#include <cstdint>

#include "tsu_common.cuh"

namespace tsu {

struct PassGeom {
  int mode = kModeShared;
  int ring_w = 0;          // diagonals per ring slot
  int seq_cap = 0;         // staged sequence words per warp (shared mode)
  int64_t hist_cap = 0;    // backtrace words per warp
  int table_cap = 0;       // step-table entries per warp
  int warp_smem = 0;       // dynamic shared memory per warp (bytes)
  int64_t ring_ints = 0;   // global ring int32 per warp (global mode)
};

constexpr int kSharedW = 384;          // shared-mode ring width (diagonals)
constexpr int kSharedSeqWords = 544;   // shared-mode staging area (uint32 words)
constexpr int kSharedMaxLen = 32000;   // int16 ring limit

// Reduced-unit score expected at edit rate `hint` for a pair of length L.
inline int64_t hint_score(int x, int go, int64_t L, double hint) {
  return (int64_t)(hint * (double)L * (double)std::max(x, go)) + 16;
}

// first: shared-mode pass (int16 ring + staged sequences) when the batch
// allows it; otherwise a global-mode pass wide enough for any pair.
inline PassGeom plan_geometry(int x, int go, int ge, int rm, int re, int32_t max_m, int32_t max_n, bool first,
                              double hint, bool want_cigar, int smem_optin, int warps_per_block) {
  PassGeom p;
  const int ns = ring_slots(rm, re);
  const int64_t maxlen = std::max(max_m, max_n);
  const int64_t s_hint = hint_score(x, go, maxlen, hint);
  const int64_t full_w = (int64_t)max_m + max_n + 3;
  const int64_t width_hint = std::min<int64_t>(full_w, 2 * s_hint / ge + 3);
  if (first && maxlen <= kSharedMaxLen) {
    p.mode = kModeShared;
    p.ring_w = (int)std::max<int64_t>(16, (std::min<int64_t>(full_w, kSharedW) + 15) & ~15);
    const int64_t seqw = 2 * ((max_m + 31) / 32 + 1) + 2 * ((max_n + 31) / 32 + 1);
    p.seq_cap = (int)std::min<int64_t>(seqw, kSharedSeqWords);
  } else {
    p.mode = kModeGlobal;
    p.ring_w = (int)full_w;
    p.seq_cap = 0;
  }
  p.warp_smem = warp_smem_bytes(rm, re, p.ring_w, p.mode, p.seq_cap);
  if ((int64_t)p.warp_smem * warps_per_block > smem_optin) {
    p.mode = kModeGlobal;
    p.ring_w = (int)full_w;
    p.seq_cap = 0;
    p.warp_smem = warp_smem_bytes(rm, re, p.ring_w, p.mode, 0);
  }
  // Backtrace words up to score s: sum_j (2j/ge + 1) ~= s^2/ge + 2s.
  p.table_cap = want_cigar ? (int)std::min<int64_t>(s_hint + 1, INT32_MAX / 2) : 0;
  if (want_cigar) {
    const int64_t sq = s_hint * s_hint / ge + 2 * s_hint + 64;
    p.hist_cap = std::min<int64_t>(std::min<int64_t>(sq, (s_hint + 1) * width_hint), INT32_MAX - 64);
  }
  p.ring_ints = p.mode == kModeShared ? 0 : (int64_t)ns * p.ring_w;
  return p;
}

// Edit-rate hint of the next retry pass.  The first retry keeps the hint
// (the first pass may have failed on ring width or staging alone); later
// ones grow it 4x up to kHintCeiling, at which the step table and the
// history cover the score bound of every pair (s_max <= max(x, o+e) *
// maxlen + o+e < s_hint), so a pass there can fail only on memory.
constexpr double kHintCeiling = 2.0;
inline double next_hint(double hint, bool first_retry) {
  if (first_retry) return hint;
  return std::min(hint * 4.0, kHintCeiling);
}

// CIGAR arena runs for a batch: 2*s/min(x, go) + 1 per pair at the hint.
inline int64_t arena_runs(int x, int go, int64_t n, int32_t max_m, int32_t max_n, double hint) {
  const int64_t maxlen = std::max(max_m, max_n);
  const int64_t per_pair = 2 * hint_score(x, go, maxlen, hint) / std::min(x, go) + 1;
  return std::max<int64_t>(n * std::min<int64_t>(per_pair, (int64_t)max_m + max_n + 1), 1024);
}

}  // namespace tsu
