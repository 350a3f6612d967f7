// tsu_estimate.h -- host-side estimate of a pair's edit rate from shared
// k-mers, used by the request server to size a long pair's wavefront memory
// (its edit-rate hint) before it runs.
//
// With edits at rate r spread over the pattern, a k-mer of the pattern
// survives intact -- and is found somewhere in the text, whatever the indels
// shifted -- with probability about (1 - r)^k, so the fraction f of sampled
// pattern k-mers present in the text gives r = 1 - f^(1/k).  k = 12 over the
// 2-bit code: a random k-mer of a 50 kbp text matches by chance with
// probability ~0.3 %, well below f at any rate the server sizes for.
// k-mers holding a byte outside ACGT are skipped.  The estimate only sizes
// memory: a pair that needs more is retried with more (the engine's pass
// ladder), so it never changes a result.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace tsu {

inline int base2(char c) {
  switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return -1;
  }
}

// Edit rate of pattern p (m bytes) against text t (n bytes), or -1 when the
// sequences are too short or hold too few ACGT k-mers to say.
inline double estimate_edit_rate(const char* p, int32_t m, const char* t, int32_t n, int max_samples = 4096) {
  constexpr int K = 12;
  constexpr uint32_t kMask = (1u << (2 * K)) - 1;
  if (m < 4 * K || n < 4 * K) return -1.0;
  // open-addressing set of the text's k-mers (key + 1; 0 = empty)
  uint32_t cap = 1;
  while (cap < 2u * (uint32_t)n) cap <<= 1;
  std::vector<uint32_t> set(cap, 0);
  auto hash = [&](uint32_t key) { return (key * 2654435761u) & (cap - 1); };
  uint32_t code = 0;
  int valid = 0;
  for (int32_t i = 0; i < n; ++i) {
    const int b = base2(t[i]);
    if (b < 0) {
      valid = 0;
      continue;
    }
    code = ((code << 2) | (uint32_t)b) & kMask;
    if (++valid < K) continue;
    for (uint32_t h = hash(code);; h = (h + 1) & (cap - 1)) {
      if (set[h] == code + 1) break;
      if (set[h] == 0) {
        set[h] = code + 1;
        break;
      }
    }
  }
  // sample pattern k-mers at a stride
  const int32_t stride = std::max<int32_t>(1, (m - K + 1) / max_samples);
  int64_t tried = 0, found = 0;
  for (int32_t s = 0; s + K <= m; s += stride) {
    uint32_t c = 0;
    bool ok = true;
    for (int j = 0; j < K; ++j) {
      const int b = base2(p[s + j]);
      if (b < 0) {
        ok = false;
        break;
      }
      c = (c << 2) | (uint32_t)b;
    }
    if (!ok) continue;
    ++tried;
    for (uint32_t h = hash(c);; h = (h + 1) & (cap - 1)) {
      if (set[h] == c + 1) {
        ++found;
        break;
      }
      if (set[h] == 0) break;
    }
  }
  if (tried < 32) return -1.0;
  const double f = std::max((double)found / (double)tried, 1e-6);
  return std::min(1.0, std::max(0.0, 1.0 - std::pow(f, 1.0 / K)));
}

}  // namespace tsu
