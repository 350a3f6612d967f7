// tsu_extend.cuh -- the extend step: longest common prefix along a diagonal.
//
// Replaces the reference's count_chars (wfa_gpu.cu:724-752: a 32-byte
// window reduced through shared memory with 5 barriers, then a byte-serial
// tail on lane 0, wfa_gpu.cu:266-281).  Here each lane extends its own
// diagonal: 16 bases of pattern and text are cut out of the 2-bit words with
// one funnel shift each, XORed, and the first set bit gives the first
// mismatch.  Reads stay inside the sequence plus its padding word because
// the window start is always < the sequence length.
#pragma once

#include "tsu_common.cuh"

namespace tsu {

// Sequence word sources: shared memory (staged copy) or global memory.
struct SharedSeq {
  const uint32_t* p;
  __device__ __forceinline__ uint32_t operator[](int i) const { return p[i]; }
};
struct GlobalSeq {
  const uint32_t* __restrict__ p;
  __device__ __forceinline__ uint32_t operator[](int i) const { return __ldg(p + i); }
};
// Global-ring groups: the pair's words staged in shared memory, or (pairs
// too long to stage) the packed words in global memory, through one generic
// pointer.
struct AnySeq {
  const uint32_t* p;
  __device__ __forceinline__ uint32_t operator[](int i) const { return p[i]; }
};

template <class S>
__device__ __forceinline__ uint32_t win16(const S& w, int pos) {
  const int i = pos >> 4;
  return __funnelshift_r(w[i], w[i + 1], (pos & 15) << 1);
}

// LCP of pattern[v..] and text[h..], at most rem characters.
template <class S>
__device__ __forceinline__ int lcp16(const S& pw, int v, const S& tw, int h, int rem) {
  int l = 0;
  while (l < rem) {
    const uint32_t d = win16(pw, v + l) ^ win16(tw, h + l);
    if (d) {
      l += (__ffs(d) - 1) >> 1;
      break;
    }
    l += 16;
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

}  // namespace tsu
