// tsu_pack.cuh -- ASCII -> 2-bit packing (the reference compares raw bytes,
// wfa_gpu.cu:735; here every A/C/G/T-only sequence is packed 32 bases per
// 64-bit word so the extend step compares 16 bases per 32-bit funnel shift).
#pragma once

#include "tsu_common.cuh"

namespace tsu {

__device__ __forceinline__ uint64_t spread32(uint32_t v) {
  uint64_t x = v;
  x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
  x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
  x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

// One warp per sequence; lane l of iteration w looks at byte 32*w + l, so each
// load instruction of the warp touches 32 consecutive bytes.  The 2-bit code
// of a base is (c >> 1) & 3 (A=0, C=1, T=2, G=3), a bijection on "ACGT"; any
// other byte marks the sequence for the byte-compare path.  kRev packs each
// sequence reversed (base p of the packed form is byte len - 1 - p), for the
// reverse passes of the bidirectional mode.
template <bool kRev = false>
static __global__ void pack_kernel(SeqView sv, PackView pk) {
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
      uint32_t c = 0x41;  // 'A' beyond the end (masked by the lengths)
      if (p < len) c = src[kRev ? len - 1 - p : p];
      const uint32_t code = (c >> 1) & 3u;
      const bool ok = (c == 0x41u) | (c == 0x43u) | (c == 0x47u) | (c == 0x54u);
      bad |= __ballot_sync(0xffffffffu, !ok);
      const uint32_t b0 = __ballot_sync(0xffffffffu, code & 1u);
      const uint32_t b1 = __ballot_sync(0xffffffffu, (code >> 1) & 1u);
      if (lane == 0) dst[w] = spread32(b0) | (spread32(b1) << 1);
    }
    if (lane == 0) {
      dst[nw] = 0;  // padding word read by the unaligned window loads
      if (!(nw & 1)) dst[nw + 1] = 0;  // the word that makes the count even
      pk.nonacgt[j] = bad ? 1 : 0;
    }
  }
}

// words per sequence: packed_words (data words, padding, even count)
static __global__ void word_count_kernel(int64_t n, const int32_t* __restrict__ pat_len, const int32_t* __restrict__ txt_len,
                                  int64_t* __restrict__ words) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < 2 * n; j += (int64_t)gridDim.x * blockDim.x) {
    const int len = j < n ? pat_len[j] : txt_len[j - n];
    words[j] = packed_words(len);
  }
}

}  // namespace tsu
