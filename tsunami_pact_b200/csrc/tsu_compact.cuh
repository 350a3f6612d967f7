// tsu_compact.cuh -- gather per-pair CIGAR runs from the arena (written in
// completion order) into pair order.
#pragma once

#include "tsu_common.cuh"

namespace tsu {

// One warp per pair, grid-stride.  The length comes from the status-masked
// scan, so a pair that failed in this call contributes 0 runs even if its
// cig_len slot holds a stale value.
static __global__ void compact_kernel(int64_t n, const uint32_t* __restrict__ arena, const int64_t* __restrict__ cig_pos,
                               const int64_t* __restrict__ out_off, uint32_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    const int64_t src = cig_pos[i];
    const int64_t dst = out_off[i];
    const int64_t len = out_off[i + 1] - dst;
    for (int64_t j = lane; j < len; j += 32) out[dst + j] = arena[src + j];
  }
}

// cigar lengths as int64 for the scan (pairs that are not OK count 0)
static __global__ void cig_len64_kernel(int64_t n, const int32_t* __restrict__ len, const int32_t* __restrict__ status,
                                 int64_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = status[i] == kPairOk ? (int64_t)len[i] : 0;
}

}  // namespace tsu
