// tsu_launch.cuh -- occupancy queries and launches of the align_kernel
// instantiations: CIGAR or score only, shared or global wavefront ring,
// 1/2/4/8/16/32 warps per pair, penalty model (gap-affine, dual gap-affine,
// gap-linear).  Each model's kernels are instantiated in a translation unit
// of their own (tsu_engine.cu, tsu_dual.cu, tsu_linear.cu), compiled in
// parallel.  Each kernel's dynamic
// shared memory limit is set to the device maximum once per device (always
// the same value, so contexts planning on several host threads cannot lower
// it under another's launch).
#pragma once

#include <cuda_runtime.h>

#include <atomic>

#include "tsu_align.cuh"

namespace tsu {

// The dual gap-affine kernels (tsu_dual.cu) and the gap-linear ones
// (tsu_linear.cu).
// lowmem: the low-memory variant of the CIGAR kernel (cigar is then
// ignored).
cudaError_t align_occupancy_dual(bool cigar, int mode, int gw, int threads, size_t smem, int optin, int* occ,
                                 bool lowmem);
void launch_align_dual(bool cigar, int mode, int gw, int blocks, int threads, size_t smem, cudaStream_t st,
                       const AlignArgs& a, bool lowmem);
cudaError_t align_occupancy_linear(bool cigar, int mode, int gw, int threads, size_t smem, int optin, int* occ,
                                   bool lowmem);
void launch_align_linear(bool cigar, int mode, int gw, int blocks, int threads, size_t smem, cudaStream_t st,
                         const AlignArgs& a, bool lowmem);

namespace launch_detail {

template <bool kCigar, int kMode, int GW, int kModel>
cudaError_t occ_one(int threads, size_t smem, int optin, int* occ) {
  static std::atomic<uint64_t> limit_set{0};  // bit d: set on device d
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev < 64 ? (1ull << dev) : 0;
  if (!bit || !(limit_set.load() & bit)) {
    e = cudaFuncSetAttribute(align_kernel<kCigar, kMode, GW, kModel>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin);
    if (e != cudaSuccess) return e;
    limit_set.fetch_or(bit);
  }
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, align_kernel<kCigar, kMode, GW, kModel>, threads, smem);
}

template <bool kCigar, int kMode, int kModel>
cudaError_t occ_gw(int gw, int threads, size_t smem, int optin, int* occ) {
  switch (gw) {
    case 1: return occ_one<kCigar, kMode, 1, kModel>(threads, smem, optin, occ);
    case 2: return occ_one<kCigar, kMode, 2, kModel>(threads, smem, optin, occ);
    case 4: return occ_one<kCigar, kMode, 4, kModel>(threads, smem, optin, occ);
    case 8: return occ_one<kCigar, kMode, 8, kModel>(threads, smem, optin, occ);
    case 16: return occ_one<kCigar, kMode, 16, kModel>(threads, smem, optin, occ);
    case 32: return occ_one<kCigar, kMode, 32, kModel>(threads, smem, optin, occ);
    default: return cudaErrorInvalidValue;
  }
}

template <int kModel>
cudaError_t occupancy(bool cigar, int mode, int gw, int threads, size_t smem, int optin, int* occ, bool lowmem) {
  if (lowmem)
    return mode == kModeShared ? occ_gw<true, kModeShared, kModel | kLowMemFlag>(gw, threads, smem, optin, occ)
                               : occ_gw<true, kModeGlobal, kModel | kLowMemFlag>(gw, threads, smem, optin, occ);
  if (cigar)
    return mode == kModeShared ? occ_gw<true, kModeShared, kModel>(gw, threads, smem, optin, occ)
                               : occ_gw<true, kModeGlobal, kModel>(gw, threads, smem, optin, occ);
  return mode == kModeShared ? occ_gw<false, kModeShared, kModel>(gw, threads, smem, optin, occ)
                             : occ_gw<false, kModeGlobal, kModel>(gw, threads, smem, optin, occ);
}

template <bool kCigar, int kMode, int kModel>
void launch_gw(int gw, int blocks, int threads, size_t smem, cudaStream_t st, const AlignArgs& a) {
  switch (gw) {
    case 1: align_kernel<kCigar, kMode, 1, kModel><<<blocks, threads, smem, st>>>(a); break;
    case 2: align_kernel<kCigar, kMode, 2, kModel><<<blocks, threads, smem, st>>>(a); break;
    case 4: align_kernel<kCigar, kMode, 4, kModel><<<blocks, threads, smem, st>>>(a); break;
    case 8: align_kernel<kCigar, kMode, 8, kModel><<<blocks, threads, smem, st>>>(a); break;
    case 16: align_kernel<kCigar, kMode, 16, kModel><<<blocks, threads, smem, st>>>(a); break;
    case 32: align_kernel<kCigar, kMode, 32, kModel><<<blocks, threads, smem, st>>>(a); break;
    default: break;
  }
}

template <int kModel>
void launch(bool cigar, int mode, int gw, int blocks, int threads, size_t smem, cudaStream_t st, const AlignArgs& a,
            bool lowmem) {
  if (lowmem) {
    if (mode == kModeShared)
      launch_gw<true, kModeShared, kModel | kLowMemFlag>(gw, blocks, threads, smem, st, a);
    else
      launch_gw<true, kModeGlobal, kModel | kLowMemFlag>(gw, blocks, threads, smem, st, a);
  } else if (cigar) {
    if (mode == kModeShared)
      launch_gw<true, kModeShared, kModel>(gw, blocks, threads, smem, st, a);
    else
      launch_gw<true, kModeGlobal, kModel>(gw, blocks, threads, smem, st, a);
  } else {
    if (mode == kModeShared)
      launch_gw<false, kModeShared, kModel>(gw, blocks, threads, smem, st, a);
    else
      launch_gw<false, kModeGlobal, kModel>(gw, blocks, threads, smem, st, a);
  }
}

}  // namespace launch_detail
}  // namespace tsu
