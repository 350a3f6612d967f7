// tsu_bidir.cu -- the BiWFA kernels in their own translation unit: the
// breakpoint kernel instantiations (bidir_kernel<GW>, tsu_bidir.cuh) and the
// base-case segment kernels (tsu_segment.cuh).
#include <cuda_runtime.h>

#include "tsu_bidir.cuh"
#include "tsu_segment.cuh"

namespace tsu {

template <int GW>
static cudaError_t occ_one(int threads, size_t smem, int* occ) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, bidir_kernel<GW>, threads, smem);
}

cudaError_t bidir_occupancy(int gw, int threads, size_t smem, int* occ) {
  switch (gw) {
    case 1: return occ_one<1>(threads, smem, occ);
    case 4: return occ_one<4>(threads, smem, occ);
    case 16: return occ_one<16>(threads, smem, occ);
    default: return cudaErrorInvalidValue;
  }
}

void launch_bidir(int gw, int blocks, int threads, size_t smem, cudaStream_t st, const BidirArgs& a) {
  switch (gw) {
    case 1: bidir_kernel<1><<<blocks, threads, smem, st>>>(a); break;
    case 4: bidir_kernel<4><<<blocks, threads, smem, st>>>(a); break;
    case 16: bidir_kernel<16><<<blocks, threads, smem, st>>>(a); break;
    default: break;
  }
}

cudaError_t segment_occupancy(const Pen& pen, int* blocks_per_sm) {
  int b16 = 0, b32 = 0;
  const size_t smem = seg_smem_bytes(pen);
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b16, segment_kernel<int16_t>, kSegThreads, smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b32, segment_kernel<int32_t>, kSegThreads, smem);
  *blocks_per_sm = b16 < b32 ? b16 : b32;
  return e;
}

void launch_segment(bool int16_history, int blocks, int threads, cudaStream_t st, const SegArgs& a) {
  const size_t smem = seg_smem_bytes(a.pen);
  if (int16_history)
    segment_kernel<int16_t><<<blocks, threads, smem, st>>>(a);
  else
    segment_kernel<int32_t><<<blocks, threads, smem, st>>>(a);
}

void launch_seg_runs(bool write, int blocks, cudaStream_t st, int64_t n, const int32_t* pre_st, const int64_t* pre_off,
                     const int32_t* pre_len, const int64_t* first, const int64_t* run_off, const int32_t* run_len,
                     const uint32_t* runs, const int32_t* status, int64_t* out_len, const int64_t* out_off,
                     uint32_t* out) {
  if (write)
    seg_runs_kernel<true><<<blocks, 256, 0, st>>>(n, pre_st, pre_off, pre_len, first, run_off, run_len, runs, status,
                                                  out_len, out_off, out);
  else
    seg_runs_kernel<false><<<blocks, 256, 0, st>>>(n, pre_st, pre_off, pre_len, first, run_off, run_len, runs, status,
                                                   out_len, out_off, out);
}

void launch_whole_pairs(int blocks, cudaStream_t st, int64_t n, const int32_t* plen, const int32_t* tlen,
                        BidirSeg* segs) {
  whole_pairs_kernel<<<blocks, 256, 0, st>>>(n, plen, tlen, segs);
}

}  // namespace tsu
