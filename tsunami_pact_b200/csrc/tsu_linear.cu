// tsu_linear.cu -- the gap-linear align_kernel instantiations
// (align_kernel<..., kModelLinear>), in their own translation unit so they
// compile beside the gap-affine kernels of tsu_engine.cu (edit and indel
// distance are gap-linear penalties).
#include "tsu_launch.cuh"

namespace tsu {

cudaError_t align_occupancy_linear(bool cigar, int mode, int gw, int threads, size_t smem, int optin, int* occ,
                                   bool lowmem) {
  return launch_detail::occupancy<kModelLinear>(cigar, mode, gw, threads, smem, optin, occ, lowmem);
}

void launch_align_linear(bool cigar, int mode, int gw, int blocks, int threads, size_t smem, cudaStream_t st,
                         const AlignArgs& a, bool lowmem) {
  launch_detail::launch<kModelLinear>(cigar, mode, gw, blocks, threads, smem, st, a, lowmem);
}

}  // namespace tsu
