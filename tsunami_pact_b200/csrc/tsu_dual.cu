// tsu_dual.cu -- the dual gap-affine align_kernel instantiations
// (align_kernel<..., kModelDual>), in their own translation unit so they
// compile beside the one-piece kernels of tsu_engine.cu.
#include "tsu_launch.cuh"

namespace tsu {

cudaError_t align_occupancy_dual(bool cigar, int mode, int gw, int threads, size_t smem, int optin, int* occ,
                                 bool lowmem) {
  return launch_detail::occupancy<kModelDual>(cigar, mode, gw, threads, smem, optin, occ, lowmem);
}

void launch_align_dual(bool cigar, int mode, int gw, int blocks, int threads, size_t smem, cudaStream_t st,
                       const AlignArgs& a, bool lowmem) {
  launch_detail::launch<kModelDual>(cigar, mode, gw, blocks, threads, smem, st, a, lowmem);
}

}  // namespace tsu
