// emu_model.cpp -- the align_kernel instantiations of one penalty model for
// the CPU warp emulator (test infrastructure), compiled once per model
// (-DEMU_MODEL=<tsu::kModel*> -DEMU_RUN_FN=<name>) so the emulator's three
// model builds run in parallel; emu_driver.cpp calls them.
#include "warp_emu.h"
// clang-format off
#include "../../tsunami_pact_b200/csrc/tsu_kernels.cuh"
// clang-format on

template <bool kCigar, int kMode, int kM = EMU_MODEL>
static void run_gw(int gw, int threads, size_t smem, const tsu::AlignArgs& a) {
  switch (gw) {
    case 1: emu::launch(1, threads, smem, [&] { tsu::align_kernel<kCigar, kMode, 1, kM>(a); }); break;
    case 2: emu::launch(1, threads, smem, [&] { tsu::align_kernel<kCigar, kMode, 2, kM>(a); }); break;
    case 4: emu::launch(1, threads, smem, [&] { tsu::align_kernel<kCigar, kMode, 4, kM>(a); }); break;
    case 8: emu::launch(1, threads, smem, [&] { tsu::align_kernel<kCigar, kMode, 8, kM>(a); }); break;
    case 16: emu::launch(1, threads, smem, [&] { tsu::align_kernel<kCigar, kMode, 16, kM>(a); }); break;
    case 32: emu::launch(1, threads, smem, [&] { tsu::align_kernel<kCigar, kMode, 32, kM>(a); }); break;
    default: std::abort();
  }
}

void EMU_RUN_FN(bool cigar, int mode, int gw, int threads, size_t smem, const tsu::AlignArgs& a, bool lowmem) {
  constexpr int kM = EMU_MODEL | tsu::kLowMemFlag;
  if (lowmem) {
    if (mode == tsu::kModeShared)
      run_gw<true, tsu::kModeShared, kM>(gw, threads, smem, a);
    else
      run_gw<true, tsu::kModeGlobal, kM>(gw, threads, smem, a);
  } else if (cigar) {
    if (mode == tsu::kModeShared)
      run_gw<true, tsu::kModeShared>(gw, threads, smem, a);
    else
      run_gw<true, tsu::kModeGlobal>(gw, threads, smem, a);
  } else {
    if (mode == tsu::kModeShared)
      run_gw<false, tsu::kModeShared>(gw, threads, smem, a);
    else
      run_gw<false, tsu::kModeGlobal>(gw, threads, smem, a);
  }
}
