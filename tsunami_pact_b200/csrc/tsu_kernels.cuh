// tsu_kernels.cuh -- all sm_100a kernels of the gap-affine WFA engine.
//
//   pack_kernel / word_count_kernel   tsu_pack.cuh
//   align_kernel<kCigar, kMode>       tsu_align.cuh (extend: tsu_extend.cuh,
//                                     backtrace: tsu_backtrace.cuh)
//   compact_kernel / cig_len64_kernel tsu_compact.cuh
#pragma once

#include "tsu_align.cuh"
#include "tsu_common.cuh"
#include "tsu_compact.cuh"
#include "tsu_pack.cuh"
