// tsu_tuning.h -- starting rung of the pass ladder per length band.
// Written by tsunami_pact_b200/tune.py (the autotuner); rebuild the library after changing it.
// band: max(m, n) < 1024, < 2048, < 4096, < 8192, < 16384, >= 16384
// rung: {ring mode (0 shared, 1 global), warps per pair}
// align time in ms per starting rung (s1 s2 s4 s8 s16 g8 g16):
//   band 0 (< 1024): 11.2 7.4 9.1 18.1 55.7 23.6 60.6
//   band 1 (< 2048): 28.8 25.7 17.4 27.5 71.6 37.1 79.9
//   band 2 (< 4096): 164.5 163.0 112.0 72.6 164.4 101.7 186.3
//   band 3 (< 8192): 420.1 434.4 441.1 364.7 423.8 361.3 508.8
//   band 4 (< 16384): 1966.8 2011.3 2104.0 2347.1 1980.9 2686.2 2628.1
//   band 5 (>= 16384): 1394.0 1411.5 1436.5 1524.3 1398.8 1543.3 1021.9
#pragma once
#define TSU_TUNING_SOURCE "tune.py on NVIDIA B200, 2026-12-03, workloads c4:100000,c3:5000"
#define TSU_BAND_START {{0, 2}, {0, 4}, {0, 8}, {1, 8}, {0, 1}, {1, 16}}
