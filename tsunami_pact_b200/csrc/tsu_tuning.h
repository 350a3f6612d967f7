// tsu_tuning.h -- starting rung of the pass ladder per length band.
// Written by tsunami_pact_b200/tune.py (the autotuner); rebuild the library after changing it.
// band: max(m, n) < 1024, < 2048, < 4096, < 8192, < 16384, >= 16384
// rung: {ring mode (0 shared, 1 global), warps per pair}
// align time in ms per starting rung (s1 s2 s4 s8 s16 g8 g16):
//   band 0 (< 1024): 45.2 61.7 76.9 154.4 477.0 198.9 521.9
//   band 1 (< 2048): 28.9 25.8 17.4 27.2 71.5 37.0 79.9
//   band 2 (< 4096): 164.4 162.7 111.7 71.7 164.2 102.0 186.2
//   band 3 (< 8192): 419.6 432.2 440.4 364.7 423.2 367.0 515.9
//   band 4 (< 16384): 1963.7 2009.0 2105.8 2342.7 1981.1 2687.5 2627.6
//   band 5 (>= 16384): 1109.0 1123.4 1156.0 1230.0 1108.5 1542.1 1023.7
#pragma once
#define TSU_TUNING_SOURCE "tune.py on NVIDIA B200, 2026-12-03, workloads c2:200000,c4:100000,c3:5000"
#define TSU_BAND_START {{0, 1}, {0, 4}, {0, 8}, {1, 8}, {0, 16}, {1, 16}}
