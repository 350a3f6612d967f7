// tsu_tuning.h -- starting rung of the pass ladder per length band.
// Written by tsunami_pact_b200/tune.py (the autotuner); rebuild the library after changing it.
// band: max(m, n) < 1024, < 2048, < 4096, < 8192, < 16384, >= 16384
// rung: {ring mode (0 shared, 1 global), warps per pair}
// align time in ms per starting rung (s1 s2 s4 s8 s16 g8 g16):
//   band 0 (< 1024): 11.2 7.4 9.1 18.0 55.7 23.6 60.5
//   band 1 (< 2048): 28.8 25.7 17.3 27.4 71.5 36.9 79.8
//   band 2 (< 4096): 164.4 162.7 112.0 72.2 164.2 101.1 186.1
//   band 3 (< 8192): 419.6 432.1 440.2 364.3 423.2 362.4 507.8
//   band 4 (< 16384): 1964.3 2009.7 2101.9 2344.7 1980.9 2689.6 2621.1
//   band 5 (>= 16384): 1111.1 1120.4 1154.4 1230.8 1108.1 1544.3 1023.3
#pragma once
#define TSU_TUNING_SOURCE "tune.py on NVIDIA B200, 2026-12-03, workloads c4:100000,c3:5000"
#define TSU_BAND_START {{0, 2}, {0, 4}, {0, 8}, {1, 8}, {0, 16}, {1, 16}}
