// tsu_tuning.h -- starting rung of the pass ladder per length band.
// Written by tsunami_pact_b200/tune.py (the autotuner); rebuild the library after changing it.
// band: max(m, n) < 1024, < 2048, < 4096, < 8192, < 16384, >= 16384
// rung: {ring mode (0 shared, 1 global), warps per pair}
// align time in ms per starting rung (s1 s2 s4 s8 s16 g8 g16 g32):
//   band 0 (< 1024): 44.1 62.8 75.4 129.7 324.8 176.3 368.5 648.4
//   band 1 (< 2048): 25.8 24.7 17.1 24.1 51.3 34.0 59.5 93.8
//   band 2 (< 4096): 125.4 128.3 95.7 65.8 124.2 98.1 146.2 208.8
//   band 3 (< 8192): 337.4 351.7 366.6 322.5 340.3 352.4 438.8 531.2
//   band 4 (< 16384): 1695.3 1740.5 1836.9 2071.5 1709.3 2659.1 2364.2 2366.0
//   band 5 (>= 16384): 1008.4 1019.4 1051.2 1127.6 1005.9 1527.8 951.8 863.5
#pragma once
#define TSU_TUNING_SOURCE "tune.py on NVIDIA B200, 2026-12-03, workloads c2:200000,c4:100000,c3:5000"
#define TSU_BAND_START {{0, 1}, {0, 4}, {0, 8}, {0, 8}, {0, 16}, {1, 32}}
