// tsu_tuning_dual.h -- starting rung of the pass ladder per length band (dual gap-affine kernels).
// Written by tsunami_pact_b200/tune.py (the autotuner); rebuild the library after changing it.
// band: max(m, n) < 1024, < 2048, < 4096, < 8192, < 16384, >= 16384
// rung: {ring mode (0 shared, 1 global), warps per pair}
// align time in ms per starting rung (s1 s2 s4 s8 s16 s32 g8 g16 g32):
//   band 0 (< 1024): 615.6 585.2 649.4 255.0 559.7 1404.8 293.8 609.3 1353.4
//   band 1 (< 2048): 109.5 105.1 107.6 116.5 105.7 240.1 76.3 115.7 210.0
//   band 2 (< 4096): 412.9 409.4 411.2 428.5 404.7 640.9 278.8 334.9 493.1
//   band 3 (< 8192): 1341.1 1345.4 1354.0 1380.0 1339.7 1630.9 1413.4 1175.8 1316.5
//   band 4 (< 16384): 13844.2 13858.7 13895.5 13997.0 13848.0 14794.0 21594.7 13260.4 12299.7
//   band 5 (>= 16384): 10181.8 10181.8 10191.0 10241.3 10183.1 10543.1 16621.1 9893.3 8588.0
#pragma once
#define TSU_TUNING_DUAL_SOURCE "tune.py on NVIDIA B200, 2026-12-03, workloads c2:100000,c4:50000,c3:2000, penalties 4/6/2/24/1"
#define TSU_BAND_START_DUAL {{0, 8}, {1, 8}, {1, 8}, {1, 16}, {1, 32}, {1, 32}}
