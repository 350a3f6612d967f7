// tsu_tuning.h -- starting rung of the pass ladder per length band.
// Written by tsunami_pact_b200/tune.py (the autotuner); defaults until it runs.
// band: max(m, n) < 1024, < 2048, < 4096, < 8192, < 16384, >= 16384
// rung: {ring mode (0 shared, 1 global), warps per pair}
#pragma once
#define TSU_TUNING_SOURCE "default"
#define TSU_BAND_START {{0, 1}, {0, 1}, {0, 4}, {0, 8}, {0, 16}, {0, 16}}
