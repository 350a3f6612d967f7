// tsu_engine_internal.h -- engine calls used by the request server
// (tsu_server.cpp).  Not part of the C ABI: C++ linkage, library-internal.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/tsunami_b200.h"

namespace tsu {
namespace engine {

// tsu_create, optionally with one stream for all work: the host-buffer
// pipeline's copy streams are then the compute stream.  The device runs a
// limited number of hardware queues (CUDA_DEVICE_MAX_CONNECTIONS) that
// streams share in turn; work queued behind a long kernel on a shared queue
// waits for it, so contexts of many host threads use one stream each.
// The penalties of a context: a distance metric (TSU_METRIC_*) and its raw
// penalties (those the metric does not use are 0).
struct Spec {
  int metric = TSU_METRIC_GAP_AFFINE;
  int32_t x = 0, o = 0, e = 0, o2 = 0, e2 = 0;
};
int create(const Spec& spec, const tsu_config* cfg, bool single_stream, tsu_ctx** out);
// The spec of tsu_create_metric's arguments; TSU_EINVAL for an unknown
// metric, a wrong penalty count or a penalty out of range.
int make_spec(int metric, const int32_t* pen, int count, Spec* out);

// Lengths of the pairs of a planned batch (host memory).
struct BatchShape {
  int64_t n = 0;
  const int32_t* plen = nullptr;
  const int32_t* tlen = nullptr;
  int64_t pattern_bytes = 0;  // bytes tsu_align_batch copies up (max offset + length)
  int64_t text_bytes = 0;
};

// Device bytes tsu_align_batch(ctx, batch, flags) will hold at its peak:
// inputs, packed words, outputs, CIGAR arena and the largest length band's
// wavefront scratch at edit-rate hint `hint` (0: the context's).  *full:
// every pair of a band in flight at once (up to what the SMs hold); *min:
// one pair in flight per band (the engine plans fewer pairs in flight when
// its budget is smaller than *full, and fails only below *min).
int predict_bytes(tsu_ctx* ctx, const BatchShape& shape, uint32_t flags, double hint, size_t* full, size_t* min);

// Device bytes the context holds now.
size_t held_bytes(const tsu_ctx* ctx);
// Budget of the next calls (bytes), and its current value.
void set_budget(tsu_ctx* ctx, size_t bytes);
size_t budget_bytes(const tsu_ctx* ctx);
// Edit-rate hint of the next calls (> 0), and its current value.
void set_hint(tsu_ctx* ctx, double hint);
double hint(const tsu_ctx* ctx);
// Choose each band's first rung by the wavefront width the hint predicts
// (tsu::fit_start) -- for hints estimated per pair.
void set_fit_start(tsu_ctx* ctx, bool on);
// Wait for the GPU by sleeping on blocking-sync events instead of spinning
// (for many contexts driven from many host threads).
void set_blocking_sync(tsu_ctx* ctx, bool on);
// Grow buffers to exactly the size asked for (no 1.5x headroom), so a
// context holds no more than its predicted peak.
void set_exact_growth(tsu_ctx* ctx, bool exact);
// Return every device buffer of the context to the pool (waits for the
// context's streams first).
int trim(tsu_ctx* ctx);
// Reserve `bytes` in the device's buffer pool (one allocation, freed at
// once: the pool keeps the memory), so later allocations of any context are
// carved from it instead of growing the pool under load.  Best effort.
void prime_pool(tsu_ctx* ctx, size_t bytes);
// After TSU_ENOMEM: the budget the failed step needed (0 if unknown).
size_t needed_bytes(const tsu_ctx* ctx);

}  // namespace engine
}  // namespace tsu
