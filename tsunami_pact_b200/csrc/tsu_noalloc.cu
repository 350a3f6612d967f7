// tsu_noalloc.cu -- tsu_align_scores_noalloc: scores for a batch that is
// already on the device, computed without allocating any device memory.
//
// Why it exists: some callers cannot call cudaMalloc -- plug-ins that live
// under a host framework which owns every device allocation through its own
// pool, and services that must not stall on the driver's allocator or fail on
// memory pressure in the middle of a request.  The context-based entry points
// (tsu_create / tsu_align_batch_device) grow a workspace with cudaMalloc and
// so cannot serve them.
//
// How: all scratch of the call lives in one fixed array compiled into this
// library, g_noalloc_scratch (kNoAllocScratchBytes = 32 MiB).  Every GPU that
// loads the library holds that array until the process exits.  The host code
// below never uses the array's name as an address: on the first call on a
// device, with that device current, it asks the driver for the array's device
// address with cudaGetSymbolAddress and caches it per device, so that first
// call does driver work.
// Each call then carves its buffers (word counts, packed sequences, per-pair
// status, the work-queue counters, and -- for pairs too wide for the shared-
// memory ring -- a global wavefront ring) out of the array, clears what must
// start at zero, and runs the same pack and align kernels as the context
// path.  Every call reuses the same array and leaves its contents behind, so
// two calls whose work overlaps on the GPU (on different streams, or from
// different host threads) race on it and corrupt each other's results; calls
// on one device must be serialized.  Batches that need more scratch than the
// array holds are refused with TSU_EOVERFLOW before the first align pass;
// nothing is truncated.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <mutex>

#include "../../include/tsunami_b200.h"
#include "tsu_kernels.cuh"
#include "tsu_plan.h"

namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;  // the fixed maximum, 32 MiB
constexpr int kMaxDevices = 64;
constexpr size_t kHeaderBytes = 256;

// The scratch array (one per GPU that loads this library).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

unsigned char* g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mu;

// Device address of the scratch array on the current device (set-up on the
// first call per device).
int scratch_on_current_device(unsigned char** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TSU_EDEVICE;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return TSU_EDEVICE;
    }
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return TSU_OK;
}

// Header words of the scratch array.
enum : int { kHdrMaxM = 0, kHdrMaxN = 1, kHdrWords = 2, kHdrBadLen = 3, kHdrQueue = 4, kHdrBadStatus = 5 };

// Longest pattern/text, packed words needed and invalid lengths, on device.
__global__ void noalloc_stats_kernel(int64_t n, const int32_t* __restrict__ plen, const int32_t* __restrict__ tlen,
                                     unsigned long long* hdr) {
  unsigned long long mm = 0, mn = 0, words = 0, bad = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t m = plen[i], t = tlen[i];
    if (m < 0 || t < 0 || m > (1 << 26) || t > (1 << 26)) {
      ++bad;
      continue;
    }
    mm = max(mm, (unsigned long long)m);
    mn = max(mn, (unsigned long long)t);
    words += (unsigned long long)(tsu::packed_words(m) + tsu::packed_words(t));
  }
  atomicMax(hdr + kHdrMaxM, mm);
  atomicMax(hdr + kHdrMaxN, mn);
  atomicAdd(hdr + kHdrWords, words);
  if (bad) atomicAdd(hdr + kHdrBadLen, bad);
}

__global__ void noalloc_count_bad_kernel(int64_t n, const int32_t* __restrict__ status, unsigned long long* hdr) {
  unsigned long long bad = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    bad += status[i] != tsu::kPairOk;
  if (bad) atomicAdd(hdr + kHdrBadStatus, bad);
}

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

// The kernel's dynamic shared memory limit is set to the device maximum, the
// value the engine's contexts set too, so concurrent callers never lower it
// under each other's launches.
template <int kMode>
cudaError_t occupancy(int threads, size_t smem, int optin, int* occ) {
  cudaError_t e =
      cudaFuncSetAttribute(tsu::align_kernel<false, kMode, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, tsu::align_kernel<false, kMode, 1>, threads, smem);
}

}  // namespace

extern "C" int tsu_align_scores_noalloc(const tsu_penalties* pen, const tsu_batch* b, int32_t* score, void* stream) {
  if (!pen || !b || b->num_pairs < 0 || b->num_pairs > INT32_MAX) return TSU_EINVAL;
  if (pen->mismatch <= 0 || pen->gap_opening < 0 || pen->gap_extension <= 0 || pen->mismatch > 1 << 20 ||
      pen->gap_opening > 1 << 20 || pen->gap_extension > 1 << 20)
    return TSU_EINVAL;
  const int64_t n = b->num_pairs;
  if (n == 0) return TSU_OK;
  if (!score || !b->pattern || !b->pattern_off || !b->pattern_len || !b->text || !b->text_off || !b->text_len)
    return TSU_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  int rc = scratch_on_current_device(&base);
  if (rc) return rc;
#define NA_CU(call)                 \
  do {                              \
    if ((call) != cudaSuccess) {    \
      cudaGetLastError();           \
      return TSU_EDEVICE;           \
    }                               \
  } while (0)
  int dev = 0;
  NA_CU(cudaGetDevice(&dev));
  int sms = 0, smem_optin = 0;
  NA_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  NA_CU(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));

  // header: cleared every call (the array keeps the previous call's bytes)
  unsigned long long* hdr = reinterpret_cast<unsigned long long*>(base);
  NA_CU(cudaMemsetAsync(hdr, 0, kHeaderBytes, st));
  noalloc_stats_kernel<<<(int)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 4), 256, 0, st>>>(
      n, b->pattern_len, b->text_len, hdr);
  NA_CU(cudaGetLastError());
  unsigned long long h[4] = {0, 0, 0, 0};
  NA_CU(cudaMemcpyAsync(h, hdr, sizeof h, cudaMemcpyDeviceToHost, st));
  NA_CU(cudaStreamSynchronize(st));
  if (h[kHdrBadLen]) return TSU_EINVAL;
  const int32_t max_m = (int32_t)h[kHdrMaxM], max_n = (int32_t)h[kHdrMaxN];
  const int64_t total_words = (int64_t)h[kHdrWords];

  // carve the array
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<int64_t*>(nullptr), static_cast<int64_t*>(nullptr),
                                (int)(2 * n), st);
  size_t at = kHeaderBytes;
  auto take = [&](size_t bytes) {
    const size_t here = at;
    at += up256(std::max<size_t>(bytes, 1));
    return base + here;
  };
  int64_t* wcnt = reinterpret_cast<int64_t*>(take(sizeof(int64_t) * 2 * n));
  int64_t* woff = reinterpret_cast<int64_t*>(take(sizeof(int64_t) * 2 * n));
  void* scan_tmp = take(scan_bytes);
  uint64_t* words = reinterpret_cast<uint64_t*>(take(sizeof(uint64_t) * (size_t)total_words));
  uint8_t* nonacgt = take((size_t)(2 * n));
  int32_t* status = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * n));
  int32_t* retry = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * n));
  int32_t* order = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * n));
  if (at > kNoAllocScratchBytes) return TSU_EOVERFLOW;  // batch beyond the fixed scratch
  unsigned char* ring_base = base + at;
  const size_t ring_room = kNoAllocScratchBytes - at;
  int g = 1;
  const tsu::Pen rp = tsu::reduce_penalties(pen->mismatch, pen->gap_opening, pen->gap_extension, -1, 0, &g);
  if (rp.slots() > 4096) return TSU_EINVAL;
  // Pairs the shared-memory ring hands back take a second pass on an HBM
  // ring of the longest pair's width; refuse the batch now, before any score
  // is written, if not even one such ring fits beside the packed input.
  const tsu::PassGeom geo_global =
      tsu::plan_geometry(rp, max_m, max_n, tsu::kModeGlobal, 1, 0.2, false, smem_optin);
  if ((size_t)geo_global.ring_ints * sizeof(int32_t) > ring_room) return TSU_EOVERFLOW;

  // pack (same kernels as the context path)
  tsu::word_count_kernel<<<(int)std::min<int64_t>((2 * n + 255) / 256, 4096), 256, 0, st>>>(n, b->pattern_len,
                                                                                            b->text_len, wcnt);
  NA_CU(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, wcnt, woff, (int)(2 * n), st));
  const tsu::SeqView sv{n,
                        reinterpret_cast<const uint8_t*>(b->pattern),
                        b->pattern_off,
                        b->pattern_len,
                        reinterpret_cast<const uint8_t*>(b->text),
                        b->text_off,
                        b->text_len};
  const tsu::PackView pk{words, woff, nonacgt};
  tsu::pack_kernel<<<(int)std::min<int64_t>((2 * n + 7) / 8, (int64_t)sms * 16), 256, 0, st>>>(sv, pk);
  NA_CU(cudaGetLastError());

  // align passes: shared-memory ring first, then a global ring for the pairs
  // it hands back (score only: no history, no step table, no arena)
  unsigned int* queue = reinterpret_cast<unsigned int*>(hdr + kHdrQueue);
  const int32_t* ord = nullptr;
  int64_t n_order = n;
  for (int pass = 0; pass < 2; ++pass) {
    const int wpb = 4;
    const tsu::PassGeom geo = tsu::plan_geometry(rp, max_m, max_n, pass == 0 ? tsu::kModeShared : tsu::kModeGlobal,
                                                 1, 0.2, false, smem_optin);
    // penalties with very deep rings: the shared-memory ring of one warp
    // does not fit a block, and every pair takes the global pass
    if (pass == 0 && geo.mode == tsu::kModeShared && (size_t)wpb * geo.group_smem > (size_t)smem_optin) continue;
    int occ = 0;
    NA_CU(geo.mode == tsu::kModeShared ? occupancy<tsu::kModeShared>(32 * wpb, (size_t)wpb * geo.group_smem, smem_optin, &occ)
                                       : occupancy<tsu::kModeGlobal>(32 * wpb, (size_t)wpb * geo.group_smem, smem_optin, &occ));
    if (occ < 1) {
      if (pass == 0) continue;
      return TSU_EDEVICE;
    }
    int64_t warps = std::min<int64_t>((int64_t)sms * occ * wpb, n_order);
    if (geo.mode == tsu::kModeGlobal)
      warps = std::min<int64_t>(warps, (int64_t)(ring_room / ((size_t)geo.ring_ints * sizeof(int32_t))));
    if (warps < 1) return TSU_EINTERNAL;  // one global ring fits: checked before the first pass
    const int bw = warps >= wpb ? wpb : (int)warps;
    warps = warps / bw * bw;
    tsu::AlignArgs a{};
    a.seq = sv;
    a.pk = pk;
    a.order = ord;
    a.n_order = n_order;
    a.pen = rp;
    a.g = g;
    a.ring_w = geo.ring_w;
    a.seq_cap = geo.seq_cap;
    a.ring_global = geo.mode == tsu::kModeGlobal ? reinterpret_cast<int32_t*>(ring_base) : nullptr;
    a.ring_stride = geo.ring_ints;
    a.score = score;
    a.status = status;
    a.queue = queue;
    a.retry = retry;
    a.retry_count = queue + 1;
    NA_CU(cudaMemsetAsync(queue, 0, 2 * sizeof(unsigned int), st));
    const size_t smem = (size_t)bw * geo.group_smem;
    if (geo.mode == tsu::kModeShared)
      tsu::align_kernel<false, tsu::kModeShared, 1><<<(int)(warps / bw), 32 * bw, smem, st>>>(a);
    else
      tsu::align_kernel<false, tsu::kModeGlobal, 1><<<(int)(warps / bw), 32 * bw, smem, st>>>(a);
    NA_CU(cudaGetLastError());
    unsigned int nretry = 0;
    NA_CU(cudaMemcpyAsync(&nretry, queue + 1, sizeof nretry, cudaMemcpyDeviceToHost, st));
    NA_CU(cudaStreamSynchronize(st));
    if (nretry == 0) break;
    if (pass == 1) return TSU_EINTERNAL;  // a global score-only pass has no capacity limit
    NA_CU(cudaMemcpyAsync(order, retry, sizeof(int32_t) * nretry, cudaMemcpyDeviceToDevice, st));
    ord = order;
    n_order = nretry;
  }
  noalloc_count_bad_kernel<<<(int)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 4), 256, 0, st>>>(n, status, hdr);
  NA_CU(cudaGetLastError());
  unsigned long long bad = 0;
  NA_CU(cudaMemcpyAsync(&bad, hdr + kHdrBadStatus, sizeof bad, cudaMemcpyDeviceToHost, st));
  NA_CU(cudaStreamSynchronize(st));
#undef NA_CU
  return bad ? TSU_EINTERNAL : TSU_OK;
}
