// tsu_engine.cu -- host runtime of the B200 gap-affine WFA engine and the
// C ABI declared in include/tsunami_b200.h.
//
// Replaces the reference host driver's device part (wfa_gpu.cu:83-135):
// instead of 12 cudaMalloc per run, a fixed 32-thread block per pair and
// `wf_length`-sized int16 wavefront slots, a context owns a grow-only device
// workspace inside a memory budget and each call runs
//   H2D -> word-count scan -> pack -> align pass(es) -> CIGAR compaction -> D2H
// on one stream.  Pairs whose wavefronts outgrow the scratch of a pass are
// re-run in a further pass with larger, global-memory scratch; nothing is
// dropped and nothing runs on the CPU.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tsunami_b200.h"
#include "tsu_engine_internal.h"
#include "tsu_bidir.cuh"
#include "tsu_kernels.cuh"
#include "tsu_launch.cuh"
#include "tsu_plan.h"

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

// Page-locked host memory.
struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct Pass {
  tsu::PassGeom g;
  int64_t groups = 0;  // pairs in flight (groups of g.gw warps)
  int blocks = 0;
  int threads = 0;     // per block
  size_t smem_bytes = 0;
};

}  // namespace

struct tsu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[8] = {};
  tsu::engine::Spec spec;  // metric and raw penalties
  tsu::Pen rp;  // reduced penalties, ring depths
  int g = 1;    // score unit
  size_t budget = 0;
  double err_hint = 0.2;
  int sms = 0;
  int smem_optin = 0;
  std::string err;
  tsu_timing timing{};
  // workspace buffers (grow-only)
  DevBuf b_pat, b_txt, b_poff, b_toff, b_plen, b_tlen;   // H2D staging of inputs
  DevBuf b_words_cnt, b_woff, b_words, b_nonacgt;         // packing
  DevBuf b_score, b_status, b_cpos, b_clen, b_clen64, b_coff, b_out;  // outputs
  DevBuf b_order, b_retry, b_counters;                    // queue, retry list, counters
  DevBuf b_scratch, b_arena, b_scan_tmp;                  // wavefront scratch of a pass (carve_scratch), CIGAR arena
  DevBuf b_out2;                                          // second CIGAR output buffer (chunk pipeline)
  DevBuf b_rwords, b_rnonacgt, b_segs, b_bout;            // bidirectional mode: reversed words, segments, cuts
  DevBuf b_bsegs, b_boff, b_blen, b_bruns, b_bfirst;      // bidirectional CIGARs: base cases, their runs
  DevBuf b_pre;                                           // bidirectional CIGARs: the whole-pair launch's results
  bool one_warp = false;  // TSU_ONE_WARP of the current call
  bool bidir = false;     // TSU_BIDIRECTIONAL of the current call
  cudaEvent_t pev[2] = {};  // per-pass timing
  std::string passlog;      // passes of the last align call (tsu_pass_log)
  cudaStream_t h2d_stream = nullptr, d2h_stream = nullptr;  // chunk pipeline copy streams
  cudaEvent_t fence_ev[2] = {};  // orders frees after the copy streams' queued work
  cudaMemPool_t pool = nullptr;  // the device's buffer pool
  bool exact_grow = false;       // grow buffers to the asked size only
  bool fit_start = false;        // start rungs by the hint's predicted width (tsu::fit_start)
  tsu::PassChoice band_start[tsu::kBands] = {};  // starting rung per length band (tsu_set_band_start)
  // The engine's own host transfers (counters, pass orders, retry lists,
  // statuses) go through page-locked buffers: a copy to or from pageable
  // memory blocks the calling thread inside the driver until its stream
  // reaches it, and several host threads' contexts then run one at a time.
  HostBuf h_scalars;  // 64 bytes: retry count, arena cursor, work counters, run total
  HostBuf h_list;     // int32 pass order / retry list
  HostBuf h_status;   // int32 pair statuses (tsu_align_batch)
  HostBuf h_bidir;    // bidirectional mode: segments down, cuts and run counts up
  std::vector<void*> h_retired;  // outgrown page-locked buffers, freed at destroy
  // events of the host-buffer pipeline (tsu_align_batch): 8 chunks at most
  cudaEvent_t cev_up[8] = {}, cev_done[8] = {}, cev_down[8] = {}, cev_t[2] = {};
  // Waits for the GPU sleep on an event instead of spinning (set by the
  // request server, whose many worker threads would otherwise spin on all
  // the host's cores); batch callers keep the driver's default.
  bool blocking_sync = false;
  // The call's fixed launch sequence runs as a CUDA graph, captured anew on
  // each call and updated into this executable graph (re-instantiated when
  // its shape changes).
  bool use_graph = true;
  bool capturing = false;
  cudaGraphExec_t gexec = nullptr;
  int64_t graph_launches = 0;
  cudaEvent_t bev[2 * tsu::kBands] = {};  // first pass of each band: start, end
  cudaEvent_t wait_ev = nullptr;  // blocking-sync event of those waits
  size_t need_bytes = 0;         // budget the last TSU_ENOMEM step needed
  size_t peak_held = 0;          // most bytes held during the current call (tsu_timing.device_bytes)
  // free ends (tsu_set_ends_free): pattern begin, pattern end, text begin,
  // text end; all 0: end-to-end
  int32_t ends_free[4] = {0, 0, 0, 0};
  // low-memory mode (tsu_set_low_memory): 0 off, > 0 checkpoint interval in
  // score steps, < 0 chosen per pass
  int32_t low_mem = 0;
  std::vector<DevBuf*> bufs() {
    return {&b_pat,  &b_txt,    &b_poff,     &b_toff,  &b_plen,  &b_tlen,   &b_words_cnt, &b_woff, &b_words,
            &b_nonacgt, &b_score, &b_status, &b_cpos, &b_clen, &b_clen64, &b_coff,      &b_out,  &b_order,
            &b_retry, &b_counters, &b_scratch, &b_arena, &b_scan_tmp, &b_out2, &b_rwords, &b_rnonacgt,
            &b_segs,  &b_bout, &b_bsegs, &b_boff, &b_blen, &b_bruns, &b_bfirst, &b_pre};
  }
  size_t held() const {
    size_t s = 0;
    for (const DevBuf* b : const_cast<tsu_ctx*>(this)->bufs()) s += b->cap;
    return s;
  }
};

namespace {

int set_err(tsu_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CU(call)                                                                                     \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return set_err(ctx, TSU_EDEVICE, "%s at %s:%d: %s", #call, __FILE__, __LINE__, cudaGetErrorString(e_)); \
  } while (0)

// Longest pattern or text of a pair: 2^26, or the dual backtrace word's
// offset range.
int32_t max_len(const tsu_ctx* ctx) { return ctx->rp.dual() ? tsu::kDualMaxLen : (1 << 26); }


// Device memory of every context comes from one stream-ordered pool per
// device: a buffer is regrown with cudaFreeAsync + cudaMallocFromPoolAsync on
// the context's stream, which never synchronises the device (cudaFree does),
// so contexts driven from several host threads -- the request server's
// workers -- do not stall each other.  Freed blocks stay in the pool
// (release threshold unlimited) for the next allocation of any context.
cudaMemPool_t device_pool(int dev) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lk(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t p = nullptr;
  if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[dev] = p;
  return p;
}

// Free a buffer in stream order after everything queued so far on the
// context's three streams (copy streams read and write some buffers).
void release(tsu_ctx* ctx, DevBuf& b) {
  if (!b.p) return;
  cudaEventRecord(ctx->fence_ev[0], ctx->h2d_stream);
  cudaEventRecord(ctx->fence_ev[1], ctx->d2h_stream);
  cudaStreamWaitEvent(ctx->stream, ctx->fence_ev[0], 0);
  cudaStreamWaitEvent(ctx->stream, ctx->fence_ev[1], 0);
  cudaFreeAsync(b.p, ctx->stream);
  b.p = nullptr;
  b.cap = 0;
}

// Grow a buffer to at least `bytes` within the context budget.  The new
// buffer is ordered on the context's stream; work on the copy streams that
// uses it must wait for that stream (alloc_fence).
int grow(tsu_ctx* ctx, DevBuf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.cap >= bytes) return TSU_OK;
  size_t nb = ctx->exact_grow ? bytes : std::max(bytes, b.cap + b.cap / 2);
  nb = (nb + 255) & ~(size_t)255;
  if (ctx->held() - b.cap + nb > ctx->budget) {
    nb = (bytes + 255) & ~(size_t)255;
    // The wavefront scratch is sized per pass and regrown by the next pass
    // that needs it (a released buffer has capacity 0): give back the one an
    // earlier call or pass left behind before refusing.
    if (ctx->held() - b.cap + nb > ctx->budget && &b != &ctx->b_scratch && ctx->b_scratch.p)
      release(ctx, ctx->b_scratch);
    if (ctx->held() - b.cap + nb > ctx->budget) {
      ctx->need_bytes = ctx->held() - b.cap + nb;
      return set_err(ctx, TSU_ENOMEM, "device budget %zu B exceeded (need %zu more)", ctx->budget, bytes);
    }
  }
  release(ctx, b);
  cudaError_t e = ctx->pool ? cudaMallocFromPoolAsync(&b.p, nb, ctx->pool, ctx->stream) : cudaErrorInvalidValue;
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    ctx->need_bytes = ctx->held() + nb;
    return set_err(ctx, TSU_ENOMEM, "device allocation of %zu B failed: %s", nb, cudaGetErrorString(e));
  }
  b.cap = nb;
  ctx->peak_held = std::max(ctx->peak_held, ctx->held());
  return TSU_OK;
}

// Wait until everything queued so far on stream s is done: a spin in the
// driver, or a sleep on a blocking-sync event (ctx->blocking_sync).
cudaError_t wait_stream(tsu_ctx* ctx, cudaStream_t s) {
  if (!ctx->blocking_sync) return cudaStreamSynchronize(s);
  cudaError_t e = cudaEventRecord(ctx->wait_ev, s);
  if (e != cudaSuccess) return e;
  return cudaEventSynchronize(ctx->wait_ev);
}

// Grow a page-locked buffer to at least `bytes` (doubling).  The outgrown
// one is kept until the context is destroyed: cudaFreeHost can synchronize
// the whole device, stalling other contexts' work.
int host_grow(tsu_ctx* ctx, HostBuf& b, size_t bytes) {
  if (b.cap >= bytes) return TSU_OK;
  const size_t nb = std::max<size_t>(std::max(bytes, 2 * b.cap), 4096);
  void* np = nullptr;
  if (cudaHostAlloc(&np, nb, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, TSU_EDEVICE, "page-locked host allocation of %zu B failed", nb);
  }
  if (b.p) ctx->h_retired.push_back(b.p);
  b.p = np;
  b.cap = nb;
  return TSU_OK;
}

// Make the copy streams wait for the allocations queued on the context's
// stream so far.
void alloc_fence(tsu_ctx* ctx) {
  cudaEventRecord(ctx->fence_ev[0], ctx->stream);
  cudaStreamWaitEvent(ctx->h2d_stream, ctx->fence_ev[0], 0);
  cudaStreamWaitEvent(ctx->d2h_stream, ctx->fence_ev[0], 0);
}

// Every buffer back to the pool, once the context's streams are idle.
int release_all(tsu_ctx* ctx) {
  wait_stream(ctx, ctx->h2d_stream);
  wait_stream(ctx, ctx->d2h_stream);
  wait_stream(ctx, ctx->stream);
  for (DevBuf* b : ctx->bufs()) release(ctx, *b);
  return wait_stream(ctx, ctx->stream) == cudaSuccess ? TSU_OK : TSU_EDEVICE;
}

template <class T>
T* P(DevBuf& b) {
  return static_cast<T*>(b.p);
}

float ev_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}


struct BatchInfo {
  int64_t n = 0;
  int32_t max_m = 0, max_n = 0;
  int64_t total_words = 0;
};

// The align_kernel instantiations (tsu_launch.cuh): gap-affine kernels here,
// dual gap-affine ones in tsu_dual.cu, gap-linear ones in tsu_linear.cu.
// lowmem: the checkpointed-history variant (CIGAR passes of a low-memory
// context).
cudaError_t align_occupancy(const tsu_ctx* ctx, bool cigar, int mode, int gw, int threads, size_t smem, int optin,
                            int* occ, bool lowmem) {
  switch (ctx->rp.model()) {
    case tsu::kModelDual: return tsu::align_occupancy_dual(cigar, mode, gw, threads, smem, optin, occ, lowmem);
    case tsu::kModelLinear: return tsu::align_occupancy_linear(cigar, mode, gw, threads, smem, optin, occ, lowmem);
    default:
      return tsu::launch_detail::occupancy<tsu::kModelAffine>(cigar, mode, gw, threads, smem, optin, occ, lowmem);
  }
}

void launch_align(const tsu_ctx* ctx, bool cigar, int mode, int gw, int blocks, int threads, size_t smem,
                  cudaStream_t st, const tsu::AlignArgs& a) {
  const bool lowmem = cigar && a.ckpt_k > 0;
  switch (ctx->rp.model()) {
    case tsu::kModelDual: tsu::launch_align_dual(cigar, mode, gw, blocks, threads, smem, st, a, lowmem); break;
    case tsu::kModelLinear: tsu::launch_align_linear(cigar, mode, gw, blocks, threads, smem, st, a, lowmem); break;
    default:
      tsu::launch_detail::launch<tsu::kModelAffine>(cigar, mode, gw, blocks, threads, smem, st, a, lowmem);
      break;
  }
}

// Scratch bytes of one group of a pass (ring, history, step table).
size_t group_scratch_bytes(const tsu::PassGeom& g) {
  return (size_t)(g.ring_ints * 4 + g.hist_cap * 4 + (int64_t)g.table_cap * 8 + (int64_t)g.ckpt_cap * g.ckpt_bytes +
                  64);
}

// Configure a pass of configuration pc over pairs of at most bi's lengths:
// geometry, then as many groups as fit the SMs, the pairs and `avail` bytes
// of scratch.
int plan_pass_within(tsu_ctx* ctx, const BatchInfo& bi, int64_t n_pairs, tsu::PassChoice pc, double hint,
                     bool want_cigar, size_t avail, Pass* out) {
  Pass p;
  const tsu::PassGeom g = tsu::plan_geometry(ctx->rp, bi.max_m, bi.max_n, pc.mode, pc.gw, hint, want_cigar,
                                             ctx->smem_optin, want_cigar ? ctx->low_mem : 0);
  p.g = g;
  const int gpc = g.groups_per_cta;
  int occ = 0;
  cudaError_t e =
      align_occupancy(ctx, want_cigar, g.mode, g.gw, g.cta_threads, (size_t)gpc * g.group_smem, ctx->smem_optin, &occ,
                      g.ckpt_k > 0);
  if (e != cudaSuccess || occ < 1) return set_err(ctx, TSU_EDEVICE, "occupancy query failed (%d)", (int)e);
  int64_t warps = (int64_t)ctx->sms * occ * gpc;  // groups
  const size_t per_warp = group_scratch_bytes(g);
  // fewer warps when the pass has fewer pairs or the budget is tight
  warps = std::min<int64_t>(warps, std::max<int64_t>(n_pairs, 1));
  if ((size_t)warps * per_warp > avail) {
    int64_t w2 = (int64_t)(avail / per_warp);
    if (w2 < 1) {
      ctx->need_bytes = ctx->budget - avail + per_warp;
      return set_err(ctx, TSU_ENOMEM, "scratch for one pair (%zu B) exceeds the budget", per_warp);
    }
    warps = w2;
  }
  int gpb = gpc;  // groups per block
  if (warps >= gpc) {
    warps = warps / gpc * gpc;
  } else {
    gpb = (int)warps;  // a single block of fewer groups
  }
  p.groups = warps;
  p.blocks = (int)(warps / gpb);
  p.threads = 32 * g.gw * gpb;
  p.smem_bytes = (size_t)gpb * g.group_smem;
  *out = p;
  return TSU_OK;
}

// plan_pass_within with the budget left beside the context's other buffers
// (the scratch buffers are regrown for the pass: their current size is free)
// and `reserve` bytes that later steps of the call still need.
int plan_pass(tsu_ctx* ctx, const BatchInfo& bi, int64_t n_pairs, tsu::PassChoice pc, double hint, bool want_cigar,
              size_t reserve, Pass* out) {
  const size_t fixed = ctx->held() - ctx->b_scratch.cap + reserve;
  const size_t avail = ctx->budget > fixed ? ctx->budget - fixed : 0;
  return plan_pass_within(ctx, bi, n_pairs, pc, hint, want_cigar, avail, out);
}

// Pairs of a run by length band (tsu::length_band of max(m, n)), each band
// ordered longest first (a counting sort by floor(log2(m + n))).  `uniform`:
// every pair in one length class and band -- run as one band in input order
// (bands stay empty).
struct BandSplit {
  std::vector<std::vector<int32_t>> bands = std::vector<std::vector<int32_t>>(tsu::kBands);
  bool uniform = true;
  int uniform_band = 0;
};

void split_bands(int64_t n, const int32_t* h_plen, const int32_t* h_tlen, BandSplit* out) {
  int64_t cnt[34] = {0};
  auto cls = [&](int64_t i) {
    const uint32_t l = (uint32_t)h_plen[i] + (uint32_t)h_tlen[i];
    return l ? 32 - __builtin_clz(l) : 0;
  };
  int cmin = 33, cmax = 0, bmin = tsu::kBands, bmax = -1;
  for (int64_t i = 0; i < n; ++i) {
    const int c = cls(i);
    ++cnt[c];
    cmin = std::min(cmin, c);
    cmax = std::max(cmax, c);
    const int b = tsu::length_band(std::max(h_plen[i], h_tlen[i]));
    bmin = std::min(bmin, b);
    bmax = std::max(bmax, b);
  }
  out->uniform = cmin == cmax && bmin == bmax;
  out->uniform_band = bmax < 0 ? 0 : bmax;
  if (out->uniform) return;
  std::vector<int32_t> by_len((size_t)n);
  int64_t start[34];
  int64_t acc = 0;
  for (int c = 33; c >= 0; --c) {
    start[c] = acc;
    acc += cnt[c];
  }
  for (int64_t i = 0; i < n; ++i) by_len[(size_t)start[cls(i)]++] = (int32_t)i;
  for (int32_t i : by_len) out->bands[(size_t)tsu::length_band(std::max(h_plen[i], h_tlen[i]))].push_back(i);
}

// Record an event on the stream; inside a stream capture as an event node
// that the graph records when it runs.
cudaError_t record(tsu_ctx* ctx, cudaEvent_t ev, cudaStream_t st) {
  return ctx->capturing ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal) : cudaEventRecord(ev, st);
}

// Queue the work of enqueue() on st: captured as a CUDA graph, updated into
// the context's executable graph (instantiated anew when the update is
// refused: another shape) and launched; or, with ctx->use_graph off, queued
// directly.  enqueue() only queues stream work (no allocation, no
// synchronisation).
template <class F>
int run_graph(tsu_ctx* ctx, cudaStream_t st, F&& enqueue) {
  if (!ctx->use_graph) return enqueue();
  CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  ctx->capturing = true;
  const int rc = enqueue();
  ctx->capturing = false;
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return rc;
  }
  if (e != cudaSuccess) return set_err(ctx, TSU_EDEVICE, "stream capture failed: %s", cudaGetErrorString(e));
  bool updated = false;
  if (ctx->gexec) {
    cudaGraphExecUpdateResultInfo info{};
    updated = cudaGraphExecUpdate(ctx->gexec, graph, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(ctx->gexec);
      ctx->gexec = nullptr;
    }
  }
  if (!updated) {
    const cudaError_t ei = cudaGraphInstantiate(&ctx->gexec, graph, 0);
    if (ei != cudaSuccess) {
      cudaGraphDestroy(graph);
      ctx->gexec = nullptr;
      return set_err(ctx, TSU_EDEVICE, "graph instantiation failed: %s", cudaGetErrorString(ei));
    }
  }
  cudaGraphDestroy(graph);
  CU(cudaGraphLaunch(ctx->gexec, st));
  ++ctx->graph_launches;
  return TSU_OK;
}

// Scratch of a pass, carved from one buffer: backtrace words, step table,
// global ring, each 256-byte aligned.
size_t scratch_bytes(const Pass& ps, bool cigar) {
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t groups = (size_t)ps.groups;
  size_t b = 0;
  if (cigar) b += up(4 * groups * (size_t)ps.g.hist_cap) + up(8 * groups * (size_t)ps.g.table_cap);
  if (ps.g.mode == tsu::kModeGlobal) b += up(4 * groups * (size_t)ps.g.ring_ints);
  if (cigar && ps.g.ckpt_k > 0) b += up(groups * (size_t)ps.g.ckpt_cap * (size_t)ps.g.ckpt_bytes);
  return std::max<size_t>(b, 256);
}

void carve_scratch(tsu_ctx* ctx, const Pass& ps, bool cigar, tsu::AlignArgs* a) {
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  char* p = P<char>(ctx->b_scratch);
  const size_t groups = (size_t)ps.groups;
  a->hist = nullptr;
  a->table = nullptr;
  a->ring_global = nullptr;
  if (cigar) {
    a->hist = reinterpret_cast<uint32_t*>(p);
    p += up(4 * groups * (size_t)ps.g.hist_cap);
    a->table = reinterpret_cast<int2*>(p);
    p += up(8 * groups * (size_t)ps.g.table_cap);
  }
  a->ckpt = nullptr;
  a->ckpt_k = a->ckpt_cap = a->ckpt_bytes = 0;
  a->ckpt_stride = 0;
  if (ps.g.mode == tsu::kModeGlobal) {
    a->ring_global = reinterpret_cast<int32_t*>(p);
    p += up(4 * groups * (size_t)ps.g.ring_ints);
  }
  if (cigar && ps.g.ckpt_k > 0) {
    a->ckpt = reinterpret_cast<uint8_t*>(p);
    a->ckpt_k = ps.g.ckpt_k;
    a->ckpt_cap = ps.g.ckpt_cap;
    a->ckpt_bytes = (int32_t)ps.g.ckpt_bytes;
    a->ckpt_stride = (int64_t)ps.g.ckpt_cap * ps.g.ckpt_bytes;
  }
}

// ---- bidirectional mode (TSU_BIDIRECTIONAL) --------------------------------

// Penalties of the bidirectional mode: the context's for gap-affine; for the
// gap-linear models (edit, indel, gap-linear) gap-affine with a zero gap
// opening -- the same M wavefronts (an I or D value never exceeds the M it
// extends), so the same search and, with the oracle's recursion at o = 0,
// the same optimal CIGARs.
tsu::Pen bidir_pen(const tsu_ctx* ctx) {
  const tsu::Pen& rp = ctx->rp;
  if (rp.model() != tsu::kModelLinear) return rp;
  return tsu::reduce_penalties(rp.x * ctx->g, 0, rp.ge * ctx->g, -1, 0, nullptr);
}

// Checks of the bidirectional mode's settings.
int bidir_check(tsu_ctx* ctx) {
  const tsu::Pen rp = bidir_pen(ctx);
  if (ctx->rp.model() == tsu::kModelDual)
    return set_err(ctx, TSU_EINVAL, "bidirectional mode: one-piece gap-affine or gap-linear penalties only");
  if (ctx->ends_free[0] | ctx->ends_free[1] | ctx->ends_free[2] | ctx->ends_free[3])
    return set_err(ctx, TSU_EINVAL, "bidirectional mode: end-to-end alignment only");
  if (ctx->low_mem) return set_err(ctx, TSU_EINVAL, "bidirectional mode: no low-memory mode");
  if (rp.rm > 64) return set_err(ctx, TSU_EINVAL, "bidirectional mode: rings deeper than 64 score units");
  return TSU_OK;
}

// Packs the pairs forward and reversed (between events ev[2] and ev[3]).
int bidir_pack(tsu_ctx* ctx, const tsu::SeqView& sv, const BatchInfo& bi, tsu::PackView* pk, tsu::PackView* pkr) {
  const int64_t n = sv.n;
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = grow(ctx, ctx->b_words_cnt, sizeof(int64_t) * 2 * n))) return rc;
  if ((rc = grow(ctx, ctx->b_woff, sizeof(int64_t) * 2 * n))) return rc;
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, P<int64_t>(ctx->b_words_cnt), P<int64_t>(ctx->b_woff), (int)(2 * n),
                                st);
  if ((rc = grow(ctx, ctx->b_scan_tmp, tmp_bytes))) return rc;
  if ((rc = grow(ctx, ctx->b_words, sizeof(uint64_t) * (size_t)bi.total_words))) return rc;
  if ((rc = grow(ctx, ctx->b_rwords, sizeof(uint64_t) * (size_t)bi.total_words))) return rc;
  if ((rc = grow(ctx, ctx->b_nonacgt, (size_t)(2 * n)))) return rc;
  if ((rc = grow(ctx, ctx->b_rnonacgt, (size_t)(2 * n)))) return rc;
  *pk = tsu::PackView{P<uint64_t>(ctx->b_words), P<int64_t>(ctx->b_woff), P<uint8_t>(ctx->b_nonacgt)};
  *pkr = tsu::PackView{P<uint64_t>(ctx->b_rwords), P<int64_t>(ctx->b_woff), P<uint8_t>(ctx->b_rnonacgt)};
  CU(cudaEventRecord(ctx->ev[2], st));
  tsu::word_count_kernel<<<std::min<int64_t>((2 * n + 255) / 256, 4096), 256, 0, st>>>(n, sv.pat_len, sv.txt_len,
                                                                                       P<int64_t>(ctx->b_words_cnt));
  size_t tb = tmp_bytes;
  CU(cub::DeviceScan::ExclusiveSum(ctx->b_scan_tmp.p, tb, P<int64_t>(ctx->b_words_cnt), P<int64_t>(ctx->b_woff),
                                   (int)(2 * n), st));
  const int64_t pblocks = std::min<int64_t>((2 * n + 7) / 8, (int64_t)ctx->sms * 16);
  tsu::pack_kernel<<<(int)pblocks, 256, 0, st>>>(sv, *pk);
  tsu::pack_kernel<true><<<(int)pblocks, 256, 0, st>>>(sv, *pkr);
  CU(cudaGetLastError());
  CU(cudaEventRecord(ctx->ev[3], st));
  return TSU_OK;
}

// Warps per segment of the breakpoint kernel by the segment's longest side.
int bidir_gw(int32_t side) { return side < 2048 ? 1 : (side < 16384 ? 4 : 16); }

// One persistent launch of the breakpoint kernel (tsu_bidir.cuh) over c
// segments (device) of one size class, one group per segment at a time (gw
// = 1, 4 or 16 warps), both rings of a group in device memory (2 directions
// x ring depth x 4 components x (max_bases + 3) values, int16 below 16 warps
// and int32 at 16, from the scratch buffer).  Writes T, comp, k, h at out + 0, out + stride, out + 2 stride,
// out + 3 stride and the statuses; adds cells and steps to d_work[0..1].
int bidir_split(tsu_ctx* ctx, const tsu::SeqView& sv, const tsu::PackView& pk, const tsu::PackView& pkr,
                const tsu::BidirSeg* segs, int64_t c, int gw, int32_t max_bases, int32_t* out, int64_t stride,
                int32_t* status, unsigned int* d_queue, unsigned long long* d_work, std::string* log) {
  cudaStream_t st = ctx->stream;
  int rc;
  const tsu::Pen rp = bidir_pen(ctx);
  const int threads = gw <= 4 ? 128 : 32 * gw;
  const int gpb = threads / (32 * gw);
  const size_t smem = (size_t)gpb * tsu::bidir_group_smem(rp, gw);
  int occ = 0;
  CU(tsu::bidir_occupancy(gw, threads, smem, &occ));
  if (occ < 1) return set_err(ctx, TSU_EDEVICE, "bidirectional kernel: no occupancy");
  const int ring_w = max_bases + 3;
  const int64_t ring_stride = (int64_t)2 * rp.rm * 4 * ring_w;  // elements per group
  const size_t ring_bytes = (size_t)tsu::bidir_ring_bytes(gw) * (size_t)ring_stride;
  int64_t groups = std::min<int64_t>((int64_t)ctx->sms * occ * gpb, c);
  const size_t fixed = ctx->held() - ctx->b_scratch.cap;
  const size_t avail = ctx->budget > fixed ? ctx->budget - fixed : 0;
  groups = std::min<int64_t>(groups, (int64_t)(avail / ring_bytes));
  if (groups < 1) return set_err(ctx, TSU_ENOMEM, "bidirectional mode: rings of one pair exceed the budget");
  int bpg = gpb;  // groups per block
  if (groups >= gpb)
    groups = groups / gpb * gpb;
  else
    bpg = (int)groups;
  const size_t need = ring_bytes * (size_t)groups;
  if (need > ctx->b_scratch.cap) {
    release(ctx, ctx->b_scratch);
    if ((rc = grow(ctx, ctx->b_scratch, need))) return rc;
  }
  CU(cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st));
  tsu::BidirArgs a{};
  a.seq = sv;
  a.pk = pk;
  a.pkr = pkr;
  a.segs = segs;
  a.n_segs = c;
  a.pen = rp;
  a.ring_w = ring_w;
  a.ring = ctx->b_scratch.p;
  a.ring_stride = ring_stride;
  a.out_T = out;
  a.out_comp = out + stride;
  a.out_k = out + 2 * stride;
  a.out_h = out + 3 * stride;
  a.status = status;
  a.queue = d_queue;
  a.work = d_work;
  tsu::launch_bidir(gw, (int)(groups / bpg), 32 * gw * bpg, (size_t)bpg * tsu::bidir_group_smem(rp, gw), st, a);
  CU(cudaGetLastError());
  ctx->timing.kernel_launches++;
  if (log) *log += (log->empty() ? "b" : " b") + std::to_string(gw) + "x" + std::to_string(groups) + ":" + std::to_string(c);
  return TSU_OK;
}

// One breakpoint level over the host segments cur: ordered by size class
// (16-warp segments first, then 4, then 1; stable, so a class keeps the
// input order), copied to the device, one launch per class.  Results per
// segment of the reordered cur: T, comp, k, h at bo + 0, c, 2c, 3c, status
// at bo + 4c (bo: 5 c int32).
int bidir_level(tsu_ctx* ctx, const tsu::SeqView& sv, const tsu::PackView& pk, const tsu::PackView& pkr,
                std::vector<tsu::BidirSeg>* cur, int32_t* bo, unsigned int* d_queue, unsigned long long* d_work,
                std::string* log) {
  cudaStream_t st = ctx->stream;
  int rc;
  const int64_t c = (int64_t)cur->size();
  {
    // stable partition into the classes 16, 4, 1 warps (three buckets)
    int64_t cnt[3] = {0, 0, 0};
    auto cls = [](const tsu::BidirSeg& q) {
      const int gw = bidir_gw(std::max(q.m, q.n));
      return gw == 16 ? 0 : (gw == 4 ? 1 : 2);
    };
    for (const tsu::BidirSeg& q : *cur) cnt[cls(q)]++;
    if (cnt[0] + cnt[1] && cnt[1] + cnt[2] && cnt[0] + cnt[2]) {  // more than one class
      int64_t pos[3] = {0, cnt[0], cnt[0] + cnt[1]};
      std::vector<tsu::BidirSeg> sorted((size_t)c);
      for (const tsu::BidirSeg& q : *cur) sorted[(size_t)pos[cls(q)]++] = q;
      cur->swap(sorted);
    }
  }
  if ((rc = grow(ctx, ctx->b_segs, sizeof(tsu::BidirSeg) * c))) return rc;
  const size_t seg_bytes = sizeof(tsu::BidirSeg) * (size_t)c;
  if ((rc = host_grow(ctx, ctx->h_bidir, std::max(seg_bytes, sizeof(int32_t) * 5 * (size_t)c)))) return rc;
  std::memcpy(ctx->h_bidir.p, cur->data(), seg_bytes);
  CU(cudaMemcpyAsync(ctx->b_segs.p, ctx->h_bidir.p, seg_bytes, cudaMemcpyHostToDevice, st));
  const tsu::BidirSeg* d_segs = P<tsu::BidirSeg>(ctx->b_segs);
  for (int64_t c0 = 0; c0 < c;) {
    const int gw = bidir_gw(std::max((*cur)[(size_t)c0].m, (*cur)[(size_t)c0].n));
    int64_t c1 = c0;
    int32_t max_bases = 0;
    while (c1 < c && bidir_gw(std::max((*cur)[(size_t)c1].m, (*cur)[(size_t)c1].n)) == gw) {
      max_bases = std::max(max_bases, (*cur)[(size_t)c1].m + (*cur)[(size_t)c1].n);
      ++c1;
    }
    if ((rc = bidir_split(ctx, sv, pk, pkr, d_segs + c0, c1 - c0, gw, max_bases, bo + c0, c, bo + 4 * c + c0, d_queue,
                          d_work, log)))
      return rc;
    c0 = c1;
  }
  return TSU_OK;
}

// Level 0's results to the pairs: score[pair] = T g (0 when none),
// status[pair].
__global__ void bidir_level0_kernel(int64_t c, const tsu::BidirSeg* __restrict__ segs, const int32_t* __restrict__ bo,
                                    int g, int32_t* __restrict__ score, int32_t* __restrict__ status) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < c; j += (int64_t)gridDim.x * blockDim.x) {
    const int32_t p = segs[j].pair;
    score[p] = bo[j] >= 0 ? bo[j] * g : 0;
    status[p] = bo[4 * c + j];
  }
}

// TSU_BIDIRECTIONAL score-only calls: pack the pairs forward and reversed,
// then one breakpoint launch over all pairs, each pair whole and free at
// both ends.  A pair's score is its lowest crossing total; for an
// end-to-end pair that is the optimal score.
int run_bidir(tsu_ctx* ctx, const tsu::SeqView& sv, int32_t* d_score, int32_t* d_status, const BatchInfo& bi,
              const int32_t* h_plen, const int32_t* h_tlen) {
  const int64_t n = sv.n;
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = bidir_check(ctx))) return rc;
  if ((rc = grow(ctx, ctx->b_bout, sizeof(int32_t) * 5 * n))) return rc;
  if ((rc = grow(ctx, ctx->b_counters, 64))) return rc;
  tsu::PackView pk, pkr;
  if ((rc = bidir_pack(ctx, sv, bi, &pk, &pkr))) return rc;
  unsigned long long* d_cnt = P<unsigned long long>(ctx->b_counters);
  CU(cudaMemsetAsync(d_cnt, 0, 64, st));
  int32_t* bo = P<int32_t>(ctx->b_bout);
  ctx->timing.kernel_launches = 3;
  std::string log;
  std::vector<tsu::BidirSeg> cur((size_t)n);
  for (int64_t i = 0; i < n; ++i) cur[(size_t)i] = tsu::BidirSeg{(int32_t)i, 0, 0, h_plen[i], h_tlen[i], 'M', 'M'};
  CU(cudaEventRecord(ctx->ev[4], st));
  if ((rc = bidir_level(ctx, sv, pk, pkr, &cur, bo, reinterpret_cast<unsigned int*>(d_cnt), d_cnt + 1, &log)))
    return rc;
  const int eblocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sms * 8);
  bidir_level0_kernel<<<eblocks, 256, 0, st>>>(n, P<tsu::BidirSeg>(ctx->b_segs), bo, ctx->g, d_score, d_status);
  CU(cudaGetLastError());
  ctx->timing.kernel_launches++;
  CU(cudaEventRecord(ctx->ev[5], st));
  CU(cudaEventRecord(ctx->ev[6], st));
  char* h = static_cast<char*>(ctx->h_scalars.p);
  CU(cudaMemcpyAsync(h, d_cnt + 1, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CU(wait_stream(ctx, st));
  ctx->timing.cells = (int64_t)reinterpret_cast<const unsigned long long*>(h)[0];
  ctx->timing.steps = (int64_t)reinterpret_cast<const unsigned long long*>(h)[1];
  ctx->passlog = log;
  return TSU_OK;
}

// TSU_BIDIRECTIONAL calls with CIGARs: the BiWFA recursion, level by level.
// First every pair runs whole through the segment kernel (tsu_segment.cuh)
// with a step cap of the base score + 1: a pair whose optimal score is at
// most the base score (tsu::bidir_base: max(2 max(x, o + e), 256) score
// units) is done there -- its crossing total would be that score, so the
// recursion would align it whole the same way -- and only the others enter
// the recursion.  Its level 0 is those pairs whole; each level's segments
// go through one breakpoint launch per size class, and the host cuts each
// segment at its crossing (k, h) into a left part (begin component,
// crossing component) and a right part (crossing component, end component)
// for the next level -- unless the crossing total is at most the base score
// or the cut leaves one side empty, when the segment is a leaf.  Leaves run
// through the segment kernel in launches of growing step caps (a leaf that
// outgrows its launch's history goes to the next), and one thread per pair
// joins its leaves' runs in order.  Scores come from the first launch or
// from level 0.
int run_bidir_cigar(tsu_ctx* ctx, const tsu::SeqView& sv, int32_t* d_score, int32_t* d_status, uint32_t* d_out_runs,
                    int64_t out_cap, int64_t* d_out_off, int64_t* runs_needed, const BatchInfo& bi,
                    const int32_t* h_plen, const int32_t* h_tlen, uint32_t** out_used, DevBuf* out_buf) {
  const int64_t n = sv.n;
  cudaStream_t st = ctx->stream;
  int rc;
  if ((rc = bidir_check(ctx))) return rc;
  const tsu::Pen rp = bidir_pen(ctx);
  if ((rc = grow(ctx, ctx->b_counters, 64))) return rc;
  if ((rc = grow(ctx, ctx->b_clen64, sizeof(int64_t) * (n + 1)))) return rc;
  if ((rc = grow(ctx, ctx->b_bfirst, sizeof(int64_t) * (n + 1)))) return rc;
  tsu::PackView pk, pkr;
  if ((rc = bidir_pack(ctx, sv, bi, &pk, &pkr))) return rc;
  unsigned long long* d_cnt = P<unsigned long long>(ctx->b_counters);
  unsigned int* d_queue = reinterpret_cast<unsigned int*>(d_cnt);
  CU(cudaMemsetAsync(d_cnt, 0, 64, st));
  ctx->timing.kernel_launches = 3;
  std::string log;
  CU(cudaEventRecord(ctx->ev[4], st));
  const int base = tsu::bidir_base(rp);
  std::vector<int32_t> pst((size_t)n, tsu::kPairOk);  // pair statuses

  // ---- leaves: segments aligned whole by the segment kernel; their runs
  // packed into one arena (an atomic cursor at d_cnt[3]; grown by copy, so
  // earlier runs stay)
  std::vector<tsu::BidirSeg> leaves;
  std::vector<int32_t> lcap, lstat, lruns;  // step cap to run at / status / runs
  std::vector<int64_t> roff;                // first run in the arena
  unsigned long long* d_cursor = d_cnt + 3;
  int64_t arena_used = 0;  // the cursor after the last launch
  int segs_occ = 0;
  CU(tsu::segment_occupancy(rp, &segs_occ));
  if (segs_occ < 1) return set_err(ctx, TSU_EDEVICE, "segment kernel: no occupancy");
  // Grow the arena by copy to hold at least `need` runs.
  auto grow_arena = [&](int64_t need) -> int {
    const size_t run_bytes = sizeof(uint32_t) * (size_t)std::max<int64_t>(need, 64);
    if (run_bytes <= ctx->b_bruns.cap) return TSU_OK;
    DevBuf nb;
    const size_t bytes = (std::max(run_bytes, ctx->b_bruns.cap + ctx->b_bruns.cap / 2) + 255) & ~(size_t)255;
    if (ctx->held() + bytes > ctx->budget) release(ctx, ctx->b_scratch);
    if (ctx->held() + bytes > ctx->budget) {
      ctx->need_bytes = ctx->held() + bytes;
      return set_err(ctx, TSU_ENOMEM, "bidirectional mode: CIGAR runs exceed the budget");
    }
    CU(cudaMallocFromPoolAsync(&nb.p, bytes, ctx->pool, st));
    nb.cap = bytes;
    if (arena_used)
      CU(cudaMemcpyAsync(nb.p, ctx->b_bruns.p, sizeof(uint32_t) * (size_t)arena_used, cudaMemcpyDeviceToDevice, st));
    ctx->peak_held = std::max(ctx->peak_held, ctx->held() + nb.cap);
    release(ctx, ctx->b_bruns);
    ctx->b_bruns = nb;
    return TSU_OK;
  };
  // One segment-kernel launch over c segments on the device (longest m + n
  // `bases`, longest side `side`) at step cap scap, the arena grown to hold
  // `expect` more runs first; results per segment at d_off, d_len, d_st.
  // Afterwards arena_used is what the arena holds, and the cursor is put
  // back there if segments found the arena full.
  auto run_segments = [&](const tsu::BidirSeg* d_segs, int64_t c, int32_t bases, int32_t side, int scap,
                          int64_t expect, int64_t* d_off, int32_t* d_len, int32_t* d_st, int32_t* d_pair_score) -> int {
    int rc2;
    if ((rc2 = grow_arena(arena_used + expect))) return rc2;
    const bool h16 = side < 32767;  // int16 history: every offset fits
    const int64_t hcap = tsu::seg_hist_cap(scap, bases);
    const int64_t wcap = tsu::seg_run_cap(rp, bases, scap);
    const size_t hist_w = ((h16 ? 2 : 4) * 3 * (size_t)hcap + 15) & ~(size_t)15;  // bytes per warp
    const size_t per_warp = hist_w + sizeof(int32_t) * (size_t)(9 * (int64_t)scap + wcap);
    const int wpb = tsu::kSegThreads / 32;
    int64_t warps = std::min<int64_t>((int64_t)ctx->sms * segs_occ * wpb, c);
    const size_t fixed = ctx->held() - ctx->b_scratch.cap;
    const size_t avail = ctx->budget > fixed ? ctx->budget - fixed : 0;
    warps = std::min<int64_t>(warps, (int64_t)(avail / per_warp));
    if (warps < 1) {
      ctx->need_bytes = fixed + per_warp;
      return set_err(ctx, TSU_ENOMEM, "bidirectional mode: base-case history of one segment exceeds the budget");
    }
    // whole blocks within the budget (rounded down); below one block's
    // worth, one smaller block
    int threads = tsu::kSegThreads;
    int64_t blocks = warps / wpb;
    if (blocks == 0) blocks = 1, threads = 32 * (int)warps;
    const size_t nw = (size_t)(blocks * (threads / 32));
    if (per_warp * nw > ctx->b_scratch.cap) {
      release(ctx, ctx->b_scratch);
      if ((rc2 = grow(ctx, ctx->b_scratch, per_warp * nw))) return rc2;
    }
    CU(cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st));
    char* const sc = P<char>(ctx->b_scratch);
    int32_t* const sc_tab = reinterpret_cast<int32_t*>(sc + nw * hist_w);
    tsu::SegArgs a{};
    a.seq = sv;
    a.pk = pk;
    a.pkr = pkr;
    a.segs = d_segs;
    a.n_segs = c;
    a.pen = rp;
    a.g = ctx->g;
    a.hist = sc;
    a.hist_cap = hist_w / ((h16 ? 2 : 4) * 3);  // cells per warp (the area is rounded up to 16 B)
    a.table = sc_tab;
    a.step_cap = scap;
    a.wruns = reinterpret_cast<uint32_t*>(sc_tab + nw * 9 * (size_t)scap);
    a.wruns_cap = wcap;
    a.runs = P<uint32_t>(ctx->b_bruns);
    a.runs_cap = (int64_t)(ctx->b_bruns.cap / sizeof(uint32_t));
    a.cursor = d_cursor;
    a.run_off = d_off;
    a.run_len = d_len;
    a.status = d_st;
    a.pair_score = d_pair_score;
    a.queue = d_queue;
    a.work = d_cnt + 1;
    tsu::launch_segment(h16, (int)blocks, threads, st, a);
    CU(cudaGetLastError());
    ctx->timing.kernel_launches++;
    log += (log.empty() ? "s" : " s") + std::to_string(scap) + "x" + std::to_string(nw) + ":" + std::to_string(c);
    unsigned long long* h_cur = reinterpret_cast<unsigned long long*>(static_cast<char*>(ctx->h_scalars.p) + 48);
    CU(cudaMemcpyAsync(h_cur, d_cursor, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CU(wait_stream(ctx, st));
    // the cursor counts the runs of segments that found the arena full too;
    // the arena keeps everything below its capacity
    arena_used = std::min<int64_t>((int64_t)*h_cur, a.runs_cap);
    if ((int64_t)*h_cur > a.runs_cap) {
      *h_cur = (unsigned long long)arena_used;
      CU(cudaMemcpyAsync(d_cursor, h_cur, sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
    }
    return TSU_OK;
  };
  // One launch over the leaves pick (indices into leaves) at step cap scap;
  // leaves that find the arena full run again after it grows.
  auto launch_leaves = [&](std::vector<int64_t> pick, int scap) -> int {
    int rc2;
    for (int attempt = 0; !pick.empty(); ++attempt) {
      if (attempt > 8) return set_err(ctx, TSU_EINTERNAL, "segment kernel: run arena keeps overflowing");
      const int64_t c = (int64_t)pick.size();
      std::vector<tsu::BidirSeg> ls((size_t)c);
      int32_t bases = 0, side = 0;
      int64_t expect = 0;  // runs expected: a quarter of the worst case, at least 16 per leaf
      for (int64_t j = 0; j < c; ++j) {
        const tsu::BidirSeg& s = leaves[(size_t)pick[(size_t)j]];
        ls[(size_t)j] = s;
        bases = std::max(bases, s.m + s.n);
        side = std::max(side, std::max(s.m, s.n));
        expect += std::max<int64_t>(16, tsu::seg_run_cap(rp, (int64_t)s.m + s.n, scap) / (attempt ? 1 : 4));
      }
      if ((rc2 = grow(ctx, ctx->b_bsegs, sizeof(tsu::BidirSeg) * std::max<int64_t>(c, 1)))) return rc2;
      if ((rc2 = grow(ctx, ctx->b_boff, sizeof(int64_t) * std::max<int64_t>(c, 1)))) return rc2;
      if ((rc2 = grow(ctx, ctx->b_blen, 2 * sizeof(int32_t) * std::max<int64_t>(c, 1)))) return rc2;
      const size_t sb = sizeof(tsu::BidirSeg) * (size_t)c;
      if ((rc2 = host_grow(ctx, ctx->h_bidir, std::max(sb, (sizeof(int64_t) + 2 * sizeof(int32_t)) * (size_t)c) + 16)))
        return rc2;
      char* hb = static_cast<char*>(ctx->h_bidir.p);
      std::memcpy(hb, ls.data(), sb);
      CU(cudaMemcpyAsync(ctx->b_bsegs.p, hb, sb, cudaMemcpyHostToDevice, st));
      int32_t* d_rlen = P<int32_t>(ctx->b_blen);
      if ((rc2 = run_segments(P<tsu::BidirSeg>(ctx->b_bsegs), c, bases, side, scap, expect, P<int64_t>(ctx->b_boff),
                              d_rlen, d_rlen + c, nullptr)))
        return rc2;
      int64_t* h_off = reinterpret_cast<int64_t*>(hb);
      int32_t* h_len = reinterpret_cast<int32_t*>(h_off + c);
      CU(cudaMemcpyAsync(h_off, ctx->b_boff.p, sizeof(int64_t) * (size_t)c, cudaMemcpyDeviceToHost, st));
      CU(cudaMemcpyAsync(h_len, d_rlen, 2 * sizeof(int32_t) * (size_t)c, cudaMemcpyDeviceToHost, st));
      CU(wait_stream(ctx, st));
      std::vector<int64_t> again;
      for (int64_t j = 0; j < c; ++j) {
        const size_t i = (size_t)pick[(size_t)j];
        const int32_t s = h_len[c + j];
        if (s == tsu::kPairArena) {
          again.push_back((int64_t)i);
          continue;
        }
        lstat[i] = s;
        if (s == tsu::kPairOk) {
          roff[i] = h_off[j];
          lruns[i] = h_len[j];
        }
      }
      pick.swap(again);
    }
    return TSU_OK;
  };
  auto add_leaf = [&](const tsu::BidirSeg& s, int cap) {
    leaves.push_back(s);
    lcap.push_back(cap);
    lstat.push_back(tsu::kPairScratch);
    lruns.push_back(0);
    roff.push_back(0);
  };

  // ---- whole pairs at the base score, bookkept on the device: segments
  // built there, results in their own arrays (pre_off, pre_len, pre_st);
  // only the statuses come back.  A pair that outgrew the cap, or found the
  // arena full, enters the recursion (which aligns a pair of score at most
  // the base whole, the same way).
  if ((rc = grow(ctx, ctx->b_pre, (sizeof(int64_t) + 2 * sizeof(int32_t)) * (size_t)std::max<int64_t>(n, 1)))) return rc;
  int64_t* const pre_off = P<int64_t>(ctx->b_pre);
  int32_t* const pre_len = reinterpret_cast<int32_t*>(pre_off + n);
  int32_t* const pre_st = pre_len + n;
  std::vector<tsu::BidirSeg> cur;
  {
    if ((rc = grow(ctx, ctx->b_bsegs, sizeof(tsu::BidirSeg) * std::max<int64_t>(n, 1)))) return rc;
    // the arena sized for every pair's worst case at this cap (about 1 KB
    // per pair at 4/6/2) when that takes at most a quarter of the budget: a
    // pair that finds it full costs a breakpoint search
    int32_t bases = 0, side = 0;
    int64_t worst = 0;
    for (int64_t i = 0; i < n; ++i) {
      bases = std::max(bases, h_plen[i] + h_tlen[i]);
      side = std::max(side, std::max(h_plen[i], h_tlen[i]));
      worst += tsu::seg_run_cap(rp, (int64_t)h_plen[i] + h_tlen[i], base + 1);
    }
    const int64_t expect = sizeof(uint32_t) * (size_t)worst <= ctx->budget / 4 ? worst : std::max<int64_t>(worst / 4, 16 * n);
    const int eblocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sms * 8);
    tsu::launch_whole_pairs(eblocks, st, n, sv.pat_len, sv.txt_len, P<tsu::BidirSeg>(ctx->b_bsegs));
    CU(cudaGetLastError());
    ctx->timing.kernel_launches++;
    if ((rc = run_segments(P<tsu::BidirSeg>(ctx->b_bsegs), n, bases, side, base + 1, expect, pre_off, pre_len, pre_st,
                           d_score)))
      return rc;
    if ((rc = host_grow(ctx, ctx->h_bidir, sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)))) return rc;
    int32_t* h_st = static_cast<int32_t*>(ctx->h_bidir.p);
    CU(cudaMemcpyAsync(h_st, pre_st, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
    CU(wait_stream(ctx, st));
    for (int64_t i = 0; i < n; ++i) {
      const int32_t s = h_st[i];
      if (s == tsu::kPairScratch || s == tsu::kPairArena)
        cur.push_back(tsu::BidirSeg{(int32_t)i, 0, 0, h_plen[i], h_tlen[i], 'M', 'M'});
      else if (s != tsu::kPairOk)
        pst[(size_t)i] = s;
    }
  }

  // ---- the recursion over the other pairs
  for (int level = 0; !cur.empty(); ++level) {
    const int64_t c = (int64_t)cur.size();
    const size_t res_bytes = sizeof(int32_t) * 5 * (size_t)c;
    if ((rc = grow(ctx, ctx->b_bout, res_bytes))) return rc;
    int32_t* bo = P<int32_t>(ctx->b_bout);
    if ((rc = bidir_level(ctx, sv, pk, pkr, &cur, bo, d_queue, d_cnt + 1, &log))) return rc;
    if (level == 0) {
      const int eblocks = (int)std::min<int64_t>((c + 255) / 256, (int64_t)ctx->sms * 8);
      bidir_level0_kernel<<<eblocks, 256, 0, st>>>(c, P<tsu::BidirSeg>(ctx->b_segs), bo, ctx->g, d_score, d_status);
      CU(cudaGetLastError());
      ctx->timing.kernel_launches++;
    }
    CU(cudaMemcpyAsync(ctx->h_bidir.p, bo, res_bytes, cudaMemcpyDeviceToHost, st));
    CU(wait_stream(ctx, st));
    const int32_t* hr = static_cast<const int32_t*>(ctx->h_bidir.p);
    std::vector<tsu::BidirSeg> next;
    for (int64_t j = 0; j < c; ++j) {
      const tsu::BidirSeg& s = cur[(size_t)j];
      int32_t& ps = pst[(size_t)s.pair];
      if (ps != tsu::kPairOk) continue;
      const int32_t T = hr[j], comp = hr[c + j], k = hr[2 * c + j], h = hr[3 * c + j], sst = hr[4 * c + j];
      if (sst != tsu::kPairOk || T < 0) {
        ps = sst != tsu::kPairOk ? sst : tsu::kPairInternal;
        continue;
      }
      if (s.m == 0 && s.n == 0) continue;
      const int32_t v = h - k, left = v + h, whole = s.m + s.n;
      if (T <= base || left <= 0 || left >= whole) {
        // a leaf starts in the first launch whose cap exceeds its crossing
        // total + 2 (o + e) + 4
        int cap = base + 2 * rp.go + 4;
        while (cap < T + 2 * rp.go + 4) cap *= 2;
        add_leaf(s, cap);
        continue;
      }
      next.push_back(tsu::BidirSeg{s.pair, s.v0, s.h0, v, h, s.begin, comp});
      next.push_back(tsu::BidirSeg{s.pair, s.v0 + v, s.h0 + h, s.m - v, s.n - h, comp, s.end});
    }
    cur.swap(next);
  }

  // ---- the recursion's leaves, in launches of growing step caps
  const int64_t max_smax = (int64_t)(std::max(bi.max_m, 0) + std::max(bi.max_n, 0)) * (rp.rm - 1) + 2 * rp.go + 1;
  for (;;) {
    int scap = INT32_MAX;
    const int64_t L = (int64_t)leaves.size();
    for (int64_t i = 0; i < L; ++i)
      if (lstat[(size_t)i] == tsu::kPairScratch && pst[(size_t)leaves[(size_t)i].pair] == tsu::kPairOk)
        scap = std::min(scap, lcap[(size_t)i]);
    if (scap == INT32_MAX) break;
    if (scap > 2 * max_smax + 2 * (base + 2 * rp.go + 4))
      return set_err(ctx, TSU_EINTERNAL, "segment kernel: step cap runaway");
    std::vector<int64_t> pick;
    for (int64_t i = 0; i < L; ++i)
      if (lstat[(size_t)i] == tsu::kPairScratch && pst[(size_t)leaves[(size_t)i].pair] == tsu::kPairOk &&
          lcap[(size_t)i] == scap)
        pick.push_back(i);
    rc = launch_leaves(pick, scap);
    if (rc) return rc;
    for (int64_t i : pick) {
      const int32_t s = lstat[(size_t)i];
      if (s == tsu::kPairScratch)
        lcap[(size_t)i] = 2 * scap;
      else if (s != tsu::kPairOk)
        pst[(size_t)leaves[(size_t)i].pair] = s;
    }
  }

  // ---- leaves in pair and position order: a counting sort by pair, then
  // each pair's few leaves by position; join their runs
  const int64_t L = (int64_t)leaves.size();
  std::vector<int64_t> first((size_t)n + 1, 0);
  for (const tsu::BidirSeg& s : leaves) first[(size_t)s.pair + 1]++;
  for (int64_t i = 0; i < n; ++i) first[(size_t)i + 1] += first[(size_t)i];
  std::vector<int64_t> idx((size_t)L);
  {
    std::vector<int64_t> fill(first.begin(), first.end() - 1);
    for (int64_t i = 0; i < L; ++i) idx[(size_t)fill[(size_t)leaves[(size_t)i].pair]++] = i;
  }
  for (int64_t p = 0; p < n; ++p)
    if (first[(size_t)p + 1] - first[(size_t)p] > 1)
      std::sort(idx.begin() + first[(size_t)p], idx.begin() + first[(size_t)p + 1], [&](int64_t a, int64_t b) {
        return leaves[(size_t)a].v0 + leaves[(size_t)a].h0 < leaves[(size_t)b].v0 + leaves[(size_t)b].h0;
      });
  if ((rc = grow(ctx, ctx->b_boff, sizeof(int64_t) * std::max<int64_t>(L, 1)))) return rc;
  if ((rc = grow(ctx, ctx->b_blen, 2 * sizeof(int32_t) * std::max<int64_t>(L, 1)))) return rc;
  int32_t* d_rlen = P<int32_t>(ctx->b_blen);
  if ((rc = host_grow(ctx, ctx->h_bidir,
                      sizeof(int64_t) * (size_t)(L + n + 1) + sizeof(int32_t) * (size_t)(L + n) + 64)))
    return rc;
  {
    char* hb = static_cast<char*>(ctx->h_bidir.p);
    int64_t* h_off = reinterpret_cast<int64_t*>(hb);
    int64_t* h_first = h_off + L;
    int32_t* h_rl = reinterpret_cast<int32_t*>(h_first + n + 1);
    int32_t* h_ps = h_rl + L;
    for (int64_t j = 0; j < L; ++j) {
      const size_t i = (size_t)idx[(size_t)j];
      h_off[j] = roff[i];
      h_rl[j] = lstat[i] == tsu::kPairOk ? lruns[i] : 0;
    }
    for (int64_t i = 0; i <= n; ++i) h_first[i] = first[(size_t)i];
    for (int64_t i = 0; i < n; ++i) h_ps[i] = pst[(size_t)i];
    if (L) {
      CU(cudaMemcpyAsync(ctx->b_boff.p, h_off, sizeof(int64_t) * L, cudaMemcpyHostToDevice, st));
      CU(cudaMemcpyAsync(d_rlen, h_rl, sizeof(int32_t) * L, cudaMemcpyHostToDevice, st));
    }
    CU(cudaMemcpyAsync(ctx->b_bfirst.p, h_first, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(d_status, h_ps, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
  }
  if (!ctx->b_bruns.p && (rc = grow(ctx, ctx->b_bruns, 256))) return rc;
  CU(cudaEventRecord(ctx->ev[5], st));
  const int rblocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sms * 8);
  int64_t* d_len = P<int64_t>(ctx->b_clen64);
  tsu::launch_seg_runs(false, rblocks, st, n, pre_st, pre_off, pre_len, P<int64_t>(ctx->b_bfirst),
                       P<int64_t>(ctx->b_boff), d_rlen, P<uint32_t>(ctx->b_bruns), d_status, d_len, nullptr, nullptr);
  CU(cudaMemsetAsync(d_len + n, 0, sizeof(int64_t), st));
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, d_len, d_out_off, (int)(n + 1), st);
  if ((rc = grow(ctx, ctx->b_scan_tmp, tb))) return rc;
  CU(cub::DeviceScan::ExclusiveSum(ctx->b_scan_tmp.p, tb, d_len, d_out_off, (int)(n + 1), st));
  int64_t* h_total = reinterpret_cast<int64_t*>(static_cast<char*>(ctx->h_scalars.p) + 32);
  CU(cudaMemcpyAsync(h_total, d_out_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  char* hc = static_cast<char*>(ctx->h_scalars.p);
  CU(cudaMemcpyAsync(hc, d_cnt + 1, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CU(wait_stream(ctx, st));
  ctx->timing.cells = (int64_t)reinterpret_cast<const unsigned long long*>(hc)[0];
  ctx->timing.steps = (int64_t)reinterpret_cast<const unsigned long long*>(hc)[1];
  const int64_t total = *h_total;
  if (runs_needed) *runs_needed = total;
  if (!d_out_runs) {
    DevBuf& ob = out_buf ? *out_buf : ctx->b_out;
    if ((rc = grow(ctx, ob, sizeof(uint32_t) * (size_t)std::max<int64_t>(total, 1)))) return rc;
    d_out_runs = P<uint32_t>(ob);
    out_cap = total;
    if (out_used) *out_used = d_out_runs;
  }
  if (total > out_cap) return TSU_EOVERFLOW;
  tsu::launch_seg_runs(true, rblocks, st, n, pre_st, pre_off, pre_len, P<int64_t>(ctx->b_bfirst),
                       P<int64_t>(ctx->b_boff), d_rlen, P<uint32_t>(ctx->b_bruns), d_status, nullptr, d_out_off,
                       d_out_runs);
  CU(cudaGetLastError());
  ctx->timing.kernel_launches += 3;
  CU(cudaEventRecord(ctx->ev[6], st));
  ctx->passlog = log;
  return TSU_OK;
}

// Core: inputs resident on the device (sv).  Writes score/status (device)
// and, for CIGARs, compacts runs into out_runs with offsets out_off
// (device, n+1 entries).  *runs_needed receives the total.
// When d_out_runs is null the runs go to the context buffer *out_buf (b_out
// unless given; grown to fit) and *out_used receives its address.
// h_plen/h_tlen: the same lengths in host memory (used to plan the passes).
//
// Pairs are split into length bands (tsu::length_band of max(m, n)), each
// band ordered longest first (a counting sort by floor(log2(m + n))) and
// started at its rung (the context's band table, tsu_set_band_start), with
// scratch sized for its longest pair, so short pairs run many to an SM and
// long ones get warp groups.  The call's fixed launch sequence -- word
// counts, scan, packing, pass orders up, counters cleared, the first pass of
// every band (longest band first), counters down -- is one CUDA graph; pairs
// that outgrew their band's first rung then climb the retry ladder, band by
// band, in passes the host plans from their lengths.  TSU_ONE_WARP keeps one
// band in input order starting at one warp per pair.
int run_device(tsu_ctx* ctx, const tsu::SeqView& sv, bool want_cigar, int32_t* d_score, int32_t* d_status,
               uint32_t* d_out_runs, int64_t out_cap, int64_t* d_out_off, int64_t* runs_needed, BatchInfo bi,
               const int32_t* h_plen, const int32_t* h_tlen, uint32_t** out_used = nullptr,
               DevBuf* out_buf = nullptr) {
  const int64_t n = sv.n;
  cudaStream_t st = ctx->stream;
  int rc;
  if (n == 0) {
    if (runs_needed) *runs_needed = 0;
    if (want_cigar && d_out_off) CU(cudaMemsetAsync(d_out_off, 0, sizeof(int64_t), st));
    return TSU_OK;
  }
  if (ctx->bidir) {
    if (want_cigar)
      return run_bidir_cigar(ctx, sv, d_score, d_status, d_out_runs, out_cap, d_out_off, runs_needed, bi, h_plen,
                             h_tlen, out_used, out_buf);
    if (runs_needed) *runs_needed = 0;
    return run_bidir(ctx, sv, d_score, d_status, bi, h_plen, h_tlen);
  }
  // ---- buffers (all grown before the launch sequence is captured)
  if ((rc = grow(ctx, ctx->b_words_cnt, sizeof(int64_t) * 2 * n))) return rc;
  if ((rc = grow(ctx, ctx->b_woff, sizeof(int64_t) * 2 * n))) return rc;
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, P<int64_t>(ctx->b_words_cnt), P<int64_t>(ctx->b_woff), (int)(2 * n), st);
  if ((rc = grow(ctx, ctx->b_scan_tmp, tmp_bytes))) return rc;
  if ((rc = grow(ctx, ctx->b_words, sizeof(uint64_t) * (size_t)bi.total_words))) return rc;
  if ((rc = grow(ctx, ctx->b_nonacgt, (size_t)(2 * n)))) return rc;
  const tsu::PackView pk{P<uint64_t>(ctx->b_words), P<int64_t>(ctx->b_woff), P<uint8_t>(ctx->b_nonacgt)};
  if ((rc = grow(ctx, ctx->b_cpos, sizeof(int64_t) * n))) return rc;
  if ((rc = grow(ctx, ctx->b_clen, sizeof(int32_t) * n))) return rc;
  if ((rc = grow(ctx, ctx->b_retry, sizeof(int32_t) * n))) return rc;
  if ((rc = grow(ctx, ctx->b_order, sizeof(int32_t) * n))) return rc;
  // counters: +16 arena cursor, +24 work (cells, steps, extension bases), +64 + 8b queue head
  // and retry count of band slot b
  constexpr size_t kCounterBytes = 64 + 8 * tsu::kBands;
  if ((rc = grow(ctx, ctx->b_counters, kCounterBytes))) return rc;
  const int min_pen = ctx->rp.min_pen();
  int64_t arena_cap = 0;
  if (want_cigar) {
    arena_cap = tsu::arena_runs(ctx->rp, n, bi.max_m, bi.max_n, ctx->err_hint);
    // the wavefront scratch of an earlier call is regrown for this call's
    // passes anyway: drop it rather than let it shrink the arena
    if (ctx->held() + sizeof(uint32_t) * (size_t)arena_cap > ctx->budget) release(ctx, ctx->b_scratch);
    size_t room = ctx->budget > ctx->held() ? ctx->budget - ctx->held() : 0;
    arena_cap = std::min<int64_t>(arena_cap, (int64_t)(room / 8));  // leave half for scratch
    if ((rc = grow(ctx, ctx->b_arena, sizeof(uint32_t) * (size_t)std::max<int64_t>(arena_cap, 1024)))) return rc;
    arena_cap = (int64_t)(ctx->b_arena.cap / sizeof(uint32_t));
    // run lengths of the compaction, allocated before the passes' scratch
    if ((rc = grow(ctx, ctx->b_clen64, sizeof(int64_t) * (n + 1)))) return rc;
  }
  // The compacted runs (at most the arena's, at most m + n per pair) are
  // allocated after the passes: each pass's scratch leaves room for them.
  int64_t len_sum = 0;
  for (int64_t i = 0; h_plen && i < n; ++i) len_sum += (int64_t)h_plen[i] + h_tlen[i];
  if (!h_plen) len_sum = n * ((int64_t)bi.max_m + bi.max_n);
  auto out_reserve = [&]() -> size_t {
    if (!want_cigar || d_out_runs) return 0;
    const DevBuf& ob = out_buf ? *out_buf : ctx->b_out;
    const size_t need = (sizeof(uint32_t) * (size_t)std::min<int64_t>(arena_cap, len_sum + 1) + 255) & ~(size_t)255;
    return (need > ob.cap ? need - ob.cap : 0) + 1024;  // + the scratch carving's alignment
  };
  char* const d_cnt = P<char>(ctx->b_counters);
  unsigned long long* const d_cursor = reinterpret_cast<unsigned long long*>(d_cnt + 16);
  unsigned long long* const d_work = reinterpret_cast<unsigned long long*>(d_cnt + 24);
  char* const h_cnt = static_cast<char*>(ctx->h_scalars.p);  // page-locked copy of the counters

  // ---- bands: pairs, first rung and first pass plan, longest band first
  struct BandRun {
    int band = 0, slot = 0;
    int64_t off = 0, n = 0;  // slice of the pass order / retry list
    BatchInfo bi;
    tsu::PassChoice pc;
    double hint = 0;
    Pass ps;
  };
  BandSplit split;
  if (!ctx->one_warp && h_plen) split_bands(n, h_plen, h_tlen, &split);
  const bool all_pairs = ctx->one_warp || !h_plen || split.uniform;  // one band of every pair, input order
  std::vector<BandRun> runs;
  std::vector<int32_t> order_all;
  if (all_pairs) {
    BandRun r;
    r.n = n;
    r.bi = bi;
    r.pc = tsu::PassChoice{tsu::kModeShared, 1};
    if (!ctx->one_warp && h_plen) r.pc = tsu::band_start_in(ctx->band_start, split.uniform_band, std::max(bi.max_m, bi.max_n));
    runs.push_back(r);
  } else {
    for (int band = tsu::kBands - 1; band >= 0; --band) {
      const std::vector<int32_t>& bp = split.bands[(size_t)band];
      if (bp.empty()) continue;
      BandRun r;
      r.band = band;
      r.off = (int64_t)order_all.size();
      r.n = (int64_t)bp.size();
      r.bi.n = r.n;
      for (int32_t i : bp) {
        r.bi.max_m = std::max(r.bi.max_m, h_plen[i]);
        r.bi.max_n = std::max(r.bi.max_n, h_tlen[i]);
      }
      r.pc = tsu::band_start_in(ctx->band_start, band, std::max(r.bi.max_m, r.bi.max_n));
      order_all.insert(order_all.end(), bp.begin(), bp.end());
      runs.push_back(r);
    }
  }
  {
    // first passes run one after the other in one scratch buffer sized for
    // the largest; each is planned within what the other buffers leave
    const size_t fixed = ctx->held() - ctx->b_scratch.cap + out_reserve();
    const size_t avail = ctx->budget > fixed ? ctx->budget - fixed : 0;
    size_t need = 0;
    for (size_t k = 0; k < runs.size(); ++k) {
      BandRun& r = runs[k];
      r.slot = (int)k;
      r.hint = ctx->err_hint;
      if (ctx->fit_start && !ctx->one_warp)
        r.pc = tsu::fit_start(r.pc, ctx->rp, r.bi.max_m, r.bi.max_n, r.hint, ctx->smem_optin);
      if ((rc = plan_pass_within(ctx, r.bi, r.n, r.pc, r.hint, want_cigar, avail, &r.ps))) return rc;
      need = std::max(need, scratch_bytes(r.ps, want_cigar));
    }
    if (need > ctx->b_scratch.cap) {
      release(ctx, ctx->b_scratch);
      if ((rc = grow(ctx, ctx->b_scratch, need))) return rc;
    }
  }
  if (!order_all.empty()) {
    if ((rc = host_grow(ctx, ctx->h_list, sizeof(int32_t) * order_all.size()))) return rc;
    memcpy(ctx->h_list.p, order_all.data(), sizeof(int32_t) * order_all.size());
  }
  auto align_args = [&](const Pass& ps, const int32_t* order, int64_t n_order, int slot, int32_t* retry) {
    tsu::AlignArgs a{};
    a.seq = sv;
    a.pk = pk;
    a.order = order;
    a.n_order = n_order;
    a.pen = ctx->rp;
    a.g = ctx->g;
    a.ring_w = ps.g.ring_w;
    a.seq_cap = ps.g.seq_cap;
    carve_scratch(ctx, ps, want_cigar, &a);
    a.ring_stride = ps.g.ring_ints;
    a.hist_cap = ps.g.hist_cap;
    a.table_cap = ps.g.table_cap;
    a.score = d_score;
    a.status = d_status;
    a.arena = want_cigar ? P<uint32_t>(ctx->b_arena) : nullptr;
    a.arena_cursor = d_cursor;
    a.arena_cap = arena_cap;
    a.cig_pos = P<int64_t>(ctx->b_cpos);
    a.cig_len = P<int32_t>(ctx->b_clen);
    a.queue = reinterpret_cast<unsigned int*>(d_cnt + 64 + 8 * slot);
    a.retry = retry;
    a.retry_count = a.queue + 1;
    a.work = d_work;
    a.ef_pb = ctx->ends_free[0];
    a.ef_pe = ctx->ends_free[1];
    a.ef_tb = ctx->ends_free[2];
    a.ef_te = ctx->ends_free[3];
    return a;
  };
  std::string passlog;  // mode, warps per pair x groups : pairs @ time, per pass (for error messages)
  auto log_pass = [&](const Pass& ps, int64_t pairs) {
    passlog += (passlog.empty() ? "" : " ") + std::string(ps.g.mode == tsu::kModeShared ? "s" : "g") +
               std::to_string(ps.g.gw) + "x" + std::to_string(ps.groups) + ":" + std::to_string(pairs);
  };

  // ---- the fixed launch sequence of the call (one CUDA graph)
  rc = run_graph(ctx, st, [&]() -> int {
    CU(record(ctx, ctx->ev[2], st));
    tsu::word_count_kernel<<<std::min<int64_t>((2 * n + 255) / 256, 4096), 256, 0, st>>>(
        n, sv.pat_len, sv.txt_len, P<int64_t>(ctx->b_words_cnt));
    size_t tb = tmp_bytes;
    CU(cub::DeviceScan::ExclusiveSum(ctx->b_scan_tmp.p, tb, P<int64_t>(ctx->b_words_cnt), P<int64_t>(ctx->b_woff),
                                     (int)(2 * n), st));
    const int64_t blocks = std::min<int64_t>((2 * n + 7) / 8, (int64_t)ctx->sms * 16);
    tsu::pack_kernel<<<(int)blocks, 256, 0, st>>>(sv, pk);
    CU(cudaGetLastError());
    CU(record(ctx, ctx->ev[3], st));
    if (!order_all.empty())
      CU(cudaMemcpyAsync(P<int32_t>(ctx->b_order), ctx->h_list.p, sizeof(int32_t) * order_all.size(),
                         cudaMemcpyHostToDevice, st));
    CU(cudaMemsetAsync(d_cnt, 0, kCounterBytes, st));
    CU(record(ctx, ctx->ev[4], st));
    for (const BandRun& r : runs) {
      const tsu::AlignArgs a = align_args(r.ps, all_pairs ? nullptr : P<int32_t>(ctx->b_order) + r.off, r.n, r.slot,
                                          P<int32_t>(ctx->b_retry) + r.off);
      CU(record(ctx, ctx->bev[2 * r.slot], st));
      launch_align(ctx, want_cigar, r.ps.g.mode, r.ps.g.gw, r.ps.blocks, r.ps.threads, r.ps.smem_bytes, st, a);
      CU(cudaGetLastError());
      CU(record(ctx, ctx->bev[2 * r.slot + 1], st));
    }
    CU(cudaMemcpyAsync(h_cnt, d_cnt, kCounterBytes, cudaMemcpyDeviceToHost, st));
    return TSU_OK;
  });
  if (rc) return rc;
  ctx->timing.kernel_launches += 3 + (int64_t)runs.size();
  CU(wait_stream(ctx, st));
  std::vector<unsigned int> first_retry(runs.size());
  for (const BandRun& r : runs) {
    first_retry[(size_t)r.slot] = *reinterpret_cast<const unsigned int*>(h_cnt + 64 + 8 * r.slot + 4);
    log_pass(r.ps, r.n);
    char t[48];
    snprintf(t, sizeof t, "@%.1fms", ev_ms(ctx->bev[2 * r.slot], ctx->bev[2 * r.slot + 1]));
    passlog += t;
  }
  ctx->passlog = passlog;
  int passes = (int)runs.size();

  // ---- retry ladders: per band, the pairs that outgrew its last rung
  bool laddered = false;
  std::vector<int32_t> rlist;
  for (const BandRun& r : runs) {
    unsigned int nretry = first_retry[(size_t)r.slot];
    if (nretry == 0) continue;
    laddered = true;
    tsu::PassChoice pc = r.pc;
    double hint = r.hint;
    int last_mode = r.ps.g.mode;
    int32_t* const d_order = P<int32_t>(ctx->b_order) + r.off;  // this band's slices
    int32_t* const d_retry = P<int32_t>(ctx->b_retry) + r.off;
    unsigned int* const d_slot = reinterpret_cast<unsigned int*>(d_cnt + 64 + 8 * r.slot);
    const int band_first_pass = passes - 1;
    for (;;) {
      ctx->timing.retried_pairs += nretry;
      if (passes - band_first_pass > 24)
        return set_err(ctx, TSU_EINTERNAL, "pairs still fail after %d passes [passes %s]", passes, passlog.c_str());
      if (last_mode == tsu::kModeGlobal && hint >= tsu::kHintCeiling)
        return set_err(ctx, TSU_ENOMEM, "%u pairs exceed the scratch one group can hold within the budget [passes %s]",
                       nretry, passlog.c_str());
      // The retry list, longest pairs first, becomes the next pass's order;
      // its lengths pick the next rung.  Global passes grow the hint.
      rlist.resize(nretry);
      if ((rc = host_grow(ctx, ctx->h_list, sizeof(int32_t) * nretry))) return rc;
      CU(cudaMemcpyAsync(ctx->h_list.p, d_retry, sizeof(int32_t) * nretry, cudaMemcpyDeviceToHost, st));
      CU(wait_stream(ctx, st));
      memcpy(rlist.data(), ctx->h_list.p, sizeof(int32_t) * nretry);
      BatchInfo pbi;
      pbi.n = nretry;
      for (int32_t i : rlist) {
        pbi.max_m = std::max(pbi.max_m, h_plen[i]);
        pbi.max_n = std::max(pbi.max_n, h_tlen[i]);
      }
      std::sort(rlist.begin(), rlist.end(),
                [&](int32_t u, int32_t v) { return (int64_t)h_plen[u] + h_tlen[u] > (int64_t)h_plen[v] + h_tlen[v]; });
      memcpy(ctx->h_list.p, rlist.data(), sizeof(int32_t) * nretry);
      CU(cudaMemcpyAsync(d_order, ctx->h_list.p, sizeof(int32_t) * nretry, cudaMemcpyHostToDevice, st));
      hint = tsu::next_hint(hint, last_mode == tsu::kModeGlobal);
      pc = ctx->one_warp ? tsu::PassChoice{tsu::kModeGlobal, 1}
                         : tsu::next_pass(pc, ctx->rp, pbi.max_m, pbi.max_n, ctx->smem_optin);
      if (want_cigar) {
        unsigned long long* h_used = reinterpret_cast<unsigned long long*>(h_cnt + 16);
        CU(cudaMemcpyAsync(h_used, d_cursor, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        CU(wait_stream(ctx, st));
        const unsigned long long used = *h_used;
        const int64_t maxlen = std::max(pbi.max_m, pbi.max_n);
        const int64_t need =
            (int64_t)used + (int64_t)nretry * (2 * tsu::hint_score(ctx->rp, maxlen, hint) / min_pen + 1);
        if (need > arena_cap) {
          // keep the runs written so far: grow by copy
          DevBuf nb;
          const size_t bytes = (sizeof(uint32_t) * (size_t)need + 255) & ~(size_t)255;
          // the last pass's scratch is regrown for the next one: free it first
          if (ctx->held() + bytes > ctx->budget) release(ctx, ctx->b_scratch);
          if (ctx->held() + bytes > ctx->budget) {
            ctx->need_bytes = ctx->held() + bytes;
            return set_err(ctx, TSU_ENOMEM, "CIGAR arena exceeds budget");
          }
          CU(cudaMallocFromPoolAsync(&nb.p, bytes, ctx->pool, st));
          nb.cap = bytes;
          const int64_t keep = std::min<int64_t>((int64_t)used, arena_cap);
          CU(cudaMemcpyAsync(nb.p, ctx->b_arena.p, sizeof(uint32_t) * (size_t)keep, cudaMemcpyDeviceToDevice, st));
          ctx->peak_held = std::max(ctx->peak_held, ctx->held() + nb.cap);
          release(ctx, ctx->b_arena);
          ctx->b_arena = nb;
          arena_cap = need;
        }
      }
      Pass ps;
      if ((rc = plan_pass(ctx, pbi, nretry, pc, hint, want_cigar, out_reserve(), &ps))) return rc;
      log_pass(ps, nretry);
      const size_t need = scratch_bytes(ps, want_cigar);
      if (need > ctx->b_scratch.cap) {
        release(ctx, ctx->b_scratch);  // plan_pass counted the scratch as free
        if ((rc = grow(ctx, ctx->b_scratch, need)))
          return set_err(ctx, rc, "%s [passes %s]", ctx->err.c_str(), passlog.c_str());
      }
      CU(cudaMemsetAsync(d_slot, 0, 8, st));  // queue head + retry count
      const tsu::AlignArgs a = align_args(ps, d_order, nretry, r.slot, d_retry);
      CU(cudaEventRecord(ctx->pev[0], st));
      launch_align(ctx, want_cigar, ps.g.mode, ps.g.gw, ps.blocks, ps.threads, ps.smem_bytes, st, a);
      ctx->timing.kernel_launches++;
      CU(cudaGetLastError());
      CU(cudaEventRecord(ctx->pev[1], st));
      ++passes;
      last_mode = ps.g.mode;
      unsigned int* h_nretry = reinterpret_cast<unsigned int*>(h_cnt + 64 + 8 * r.slot + 4);
      CU(cudaMemcpyAsync(h_nretry, d_slot + 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
      CU(wait_stream(ctx, st));
      nretry = *h_nretry;
      char t[48];
      snprintf(t, sizeof t, "@%.1fms", ev_ms(ctx->pev[0], ctx->pev[1]));
      passlog += t;
      ctx->passlog = passlog;
      if (nretry == 0) break;
    }
  }
  CU(cudaEventRecord(ctx->ev[5], st));
  if (laddered) {
    CU(cudaMemcpyAsync(h_cnt + 24, d_work, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CU(wait_stream(ctx, st));
  }
  ctx->timing.cells = (int64_t)reinterpret_cast<const unsigned long long*>(h_cnt + 24)[0];
  ctx->timing.steps = (int64_t)reinterpret_cast<const unsigned long long*>(h_cnt + 24)[1];
  ctx->timing.ext_bases = (int64_t)reinterpret_cast<const unsigned long long*>(h_cnt + 24)[2];

  // ---- CIGAR compaction
  if (want_cigar) {
    if ((rc = grow(ctx, ctx->b_clen64, sizeof(int64_t) * (n + 1)))) return rc;
    tsu::cig_len64_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(
        n, P<int32_t>(ctx->b_clen), d_status, P<int64_t>(ctx->b_clen64));
    CU(cudaMemsetAsync(P<int64_t>(ctx->b_clen64) + n, 0, sizeof(int64_t), st));
    ctx->timing.kernel_launches++;
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, P<int64_t>(ctx->b_clen64), d_out_off, (int)(n + 1), st);
    if ((rc = grow(ctx, ctx->b_scan_tmp, tb))) return rc;
    CU(cub::DeviceScan::ExclusiveSum(ctx->b_scan_tmp.p, tb, P<int64_t>(ctx->b_clen64), d_out_off, (int)(n + 1), st));
    ctx->timing.kernel_launches++;
    int64_t* h_total = reinterpret_cast<int64_t*>(static_cast<char*>(ctx->h_scalars.p) + 32);
    CU(cudaMemcpyAsync(h_total, d_out_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CU(wait_stream(ctx, st));
    const int64_t total = *h_total;
    if (runs_needed) *runs_needed = total;
    if (!d_out_runs) {
      DevBuf& ob = out_buf ? *out_buf : ctx->b_out;
      if ((rc = grow(ctx, ob, sizeof(uint32_t) * (size_t)std::max<int64_t>(total, 1)))) return rc;
      d_out_runs = P<uint32_t>(ob);
      out_cap = total;
      if (out_used) *out_used = d_out_runs;
    }
    if (total > out_cap) return TSU_EOVERFLOW;
    const int64_t blocks = std::min<int64_t>((n + 7) / 8, (int64_t)ctx->sms * 16);
    tsu::compact_kernel<<<(int)blocks, 256, 0, st>>>(n, P<uint32_t>(ctx->b_arena), P<int64_t>(ctx->b_cpos), d_out_off,
                                                    d_out_runs);
    ctx->timing.kernel_launches++;
    CU(cudaGetLastError());
  }
  CU(cudaEventRecord(ctx->ev[6], st));
  return TSU_OK;
}

// Chunks of the host-buffer pipeline (tsu_align_batch): 131072 pairs or
// more each, at most 8.
int chunk_count(int64_t n) { return (int)std::min<int64_t>(8, std::max<int64_t>(1, n / 131072)); }

int check_batch_host(tsu_ctx* ctx, const tsu_batch* b, BatchInfo* bi, int64_t* pat_bytes, int64_t* txt_bytes) {
  if (!b || b->num_pairs < 0) return set_err(ctx, TSU_EINVAL, "null batch or negative num_pairs");
  if (b->num_pairs > INT32_MAX) return set_err(ctx, TSU_EINVAL, "num_pairs > INT32_MAX");
  if (b->num_pairs && (!b->pattern || !b->pattern_off || !b->pattern_len || !b->text || !b->text_off || !b->text_len))
    return set_err(ctx, TSU_EINVAL, "null sequence pointer");
  int64_t pe = 0, te = 0, words = 0;
  int32_t mm = 0, mn = 0;
  for (int64_t i = 0; i < b->num_pairs; ++i) {
    const int32_t m = b->pattern_len[i], n = b->text_len[i];
    if (m < 0 || n < 0 || m > max_len(ctx) || n > max_len(ctx) || b->pattern_off[i] < 0 || b->text_off[i] < 0)
      return set_err(ctx, TSU_EINVAL, "pair %lld: bad length/offset", (long long)i);
    pe = std::max(pe, b->pattern_off[i] + m);
    te = std::max(te, b->text_off[i] + n);
    mm = std::max(mm, m);
    mn = std::max(mn, n);
    words += tsu::packed_words(m) + tsu::packed_words(n);
  }
  bi->n = b->num_pairs;
  bi->max_m = mm;
  bi->max_n = mn;
  bi->total_words = words;
  *pat_bytes = pe;
  *txt_bytes = te;
  return TSU_OK;
}

// Per-pair statuses -> call status.
int collect_status(tsu_ctx* ctx, const int32_t* hs, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    if (hs[i] != tsu::kPairOk)
      return set_err(ctx, hs[i] == tsu::kPairInternal ? TSU_EINTERNAL : TSU_ENOMEM, "pair %lld status %d",
                     (long long)i, hs[i]);
  return TSU_OK;
}

}  // namespace

// ===========================================================================
// Engine calls of the request server (tsu_engine_internal.h)
// ===========================================================================
namespace tsu {
namespace engine {

int predict_bytes(tsu_ctx* ctx, const BatchShape& sh, uint32_t flags, double hint, size_t* full, size_t* min) {
  if (!ctx || sh.n < 0 || (sh.n && (!sh.plen || !sh.tlen)) || !full || !min) return TSU_EINVAL;
  if (hint <= 0) hint = ctx->err_hint;
  const bool want_cigar = !(flags & TSU_SCORE_ONLY);
  const bool one_warp = (flags & TSU_ONE_WARP) != 0;
  const int64_t n = sh.n;
  auto r = [](size_t b) { return (std::max<size_t>(b, 16) + 255) & ~(size_t)255; };
  auto scan_tmp = [](int64_t items) {
    size_t t = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t, (const int64_t*)nullptr, (int64_t*)nullptr, (int)std::max<int64_t>(items, 1));
    return t;
  };
  const int K = chunk_count(n);
  // buffers of the whole call (tsu_align_batch)
  size_t call = r((size_t)sh.pattern_bytes) + r((size_t)sh.text_bytes) + 2 * r(8 * (size_t)n) +
                4 * r(4 * (size_t)n) + (want_cigar ? r(8 * (size_t)(n + K + 1)) : 0);
  if (flags & TSU_BIDIRECTIONAL) {
    // bidirectional mode, per chunk: packing forward and reversed, a level's
    // segments and cuts, for CIGARs the leaves' bookkeeping and runs (at most
    // m + n per pair); scratch: the breakpoint rings of the largest size
    // class (groups x 2 directions x ring depth x 4 x (m + n + 3) int32) or
    // the leaf warps' history at the base step cap, whichever is larger
    const tsu::Pen rp = bidir_pen(ctx);
    size_t chunk_max = 0, scratch_full = 0, scratch_min = 0;
    const int cap0 = tsu::bidir_base(rp) + 2 * rp.go + 4;
    for (int c = 0; c < K; ++c) {
      const int64_t c0 = n * c / K, nc = n * (c + 1) / K - c0;
      if (nc == 0) continue;
      int64_t words = 0, len_sum = 0;
      int32_t cls_bases[3] = {0, 0, 0};
      int64_t cls_n[3] = {0, 0, 0};
      for (int64_t i = 0; i < nc; ++i) {
        const int32_t m = sh.plen[c0 + i], t = sh.tlen[c0 + i];
        words += tsu::packed_words(m) + tsu::packed_words(t);
        len_sum += (int64_t)m + t;
        const int gw = bidir_gw(std::max(m, t)), k = gw == 1 ? 0 : (gw == 4 ? 1 : 2);
        cls_bases[k] = std::max(cls_bases[k], m + t);
        cls_n[k]++;
      }
      size_t f = 2 * r(16 * (size_t)nc) + 2 * r(8 * (size_t)words) + 2 * r(2 * (size_t)nc) +
                 r(sizeof(tsu::BidirSeg) * (size_t)nc) + r(20 * (size_t)nc) + r(64) + r(scan_tmp(2 * nc));
      if (want_cigar) {
        // leaves per pair: about 2 T / base for a crossing total T, here
        // the hint's score of the longest pair
        const int32_t maxb = std::max(cls_bases[0], std::max(cls_bases[1], cls_bases[2]));
        const int64_t leaves =
            nc * std::max<int64_t>(1, 2 * tsu::hint_score(rp, std::max(1, maxb / 2), hint) / tsu::bidir_base(rp));
        f += 2 * r(8 * (size_t)(nc + 1)) + r(sizeof(tsu::BidirSeg) * (size_t)leaves) + r(16 * (size_t)leaves) +
             2 * r(4 * (size_t)(len_sum + 1)) + r(scan_tmp(nc + 1));
      }
      chunk_max = std::max(chunk_max, f);
      const int gws[3] = {1, 4, 16};
      for (int k = 0; k < 3; ++k) {
        if (!cls_n[k]) continue;
        const size_t ring = (size_t)tsu::bidir_ring_bytes(gws[k]) * 2 * (size_t)rp.rm * 4 * ((size_t)cls_bases[k] + 3);
        const int64_t groups = std::min<int64_t>(cls_n[k], (int64_t)ctx->sms * (gws[k] <= 4 ? 5 * (4 / gws[k]) : 1));
        scratch_full = std::max(scratch_full, (size_t)groups * ring);
        scratch_min = std::max(scratch_min, ring);
      }
      if (want_cigar) {
        const int32_t bases = std::max(cls_bases[0], std::max(cls_bases[1], cls_bases[2]));
        const size_t per_warp = sizeof(int32_t) * (size_t)(3 * tsu::seg_hist_cap(cap0, bases) + 9 * (int64_t)cap0);
        scratch_full = std::max(scratch_full, per_warp * (size_t)std::min<int64_t>(nc, (int64_t)ctx->sms * 24));
        scratch_min = std::max(scratch_min, per_warp * 4);
      }
    }
    const size_t slack = 64 << 10;
    *full = call + chunk_max + scratch_full + slack;
    *min = call + chunk_max + scratch_min + slack;
    return TSU_OK;
  }
  // buffers of a chunk (run_device): reused chunk after chunk, so the largest
  // chunk sets them; scratch: the largest first pass of any band
  size_t chunk_max = 0, scratch_full = 0, scratch_min = 0;
  for (int c = 0; c < K; ++c) {
    const int64_t c0 = n * c / K, nc = n * (c + 1) / K - c0;
    if (nc == 0) continue;
    const int32_t* pl = sh.plen + c0;
    const int32_t* tl = sh.tlen + c0;
    BatchInfo ci;
    ci.n = nc;
    int64_t len_sum = 0;
    for (int64_t i = 0; i < nc; ++i) {
      ci.max_m = std::max(ci.max_m, pl[i]);
      ci.max_n = std::max(ci.max_n, tl[i]);
      ci.total_words += tsu::packed_words(pl[i]) + tsu::packed_words(tl[i]);
      len_sum += (int64_t)pl[i] + tl[i];
    }
    size_t f = 2 * r(16 * (size_t)nc) + r(8 * (size_t)ci.total_words) + r(2 * (size_t)nc) + r(8 * (size_t)nc) +
               3 * r(4 * (size_t)nc) + r(64);
    size_t tmp = scan_tmp(2 * nc);
    if (want_cigar) {
      const int64_t arena = std::max<int64_t>(tsu::arena_runs(ctx->rp, nc, ci.max_m, ci.max_n, hint), 1024);
      const int64_t out_runs = std::min<int64_t>(arena, len_sum + 1);
      f += r(4 * (size_t)arena) + r(8 * (size_t)(nc + 1)) + (K > 1 ? 2 : 1) * r(4 * (size_t)out_runs);
      tmp = std::max(tmp, scan_tmp(nc + 1));
    }
    chunk_max = std::max(chunk_max, f + r(tmp));
    BandSplit split;
    if (!one_warp) split_bands(nc, pl, tl, &split);
    const bool all_pairs = one_warp || split.uniform;
    for (int band = 0; band < tsu::kBands; ++band) {
      if (all_pairs && band != 0) break;
      if (!all_pairs && split.bands[(size_t)band].empty()) continue;
      BatchInfo pbi = ci;
      int64_t np = nc;
      tsu::PassChoice pc{tsu::kModeShared, 1};
      if (all_pairs) {
        if (!one_warp) pc = tsu::band_start_in(ctx->band_start, split.uniform_band, std::max(ci.max_m, ci.max_n));
      } else {
        const std::vector<int32_t>& bp = split.bands[(size_t)band];
        pbi = BatchInfo{};
        np = pbi.n = (int64_t)bp.size();
        for (int32_t i : bp) {
          pbi.max_m = std::max(pbi.max_m, pl[i]);
          pbi.max_n = std::max(pbi.max_n, tl[i]);
        }
        pc = tsu::band_start_in(ctx->band_start, band, std::max(pbi.max_m, pbi.max_n));
      }
      if (ctx->fit_start && !one_warp)
        pc = tsu::fit_start(pc, ctx->rp, pbi.max_m, pbi.max_n, hint, ctx->smem_optin);
      Pass ps;
      const int rc = plan_pass_within(ctx, pbi, np, pc, hint, want_cigar, SIZE_MAX / 4, &ps);
      if (rc) return rc;
      const size_t per = group_scratch_bytes(ps.g);
      scratch_full = std::max(scratch_full, (size_t)ps.groups * per);
      scratch_min = std::max(scratch_min, per);
    }
  }
  const size_t slack = 64 << 10;  // 256-byte rounding of the buffers
  *full = call + chunk_max + scratch_full + slack;
  *min = call + chunk_max + scratch_min + slack;
  return TSU_OK;
}

int make_spec(int metric, const int32_t* pen, int count, Spec* out) {
  static const int kCount[5] = {0, 0, 2, 3, 5};  // penalties per TSU_METRIC_*
  if (!out || metric < TSU_METRIC_INDEL || metric > TSU_METRIC_GAP_AFFINE_2P) return TSU_EINVAL;
  if (count != kCount[metric] || (count && !pen)) return TSU_EINVAL;
  auto in = [](int32_t v, int32_t lo) { return v >= lo && v <= (1 << 20); };
  Spec s;
  s.metric = metric;
  switch (metric) {
    case TSU_METRIC_INDEL: s.x = 3; s.e = 1; break;  // a mismatch (3) never beats D + I (2)
    case TSU_METRIC_EDIT: s.x = 1; s.e = 1; break;
    case TSU_METRIC_GAP_LINEAR:
      if (!in(pen[0], 1) || !in(pen[1], 1)) return TSU_EINVAL;
      s.x = pen[0];
      s.e = pen[1];
      break;
    case TSU_METRIC_GAP_AFFINE_2P:
      if (!in(pen[3], 0) || !in(pen[4], 1)) return TSU_EINVAL;
      s.o2 = pen[3];
      s.e2 = pen[4];
      [[fallthrough]];
    default:
      if (!in(pen[0], 1) || !in(pen[1], 0) || !in(pen[2], 1)) return TSU_EINVAL;
      s.x = pen[0];
      s.o = pen[1];
      s.e = pen[2];
      break;
  }
  *out = s;
  return TSU_OK;
}

int create(const Spec& spec, const tsu_config* cfg, bool single_stream, tsu_ctx** out) {
  tsu_ctx* ctx = nullptr;
  if (!out) return TSU_EINVAL;
  *out = nullptr;
  ctx = new tsu_ctx();
  ctx->spec = spec;
  switch (spec.metric) {
    case TSU_METRIC_GAP_AFFINE:
      ctx->rp = tsu::reduce_penalties(spec.x, spec.o, spec.e, -1, 0, &ctx->g);
      break;
    case TSU_METRIC_GAP_AFFINE_2P:
      ctx->rp = tsu::reduce_penalties(spec.x, spec.o, spec.e, spec.o2, spec.e2, &ctx->g);
      break;
    default:  // indel, edit, gap-linear
      ctx->rp = tsu::reduce_linear(spec.x, spec.e, &ctx->g);
      break;
  }
  if (ctx->rp.slots() > 4096) {
    delete ctx;
    return TSU_EINVAL;  // reduced penalties too large for the wavefront ring
  }
  ctx->device = cfg ? cfg->device : 0;
  for (int b = 0; b < tsu::kBands; ++b) ctx->band_start[b] = tsu::band_start_table(ctx->rp.dual())[b];
  ctx->err_hint = (cfg && cfg->max_error_hint > 0) ? cfg->max_error_hint : 0.2;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) {
    delete ctx;
    return TSU_EDEVICE;
  }
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) {
    delete ctx;
    return TSU_EDEVICE;
  }
  ctx->sms = prop.multiProcessorCount;
  ctx->smem_optin = (int)prop.sharedMemPerBlockOptin;
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  ctx->budget = (cfg && cfg->mem_budget) ? cfg->mem_budget : (size_t)(0.8 * (double)fr);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return TSU_EDEVICE;
  }
  for (auto& ev : ctx->ev) cudaEventCreate(&ev);
  for (auto& ev : ctx->pev) cudaEventCreate(&ev);
  for (auto& ev : ctx->fence_ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  for (int c = 0; c < 8; ++c) {
    cudaEventCreateWithFlags(&ctx->cev_up[c], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ctx->cev_done[c], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ctx->cev_down[c], cudaEventDisableTiming);
  }
  for (auto& ev : ctx->cev_t) cudaEventCreate(&ev);
  cudaEventCreateWithFlags(&ctx->wait_ev, cudaEventBlockingSync | cudaEventDisableTiming);
  if (single_stream) {
    ctx->h2d_stream = ctx->d2h_stream = ctx->stream;
  } else {
    cudaStreamCreateWithFlags(&ctx->h2d_stream, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&ctx->d2h_stream, cudaStreamNonBlocking);
  }
  ctx->pool = device_pool(ctx->device);
  for (auto& ev : ctx->bev) cudaEventCreate(&ev);
  {
    // TSU_GRAPH=0 queues the launch sequence directly instead of as a graph
    const char* gv = getenv("TSU_GRAPH");
    ctx->use_graph = !(gv && gv[0] == '0');
  }
  if (!ctx->pool || host_grow(ctx, ctx->h_scalars, 256) != TSU_OK) {
    tsu_destroy(ctx);
    return TSU_EDEVICE;
  }
  *out = ctx;
  return TSU_OK;
}

size_t held_bytes(const tsu_ctx* ctx) { return ctx ? ctx->held() : 0; }

void set_budget(tsu_ctx* ctx, size_t bytes) {
  if (ctx) ctx->budget = bytes;
}

size_t budget_bytes(const tsu_ctx* ctx) { return ctx ? ctx->budget : 0; }

void set_hint(tsu_ctx* ctx, double h) {
  if (ctx && h > 0) ctx->err_hint = h;
}

double hint(const tsu_ctx* ctx) { return ctx ? ctx->err_hint : 0.0; }

void set_fit_start(tsu_ctx* ctx, bool on) {
  if (ctx) ctx->fit_start = on;
}

void set_blocking_sync(tsu_ctx* ctx, bool on) {
  if (ctx) ctx->blocking_sync = on;
}

void set_exact_growth(tsu_ctx* ctx, bool exact) {
  if (ctx) ctx->exact_grow = exact;
}

int trim(tsu_ctx* ctx) {
  if (!ctx) return TSU_EINVAL;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return TSU_EDEVICE;
  return release_all(ctx);
}

size_t needed_bytes(const tsu_ctx* ctx) { return ctx ? ctx->need_bytes : 0; }

void prime_pool(tsu_ctx* ctx, size_t bytes) {
  if (!ctx || !bytes || cudaSetDevice(ctx->device) != cudaSuccess) return;
  void* p = nullptr;
  if (cudaMallocFromPoolAsync(&p, bytes, ctx->pool, ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  cudaFreeAsync(p, ctx->stream);
  wait_stream(ctx, ctx->stream);
}

}  // namespace engine
}  // namespace tsu

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* tsu_status_str(int s) {
  switch (s) {
    case TSU_OK: return "ok";
    case TSU_EINVAL: return "invalid argument";
    case TSU_ENOMEM: return "device memory budget exceeded";
    case TSU_EDEVICE: return "CUDA device error";
    case TSU_ETIMEOUT: return "timed out";
    case TSU_EOVERFLOW: return "output buffer too small";
    case TSU_EBUSY: return "busy / admission refused";
    case TSU_ENOTFOUND: return "not found";
    case TSU_EINTERNAL: return "internal error";
    case TSU_EIO: return "i/o error";
    case TSU_EPENDING: return "request not finished";
    default: return "unknown status";
  }
}

const char* tsu_last_error(const tsu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

const char* tsu_pass_log(const tsu_ctx* ctx) { return ctx ? ctx->passlog.c_str() : ""; }

int tsu_create_metric(int metric, const int32_t* penalties, int num_penalties, const tsu_config* cfg,
                      tsu_ctx** out) {
  if (!out) return TSU_EINVAL;
  *out = nullptr;
  tsu::engine::Spec spec;
  const int rc = tsu::engine::make_spec(metric, penalties, num_penalties, &spec);
  return rc ? rc : tsu::engine::create(spec, cfg, false, out);
}

int tsu_create(const tsu_penalties* pen, const tsu_config* cfg, tsu_ctx** out) {
  if (!pen) return TSU_EINVAL;
  const int32_t p[3] = {pen->mismatch, pen->gap_opening, pen->gap_extension};
  return tsu_create_metric(TSU_METRIC_GAP_AFFINE, p, 3, cfg, out);
}

int tsu_create_dual(const tsu_penalties2* pen, const tsu_config* cfg, tsu_ctx** out) {
  if (!pen) return TSU_EINVAL;
  const int32_t p[5] = {pen->mismatch, pen->gap_opening, pen->gap_extension, pen->gap_opening2, pen->gap_extension2};
  return tsu_create_metric(TSU_METRIC_GAP_AFFINE_2P, p, 5, cfg, out);
}

int tsu_destroy(tsu_ctx* ctx) {
  if (!ctx) return TSU_EINVAL;
  cudaSetDevice(ctx->device);
  release_all(ctx);
  for (auto& ev : ctx->ev) cudaEventDestroy(ev);
  for (auto& ev : ctx->pev) cudaEventDestroy(ev);
  for (auto& ev : ctx->fence_ev) cudaEventDestroy(ev);
  for (int c = 0; c < 8; ++c) {
    cudaEventDestroy(ctx->cev_up[c]);
    cudaEventDestroy(ctx->cev_done[c]);
    cudaEventDestroy(ctx->cev_down[c]);
  }
  for (auto& ev : ctx->cev_t) cudaEventDestroy(ev);
  if (ctx->wait_ev) cudaEventDestroy(ctx->wait_ev);
  for (auto& ev : ctx->bev) cudaEventDestroy(ev);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  for (HostBuf* hb : {&ctx->h_scalars, &ctx->h_list, &ctx->h_status, &ctx->h_bidir})
    if (hb->p) cudaFreeHost(hb->p);
  for (void* p : ctx->h_retired) cudaFreeHost(p);
  if (ctx->h2d_stream && ctx->h2d_stream != ctx->stream) cudaStreamDestroy(ctx->h2d_stream);
  if (ctx->d2h_stream && ctx->d2h_stream != ctx->stream) cudaStreamDestroy(ctx->d2h_stream);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TSU_OK;
}

int tsu_get_timing(const tsu_ctx* ctx, tsu_timing* out) {
  if (!ctx || !out) return TSU_EINVAL;
  *out = ctx->timing;
  return TSU_OK;
}

int tsu_align_batch(tsu_ctx* ctx, const tsu_batch* b, tsu_result* res, uint32_t flags) {
  if (!ctx || !res || !res->score) return ctx ? set_err(ctx, TSU_EINVAL, "null result") : TSU_EINVAL;
  const bool want_cigar = !(flags & TSU_SCORE_ONLY);
  ctx->one_warp = (flags & TSU_ONE_WARP) != 0;
  ctx->bidir = (flags & TSU_BIDIRECTIONAL) != 0;
  if (want_cigar && !res->cigar_offset) return set_err(ctx, TSU_EINVAL, "cigar_offset required");
  BatchInfo bi;
  int64_t pb = 0, tb = 0;
  int rc = check_batch_host(ctx, b, &bi, &pb, &tb);
  if (rc) return rc;
  CU(cudaSetDevice(ctx->device));
  ctx->timing = tsu_timing{};
  ctx->peak_held = ctx->held();
  const int64_t n = bi.n;
  cudaStream_t st = ctx->stream;
  // Pipeline of K chunks of consecutive pairs on three streams: chunk c's
  // sequence bytes go up on h2d_stream while chunk c-1 aligns on the compute
  // stream and chunk c-2's results come down on d2h_stream.  A chunk's bytes
  // are copied to the same offsets in the device buffers, so the offsets the
  // caller gave stay valid; chunks of non-monotonic offsets just copy a wider
  // (overlapping, identical) byte range.
  const int K = chunk_count(n);
  if ((rc = grow(ctx, ctx->b_pat, (size_t)pb))) return rc;
  if ((rc = grow(ctx, ctx->b_txt, (size_t)tb))) return rc;
  if ((rc = grow(ctx, ctx->b_poff, sizeof(int64_t) * n))) return rc;
  if ((rc = grow(ctx, ctx->b_toff, sizeof(int64_t) * n))) return rc;
  if ((rc = grow(ctx, ctx->b_plen, sizeof(int32_t) * n))) return rc;
  if ((rc = grow(ctx, ctx->b_tlen, sizeof(int32_t) * n))) return rc;
  if ((rc = grow(ctx, ctx->b_score, sizeof(int32_t) * n))) return rc;
  if ((rc = grow(ctx, ctx->b_status, sizeof(int32_t) * n))) return rc;
  if (want_cigar && (rc = grow(ctx, ctx->b_coff, sizeof(int64_t) * (n + K + 1)))) return rc;
  alloc_fence(ctx);  // the copy streams write the buffers just grown
  std::vector<int64_t> cs((size_t)K + 1);  // chunk boundaries (pairs)
  for (int c = 0; c <= K; ++c) cs[(size_t)c] = n * c / K;
  cudaEvent_t* ev_up = ctx->cev_up;  // K <= 8 (chunk_count)
  cudaEvent_t* ev_done = ctx->cev_done;
  cudaEvent_t* ev_down = ctx->cev_down;
  cudaEvent_t t_begin = ctx->cev_t[0], t_end = ctx->cev_t[1];
  if ((rc = host_grow(ctx, ctx->h_status, sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)))) return rc;
  int32_t* hs = static_cast<int32_t*>(ctx->h_status.p);
  CU(cudaEventRecord(t_begin, ctx->h2d_stream));
  int64_t h2d = 0;
  if (n) {
    CU(cudaMemcpyAsync(ctx->b_poff.p, b->pattern_off, sizeof(int64_t) * n, cudaMemcpyHostToDevice, ctx->h2d_stream));
    CU(cudaMemcpyAsync(ctx->b_toff.p, b->text_off, sizeof(int64_t) * n, cudaMemcpyHostToDevice, ctx->h2d_stream));
    CU(cudaMemcpyAsync(ctx->b_plen.p, b->pattern_len, sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->h2d_stream));
    CU(cudaMemcpyAsync(ctx->b_tlen.p, b->text_len, sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->h2d_stream));
    h2d += n * 24;
  }
  std::vector<BatchInfo> cbi((size_t)K);
  for (int c = 0; c < K; ++c) {
    int64_t p0 = INT64_MAX, p1 = 0, t0 = INT64_MAX, t1 = 0;
    BatchInfo& ci = cbi[(size_t)c];
    ci.n = cs[(size_t)c + 1] - cs[(size_t)c];
    for (int64_t i = cs[(size_t)c]; i < cs[(size_t)c + 1]; ++i) {
      const int32_t m = b->pattern_len[i], t = b->text_len[i];
      p0 = std::min(p0, b->pattern_off[i]);
      p1 = std::max(p1, b->pattern_off[i] + m);
      t0 = std::min(t0, b->text_off[i]);
      t1 = std::max(t1, b->text_off[i] + t);
      ci.max_m = std::max(ci.max_m, m);
      ci.max_n = std::max(ci.max_n, t);
      ci.total_words += tsu::packed_words(m) + tsu::packed_words(t);
    }
    if (p1 > p0) {
      CU(cudaMemcpyAsync(P<char>(ctx->b_pat) + p0, b->pattern + p0, (size_t)(p1 - p0), cudaMemcpyHostToDevice,
                         ctx->h2d_stream));
      h2d += p1 - p0;
    }
    if (t1 > t0) {
      CU(cudaMemcpyAsync(P<char>(ctx->b_txt) + t0, b->text + t0, (size_t)(t1 - t0), cudaMemcpyHostToDevice,
                         ctx->h2d_stream));
      h2d += t1 - t0;
    }
    CU(cudaEventRecord(ev_up[(size_t)c], ctx->h2d_stream));
  }
  ctx->timing.h2d_bytes = h2d;
  int64_t needed = 0, d2h = 0;
  double pack_ms = 0, align_ms = 0, compact_ms = 0;
  int64_t launches = 0, retried = 0, cells = 0, steps = 0, ext_bases = 0;
  std::vector<int64_t> run_base((size_t)K + 1, 0);
  for (int c = 0; c < K; ++c) {
    const int64_t c0 = cs[(size_t)c], nc = cbi[(size_t)c].n;
    DevBuf& ob = (c & 1) ? ctx->b_out2 : ctx->b_out;
    // the output buffer is reused two chunks later: its download must be done
    if (c >= 2) {
      if (ctx->blocking_sync) {
        CU(wait_stream(ctx, ctx->d2h_stream));  // sleeps until that download (and any later one) is done
      } else {
        CU(cudaEventSynchronize(ev_down[(size_t)c - 2]));
      }
    }
    CU(cudaStreamWaitEvent(st, ev_up[(size_t)c], 0));
    tsu::SeqView sv{nc, P<uint8_t>(ctx->b_pat), P<int64_t>(ctx->b_poff) + c0, P<int32_t>(ctx->b_plen) + c0,
                    P<uint8_t>(ctx->b_txt), P<int64_t>(ctx->b_toff) + c0, P<int32_t>(ctx->b_tlen) + c0};
    int64_t* d_coff = want_cigar ? P<int64_t>(ctx->b_coff) + c0 + c : nullptr;  // nc + 1 chunk-local offsets
    int64_t cneed = 0;
    uint32_t* d_runs = nullptr;
    ctx->timing.kernel_launches = 0;
    ctx->timing.retried_pairs = 0;
    rc = run_device(ctx, sv, want_cigar, P<int32_t>(ctx->b_score) + c0, P<int32_t>(ctx->b_status) + c0, nullptr, 0,
                    d_coff, &cneed, cbi[(size_t)c], b->pattern_len + c0, b->text_len + c0, &d_runs, &ob);
    if (rc) return rc;
    if (nc) {
      pack_ms += ev_ms(ctx->ev[2], ctx->ev[3]);
      align_ms += ev_ms(ctx->ev[4], ctx->ev[5]);
      if (want_cigar) compact_ms += ev_ms(ctx->ev[5], ctx->ev[6]);
    }
    launches += ctx->timing.kernel_launches;
    retried += ctx->timing.retried_pairs;
    cells += ctx->timing.cells;
    steps += ctx->timing.steps;
    ext_bases += ctx->timing.ext_bases;
    CU(cudaEventRecord(ev_done[(size_t)c], st));
    CU(cudaStreamWaitEvent(ctx->d2h_stream, ev_done[(size_t)c], 0));
    if (nc) {
      CU(cudaMemcpyAsync(res->score + c0, P<int32_t>(ctx->b_score) + c0, sizeof(int32_t) * nc,
                         cudaMemcpyDeviceToHost, ctx->d2h_stream));
      CU(cudaMemcpyAsync(hs + c0, P<int32_t>(ctx->b_status) + c0, sizeof(int32_t) * nc,
                         cudaMemcpyDeviceToHost, ctx->d2h_stream));
      d2h += nc * 8;
    }
    if (want_cigar) {
      // chunk-local offsets land at cigar_offset[c0 ..]; made global below
      CU(cudaMemcpyAsync(res->cigar_offset + c0, d_coff, sizeof(int64_t) * nc, cudaMemcpyDeviceToHost,
                         ctx->d2h_stream));
      d2h += nc * 8;
      run_base[(size_t)c + 1] = run_base[(size_t)c] + cneed;
      if (res->cigar && run_base[(size_t)c + 1] <= res->cigar_capacity && cneed) {
        CU(cudaMemcpyAsync(res->cigar + run_base[(size_t)c], d_runs, sizeof(uint32_t) * cneed,
                           cudaMemcpyDeviceToHost, ctx->d2h_stream));
        d2h += cneed * 4;
      }
      needed += cneed;
    }
    CU(cudaEventRecord(ev_down[(size_t)c], ctx->d2h_stream));
  }
  CU(cudaEventRecord(t_end, ctx->d2h_stream));
  CU(ctx->blocking_sync ? wait_stream(ctx, ctx->d2h_stream) : cudaEventSynchronize(t_end));
  ctx->timing.d2h_bytes = d2h;
  ctx->timing.pack_ms = pack_ms;
  ctx->timing.align_ms = align_ms;
  ctx->timing.compact_ms = compact_ms;
  ctx->timing.kernel_launches = launches;
  ctx->timing.retried_pairs = retried;
  ctx->timing.cells = cells;
  ctx->timing.steps = steps;
  ctx->timing.ext_bases = ext_bases;
  ctx->timing.device_bytes = (int64_t)ctx->peak_held;
  ctx->timing.total_ms = ev_ms(t_begin, t_end);
  ctx->timing.h2d_ms = 0;  // overlapped with the alignment
  ctx->timing.d2h_ms = 0;
  if (want_cigar) {
    for (int c = 0; c < K; ++c)
      for (int64_t i = cs[(size_t)c]; i < cs[(size_t)c + 1]; ++i) res->cigar_offset[i] += run_base[(size_t)c];
    res->cigar_offset[n] = needed;
    res->cigar_needed = needed;
  }
  if (res->pair_status) memcpy(res->pair_status, hs, sizeof(int32_t) * n);
  if ((rc = collect_status(ctx, hs, n))) return rc;
  if (want_cigar && (needed > res->cigar_capacity || !res->cigar)) return TSU_EOVERFLOW;
  return TSU_OK;
}

int tsu_align_fixed(tsu_ctx* ctx, const char* pattern, const char* text, int64_t num, int32_t plen, int32_t tlen,
                    int32_t* score, uint32_t flags) {
  if (!ctx) return TSU_EINVAL;
  if (num < 0 || plen < 0 || tlen < 0 || (num && (!pattern || !text || !score)))
    return set_err(ctx, TSU_EINVAL, "bad fixed-stride arguments");
  std::vector<int64_t> po((size_t)num), to((size_t)num);
  std::vector<int32_t> pl((size_t)num, plen), tl((size_t)num, tlen);
  for (int64_t i = 0; i < num; ++i) {
    po[(size_t)i] = i * (int64_t)plen;
    to[(size_t)i] = i * (int64_t)tlen;
  }
  tsu_batch b{num, pattern, po.data(), pl.data(), text, to.data(), tl.data()};
  tsu_result r{};
  r.score = score;
  return tsu_align_batch(ctx, &b, &r, flags | TSU_SCORE_ONLY);
}

int tsu_align_batch_device(tsu_ctx* ctx, const tsu_batch* b, tsu_result* res, uint32_t flags) {
  if (!ctx || !b || !res || !res->score) return ctx ? set_err(ctx, TSU_EINVAL, "null argument") : TSU_EINVAL;
  const bool want_cigar = !(flags & TSU_SCORE_ONLY);
  ctx->one_warp = (flags & TSU_ONE_WARP) != 0;
  ctx->bidir = (flags & TSU_BIDIRECTIONAL) != 0;
  if (want_cigar && !res->cigar_offset) return set_err(ctx, TSU_EINVAL, "cigar_offset required");
  CU(cudaSetDevice(ctx->device));
  ctx->timing = tsu_timing{};
  ctx->peak_held = ctx->held();
  const int64_t n = b->num_pairs;
  if (n < 0 || n > INT32_MAX) return set_err(ctx, TSU_EINVAL, "bad num_pairs");
  cudaStream_t st = ctx->stream;
  // batch info: lengths are on the device; bring them over once.
  BatchInfo bi;
  bi.n = n;
  std::vector<int32_t> pl((size_t)n), tl((size_t)n);
  {
    if (n) {
      CU(cudaMemcpyAsync(pl.data(), b->pattern_len, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
      CU(cudaMemcpyAsync(tl.data(), b->text_len, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
      CU(wait_stream(ctx, st));
    }
    for (int64_t i = 0; i < n; ++i) {
      if (pl[(size_t)i] < 0 || tl[(size_t)i] < 0 || pl[(size_t)i] > max_len(ctx) || tl[(size_t)i] > max_len(ctx))
        return set_err(ctx, TSU_EINVAL, "pair %lld: bad length", (long long)i);
      bi.max_m = std::max(bi.max_m, pl[(size_t)i]);
      bi.max_n = std::max(bi.max_n, tl[(size_t)i]);
      bi.total_words += tsu::packed_words(pl[(size_t)i]) + tsu::packed_words(tl[(size_t)i]);
    }
  }
  CU(cudaEventRecord(ctx->ev[0], st));
  CU(cudaEventRecord(ctx->ev[1], st));
  tsu::SeqView sv{n, (const uint8_t*)b->pattern, b->pattern_off, b->pattern_len, (const uint8_t*)b->text, b->text_off,
                  b->text_len};
  int32_t* d_status = res->pair_status;
  if (!d_status) {
    int rc = grow(ctx, ctx->b_status, sizeof(int32_t) * std::max<int64_t>(n, 1));
    if (rc) return rc;
    d_status = P<int32_t>(ctx->b_status);
  }
  int64_t needed = 0;
  int rc = run_device(ctx, sv, want_cigar, res->score, d_status, res->cigar, res->cigar_capacity, res->cigar_offset,
                      &needed, bi, pl.data(), tl.data());
  res->cigar_needed = needed;
  if (rc) return rc;
  CU(cudaEventRecord(ctx->ev[7], st));
  CU(wait_stream(ctx, st));
  ctx->timing.pack_ms = n ? ev_ms(ctx->ev[2], ctx->ev[3]) : 0;
  ctx->timing.align_ms = n ? ev_ms(ctx->ev[4], ctx->ev[5]) : 0;
  ctx->timing.compact_ms = (n && want_cigar) ? ev_ms(ctx->ev[5], ctx->ev[6]) : 0;
  ctx->timing.total_ms = ev_ms(ctx->ev[0], ctx->ev[7]);
  ctx->timing.device_bytes = (int64_t)ctx->peak_held;
  // statuses
  std::vector<int32_t> hs((size_t)n);
  if (n) {
    CU(cudaMemcpy(hs.data(), d_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
  }
  return collect_status(ctx, hs.data(), n);
}

int tsu_set_ends_free(tsu_ctx* ctx, int32_t pattern_begin_free, int32_t pattern_end_free, int32_t text_begin_free,
                      int32_t text_end_free) {
  if (!ctx) return TSU_EINVAL;
  if (pattern_begin_free < 0 || pattern_end_free < 0 || text_begin_free < 0 || text_end_free < 0)
    return set_err(ctx, TSU_EINVAL, "negative free end");
  ctx->ends_free[0] = pattern_begin_free;
  ctx->ends_free[1] = pattern_end_free;
  ctx->ends_free[2] = text_begin_free;
  ctx->ends_free[3] = text_end_free;
  return TSU_OK;
}

int tsu_set_low_memory(tsu_ctx* ctx, int32_t checkpoint_interval) {
  if (!ctx) return TSU_EINVAL;
  ctx->low_mem = checkpoint_interval;
  return TSU_OK;
}

int tsu_get_ends_free(const tsu_ctx* ctx, int32_t* out4) {
  if (!ctx || !out4) return TSU_EINVAL;
  for (int i = 0; i < 4; ++i) out4[i] = ctx->ends_free[i];
  return TSU_OK;
}

int tsu_set_band_start(tsu_ctx* ctx, int band, int mode, int warps_per_pair) {
  if (!ctx) return TSU_EINVAL;
  const int gw = warps_per_pair;
  if (band < 0 || band >= tsu::kBands || (mode != tsu::kModeShared && mode != tsu::kModeGlobal) ||
      (gw != 1 && gw != 2 && gw != 4 && gw != 8 && gw != 16 && gw != 32))
    return set_err(ctx, TSU_EINVAL, "band %d, mode %d, %d warps per pair: not a rung", band, mode, gw);
  ctx->band_start[band] = tsu::PassChoice{mode, gw};
  return TSU_OK;
}

int tsu_get_band_start(const tsu_ctx* ctx, int band, int* mode, int* warps_per_pair) {
  if (!ctx || band < 0 || band >= tsu::kBands || !mode || !warps_per_pair) return TSU_EINVAL;
  *mode = ctx->band_start[band].mode;
  *warps_per_pair = ctx->band_start[band].gw;
  return TSU_OK;
}

int tsu_predict_bytes(tsu_ctx* ctx, const tsu_batch* b, uint32_t flags, size_t* full, size_t* min) {
  if (!ctx || !full || !min) return TSU_EINVAL;
  BatchInfo bi;
  int64_t pb = 0, tb = 0;
  int rc = check_batch_host(ctx, b, &bi, &pb, &tb);
  if (rc) return rc;
  CU(cudaSetDevice(ctx->device));
  tsu::engine::BatchShape sh;
  sh.n = bi.n;
  sh.plen = b->pattern_len;
  sh.tlen = b->text_len;
  sh.pattern_bytes = pb;
  sh.text_bytes = tb;
  return tsu::engine::predict_bytes(ctx, sh, flags, 0.0, full, min);
}

int64_t tsu_cigar_to_ops(const uint32_t* runs, int64_t nruns, char* out, int64_t cap) {
  static const char code2c[16] = {'M', 'I', 'D', 'N', 'S', 'H', 'P', '=', 'X', '?', '?', '?', '?', '?', '?', '?'};
  int64_t w = 0;
  for (int64_t i = 0; i < nruns; ++i) {
    const int64_t len = runs[i] >> 4;
    const char c = code2c[runs[i] & 15];
    if (w + len > cap) return -1;
    memset(out + w, c, (size_t)len);
    w += len;
  }
  return w;
}

int64_t tsu_cigar_to_string(const uint32_t* runs, int64_t nruns, char* out, int64_t cap) {
  static const char code2c[16] = {'M', 'I', 'D', 'N', 'S', 'H', 'P', '=', 'X', '?', '?', '?', '?', '?', '?', '?'};
  int64_t w = 0;
  char tmp[24];
  for (int64_t i = 0; i < nruns; ++i) {
    int k = snprintf(tmp, sizeof tmp, "%u%c", runs[i] >> 4, code2c[runs[i] & 15]);
    if (w + k > cap) return -1;
    memcpy(out + w, tmp, (size_t)k);
    w += k;
  }
  return w;
}

}  // extern "C"
