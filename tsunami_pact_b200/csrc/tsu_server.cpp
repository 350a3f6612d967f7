// tsu_server.cpp -- C ABI of the request server (include/tsunami_b200.h):
// the scheduler of tsu_serve.h over engine contexts.
//
// Each worker is one tsu_ctx (its own streams and device buffers, growing to
// exactly the size asked, from the device's stream-ordered pool) driven by
// its own host thread through tsu_align_batch -- the batch path, so a served
// request gets the kernels, the length bands and the retry ladder of a batch
// call.  A further context (no buffers) predicts the device memory of
// requests and jobs.  Jobs go through page-locked staging buffers of the
// worker: copies from or to pageable memory block the worker's thread inside
// the driver while its stream is busy, and with many workers that
// serializes jobs that would otherwise overlap on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tsunami_b200.h"
#include "tsu_engine_internal.h"
#include "tsu_serve.h"

namespace {

using tsu::serve::Output;
using tsu::serve::Pairs;

// A growing page-locked host buffer.  Outgrown buffers are kept until the
// worker ends: cudaFreeHost can synchronize the whole device, which would
// stall every other worker's jobs.
class HostStage {
 public:
  ~HostStage() {
    for (char* p : retired_) cudaFreeHost(p);
    if (p_) cudaFreeHost(p_);
  }
  // At least `bytes`, doubling; nullptr if the allocation fails.
  char* get(size_t bytes) {
    if (bytes > cap_) {
      const size_t nb = std::max<size_t>(std::max(bytes, 2 * cap_), 4 << 20);
      char* np = nullptr;
      if (cudaHostAlloc(reinterpret_cast<void**>(&np), nb, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
      if (p_) retired_.push_back(p_);
      p_ = np;
      cap_ = nb;
    }
    return p_;
  }

 private:
  char* p_ = nullptr;
  size_t cap_ = 0;
  std::vector<char*> retired_;
};

size_t up16(size_t b) { return (b + 15) & ~(size_t)15; }

class EngineExecutor final : public tsu::serve::Executor {
 public:
  explicit EngineExecutor(tsu_ctx* ctx) : ctx_(ctx), default_hint_(tsu::engine::hint(ctx)) {
    tsu::engine::set_exact_growth(ctx_, true);
    tsu::engine::set_blocking_sync(ctx_, true);
    in_.get(16 << 20);  // page-locked staging allocated now, not under load
    out_.get(16 << 20);
  }
  ~EngineExecutor() override { tsu_destroy(ctx_); }

  int predict(int64_t n, const int32_t* plen, const int32_t* tlen, int64_t pb, int64_t tb, uint32_t flags,
              double hint, size_t* full, size_t* min) override {
    tsu::engine::BatchShape sh;
    sh.n = n;
    sh.plen = plen;
    sh.tlen = tlen;
    sh.pattern_bytes = pb;
    sh.text_bytes = tb;
    tsu::engine::set_fit_start(ctx_, (flags & tsu::serve::kFitStart) != 0);
    tsu_set_low_memory(ctx_, (flags & tsu::serve::kLowMem) ? -1 : 0);
    return tsu::engine::predict_bytes(ctx_, sh, flags & (TSU_SCORE_ONLY | TSU_BIDIRECTIONAL), hint, full, min);
  }
  size_t held() override { return tsu::engine::held_bytes(ctx_); }
  void set_budget(size_t bytes) override { tsu::engine::set_budget(ctx_, bytes); }
  int trim() override { return tsu::engine::trim(ctx_); }
  size_t needed() override { return tsu::engine::needed_bytes(ctx_); }
  std::string error() override { return tsu_last_error(ctx_); }

  int run(const Pairs& in, uint32_t flags, double hint, Output* out) override {
    tsu::engine::set_hint(ctx_, hint > 0 ? hint : default_hint_);
    tsu::engine::set_fit_start(ctx_, (flags & tsu::serve::kFitStart) != 0);
    tsu_set_low_memory(ctx_, (flags & tsu::serve::kLowMem) ? -1 : 0);
    const size_t n = (size_t)in.n();
    const bool cig = !(flags & TSU_SCORE_ONLY);
    int64_t cap = 1;  // a pair has at most m + n runs
    for (size_t i = 0; i < n; ++i) cap += (int64_t)in.plen[i] + in.tlen[i];
    // inputs: pattern bytes | text bytes | offsets | lengths
    const size_t a_pat = 0, a_txt = up16(in.pat.size() + 1), a_poff = a_txt + up16(in.txt.size() + 1);
    const size_t a_toff = a_poff + up16(8 * n), a_plen = a_toff + up16(8 * n), a_tlen = a_plen + up16(4 * n);
    char* hi = in_.get(a_tlen + up16(4 * n));
    // outputs: scores | statuses | CIGAR offsets | runs
    const size_t o_st = up16(4 * n), o_coff = o_st + up16(4 * n), o_runs = o_coff + up16(8 * (n + 1));
    char* ho = out_.get(o_runs + (cig ? 4 * (size_t)cap : 0));
    if (!hi || !ho) return TSU_ENOMEM;
    if (!in.pat.empty()) memcpy(hi + a_pat, in.pat.data(), in.pat.size());
    if (!in.txt.empty()) memcpy(hi + a_txt, in.txt.data(), in.txt.size());
    memcpy(hi + a_poff, in.poff.data(), 8 * n);
    memcpy(hi + a_toff, in.toff.data(), 8 * n);
    memcpy(hi + a_plen, in.plen.data(), 4 * n);
    memcpy(hi + a_tlen, in.tlen.data(), 4 * n);
    tsu_batch b{(int64_t)n,
                hi + a_pat,
                reinterpret_cast<const int64_t*>(hi + a_poff),
                reinterpret_cast<const int32_t*>(hi + a_plen),
                hi + a_txt,
                reinterpret_cast<const int64_t*>(hi + a_toff),
                reinterpret_cast<const int32_t*>(hi + a_tlen)};
    int32_t* h_score = reinterpret_cast<int32_t*>(ho);
    int32_t* h_status = reinterpret_cast<int32_t*>(ho + o_st);
    for (size_t i = 0; i < n; ++i) h_status[i] = -1;
    tsu_result r{};
    r.score = h_score;
    r.pair_status = h_status;
    if (cig) {
      r.cigar = reinterpret_cast<uint32_t*>(ho + o_runs);
      r.cigar_capacity = cap;
      r.cigar_offset = reinterpret_cast<int64_t*>(ho + o_coff);
    }
    const int rc = tsu_align_batch(ctx_, &b, &r, flags & (TSU_SCORE_ONLY | TSU_BIDIRECTIONAL));
    out->score.assign(h_score, h_score + n);
    out->pair_status.assign(h_status, h_status + n);
    if (rc == TSU_OK && cig) {
      out->coff.assign(r.cigar_offset, r.cigar_offset + n + 1);
      out->cigar.assign(r.cigar, r.cigar + r.cigar_needed);
    }
    return rc;
  }

 private:
  tsu_ctx* ctx_;
  double default_hint_;
  HostStage in_, out_;
};

int make_ctx(const tsu::engine::Spec& pen, int device, double hint, size_t budget, tsu_ctx** out) {
  tsu_config c{};
  c.device = device;
  c.mem_budget = budget;
  c.max_error_hint = hint;
  return tsu::engine::create(pen, &c, true, out);
}

}  // namespace

struct tsu_server {
  std::unique_ptr<tsu::serve::Server> s;
  std::string err;
};

namespace {

int server_create(const tsu::engine::Spec& pen, const tsu_server_config* cfg, tsu_server** out) {
  *out = nullptr;
  tsu_server_config c{};
  if (cfg) c = *cfg;
  if (c.workers < 0 || c.workers > 256 || c.max_queue < 0 || c.max_job_pairs < 0 || c.max_job_requests < 0 ||
      c.watchdog_ms < 0 || c.max_error_hint < 0)
    return TSU_EINVAL;
  tsu::serve::Config sc;
  sc.workers = c.workers ? c.workers : 32;
  sc.max_queue = c.max_queue ? c.max_queue : (1 << 16);
  sc.max_job_pairs = c.max_job_pairs ? c.max_job_pairs : 16384;
  sc.max_job_requests = c.max_job_requests ? c.max_job_requests : 64;
  sc.watchdog_ms = c.watchdog_ms;
  sc.resident_cap = c.resident_bytes;
  sc.heavy_len = c.heavy_len == 0 ? 8192 : (c.heavy_len < 0 ? 0 : c.heavy_len);
  sc.heavy_workers = c.heavy_workers > 0 ? c.heavy_workers : std::max(1, sc.workers - 2);
  sc.estimate = c.estimate_hint >= 0;
  // Jobs of different workers overlap only on different hardware queues: ask
  // for the most (32) unless the process chose otherwise.  It takes effect
  // if this is the process's first CUDA work on the device.
  setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
  // the planner context: no buffers; its create resolves the default budget
  tsu_ctx* planner = nullptr;
  int rc = make_ctx(pen, c.device, c.max_error_hint, c.mem_budget, &planner);
  if (rc) return rc;
  std::unique_ptr<tsu::serve::Executor> plan(new EngineExecutor(planner));
  sc.budget = tsu::engine::budget_bytes(planner);  // mem_budget, or 80% of the free memory when 0
  std::vector<std::unique_ptr<tsu::serve::Executor>> ws;
  for (int i = 0; i < sc.workers; ++i) {
    tsu_ctx* ctx = nullptr;
    rc = make_ctx(pen, c.device, c.max_error_hint, sc.budget, &ctx);
    if (rc) return rc;  // unique_ptrs destroy the contexts made so far
    ws.emplace_back(new EngineExecutor(ctx));
  }
  // the device pool holds the whole budget from the start
  tsu::engine::prime_pool(planner, sc.budget);
  auto* srv = new tsu_server();
  srv->s = std::make_unique<tsu::serve::Server>(sc, std::move(ws), std::move(plan));
  *out = srv;
  return TSU_OK;
}

}  // namespace

extern "C" {

int tsu_server_create_metric(int metric, const int32_t* penalties, int num_penalties, const tsu_server_config* cfg,
                             tsu_server** out) {
  if (!out) return TSU_EINVAL;
  *out = nullptr;
  tsu::engine::Spec spec;
  const int rc = tsu::engine::make_spec(metric, penalties, num_penalties, &spec);
  return rc ? rc : server_create(spec, cfg, out);
}

int tsu_server_create(const tsu_penalties* pen, const tsu_server_config* cfg, tsu_server** out) {
  if (!pen) return TSU_EINVAL;
  const int32_t p[3] = {pen->mismatch, pen->gap_opening, pen->gap_extension};
  return tsu_server_create_metric(TSU_METRIC_GAP_AFFINE, p, 3, cfg, out);
}

int tsu_server_create_dual(const tsu_penalties2* pen, const tsu_server_config* cfg, tsu_server** out) {
  if (!pen) return TSU_EINVAL;
  const int32_t p[5] = {pen->mismatch, pen->gap_opening, pen->gap_extension, pen->gap_opening2, pen->gap_extension2};
  return tsu_server_create_metric(TSU_METRIC_GAP_AFFINE_2P, p, 5, cfg, out);
}

int tsu_server_destroy(tsu_server* srv) {
  if (!srv) return TSU_EINVAL;
  srv->s->shutdown();
  srv->s.reset();
  delete srv;
  return TSU_OK;
}

int tsu_submit(tsu_server* srv, const tsu_batch* request, uint32_t flags, uint64_t* id) {
  if (!srv) return TSU_EINVAL;
  return srv->s->submit(request, flags, id);
}

int tsu_poll(tsu_server* srv, uint64_t id, tsu_result* res, tsu_request_info* info) {
  if (!srv) return TSU_EINVAL;
  return srv->s->poll(id, res, info);
}

int tsu_wait(tsu_server* srv, uint64_t id, double timeout_ms, tsu_result* res, tsu_request_info* info) {
  if (!srv) return TSU_EINVAL;
  return srv->s->wait(id, timeout_ms, res, info);
}

int tsu_cancel(tsu_server* srv, uint64_t id) {
  if (!srv) return TSU_EINVAL;
  return srv->s->cancel(id);
}

int tsu_server_get_stats(tsu_server* srv, tsu_server_stats* out) {
  if (!srv || !out) return TSU_EINVAL;
  srv->s->stats(out);
  return TSU_OK;
}

int tsu_server_reset_stats(tsu_server* srv) {
  if (!srv) return TSU_EINVAL;
  srv->s->reset_stats();
  return TSU_OK;
}

const char* tsu_server_last_error(tsu_server* srv) {
  if (!srv) return "null server";
  static thread_local std::string msg;
  msg = srv->s->error();
  return msg.c_str();
}

}  // extern "C"
