// tsu_serve.h -- request scheduler of the alignment server (host only, no
// CUDA).  The server's C ABI (tsu_server.cpp) runs it over engine contexts;
// the tests run it over a fake executor on the CPU.
//
// No counterpart in the reference, which aligns one file per process
// (wfa_gpu.cu:43-188).  Design:
//   * submit copies a request's pairs into the server and splits them into
//     parts: one part with its light pairs (max(m, n) < heavy_len) and one
//     part per heavy pair.  Each part carries its predicted device memory
//     (Executor::predict: inputs, packed words, outputs, CIGAR arena and
//     wavefront scratch at its edit-rate hint, bounded by the
//     penalty-derived score bound of each pair);
//   * light parts wait in one FIFO queue, heavy parts in another;
//   * a pool of workers, each an Executor with its own CUDA streams and
//     device buffers, runs jobs.  A light job is the oldest light part plus
//     the light parts queued behind it (same flags, up to max_job_pairs
//     pairs and max_job_requests parts), aligned in one engine call -- so
//     requests that arrive while others run are batched into the next job;
//     a heavy job is one heavy pair, so its memory is sized by that pair and
//     returned when that pair is done.  At most heavy_workers heavy jobs run
//     at once, so light jobs always find a worker.  Jobs of different
//     workers overlap on the device;
//   * admission: a job starts when a worker is idle and its predicted bytes
//     fit in the budget beside what the other workers were granted or still
//     hold.  Idle workers keep their buffers (resident state) up to
//     resident_cap and until the memory is needed elsewhere.  A job of
//     several parts that does not fit is halved down to one part; a part
//     that fits only with fewer pairs in flight runs when nothing else does;
//     a CIGAR part that cannot fit even then runs in low-memory mode
//     (checkpointed history) if that fits, else fails with TSU_ENOMEM.  Each queue
//     starts its parts in order (no overtaking within a queue);
//   * a request is done when all its parts are: its results are assembled
//     in its own pair order and made visible to poll/wait; latency is
//     measured from submit to that moment;
//   * a job of several parts that fails is re-queued at the head as
//     single-part jobs, so a failure stays with the request that caused it;
//     a single part that ran out of memory is re-queued with the reservation
//     the engine asked for (up to 3 attempts); a failed part fails its
//     request and drops the request's other parts;
//   * watchdog: a job running longer than watchdog_ms fails its requests
//     with TSU_ETIMEOUT; the worker's late results are discarded and it
//     takes no new job until it returns.
// Alignment of a pair does not depend on the other pairs of its job, so a
// request's results are the same alone and in any mix.
#pragma once

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tsunami_b200.h"
#include "tsu_estimate.h"

namespace tsu {
namespace serve {

// Executor flag beside TSU_SCORE_ONLY: the hint is a per-pair estimate, so
// choose the first rung by the width it predicts (tsu::fit_start).
constexpr uint32_t kFitStart = 0x100;
// Executor flag: align with checkpointed history (low-memory mode).  Set by
// admission on a CIGAR part whose smallest footprint exceeds the budget, when
// the low-memory footprint fits: such a request runs instead of failing.
constexpr uint32_t kLowMem = 0x200;

using Clock = std::chrono::steady_clock;

inline double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Pairs owned by the server: sequences packed back to back.
struct Pairs {
  std::vector<char> pat, txt;
  std::vector<int64_t> poff, toff;
  std::vector<int32_t> plen, tlen;

  int64_t n() const { return (int64_t)plen.size(); }

  // Compact copy of a caller's batch (validated by the caller).
  void assign(const tsu_batch& b) {
    const int64_t n = b.num_pairs;
    int64_t pb = 0, tb = 0;
    for (int64_t i = 0; i < n; ++i) {
      pb += b.pattern_len[i];
      tb += b.text_len[i];
    }
    pat.resize((size_t)pb);
    txt.resize((size_t)tb);
    poff.resize((size_t)n);
    toff.resize((size_t)n);
    plen.assign(b.pattern_len, b.pattern_len + n);
    tlen.assign(b.text_len, b.text_len + n);
    int64_t p = 0, t = 0;
    for (int64_t i = 0; i < n; ++i) {
      poff[(size_t)i] = p;
      toff[(size_t)i] = t;
      if (plen[(size_t)i]) memcpy(pat.data() + p, b.pattern + b.pattern_off[i], (size_t)plen[(size_t)i]);
      if (tlen[(size_t)i]) memcpy(txt.data() + t, b.text + b.text_off[i], (size_t)tlen[(size_t)i]);
      p += plen[(size_t)i];
      t += tlen[(size_t)i];
    }
  }

  // Append pairs idx of o.
  void append(const Pairs& o, const std::vector<int32_t>& idx) {
    for (int32_t i : idx) {
      poff.push_back((int64_t)pat.size());
      toff.push_back((int64_t)txt.size());
      const int32_t m = o.plen[(size_t)i], n = o.tlen[(size_t)i];
      pat.insert(pat.end(), o.pat.begin() + o.poff[(size_t)i], o.pat.begin() + o.poff[(size_t)i] + m);
      txt.insert(txt.end(), o.txt.begin() + o.toff[(size_t)i], o.txt.begin() + o.toff[(size_t)i] + n);
      plen.push_back(m);
      tlen.push_back(n);
    }
  }

  tsu_batch view() const {
    static const char kEmpty[1] = {0};
    return tsu_batch{n(), pat.empty() ? kEmpty : pat.data(), poff.data(), plen.data(),
                     txt.empty() ? kEmpty : txt.data(), toff.data(), tlen.data()};
  }
};

// Results of a job or of one request.  pair_status starts at -1 ("not
// computed"); coff/cigar only without TSU_SCORE_ONLY.
struct Output {
  int status = TSU_OK;
  std::vector<int32_t> score, pair_status;
  std::vector<int64_t> coff;  // n + 1
  std::vector<uint32_t> cigar;
};

// One worker's device side (or a fake of it).  Calls on one executor come
// from one thread at a time.  hint: the edit rate sizing wavefront scratch
// (0: the executor's default).
class Executor {
 public:
  virtual ~Executor() = default;
  // Predicted device bytes to align `plen`/`tlen` (n pairs, pb/tb sequence
  // bytes) in one call: every pair of a band in flight (*full) or one (*min).
  virtual int predict(int64_t n, const int32_t* plen, const int32_t* tlen, int64_t pb, int64_t tb, uint32_t flags,
                      double hint, size_t* full, size_t* min) = 0;
  virtual size_t held() = 0;                  // device bytes held now
  virtual void set_budget(size_t bytes) = 0;  // for the next run
  virtual int trim() = 0;                     // release every buffer
  // Align every pair; fills out->score and out->pair_status (and CIGARs).
  virtual int run(const Pairs& in, uint32_t flags, double hint, Output* out) = 0;
  virtual size_t needed() = 0;  // after TSU_ENOMEM: the bytes the run needed (0: unknown)
  virtual std::string error() = 0;
};

struct Config {
  int workers = 4;
  size_t budget = 0;              // device bytes for all workers
  int64_t max_queue = 1 << 16;    // queued requests before submit says TSU_EBUSY
  int64_t max_job_pairs = 16384;  // pairs merged into one light job
  int max_job_requests = 64;      // parts merged into one light job
  double watchdog_ms = 0;         // 0: off
  size_t resident_cap = 0;        // bytes an idle worker may keep (0: budget / (2 * workers))
  int32_t heavy_len = 8192;       // max(m, n) from which a pair is a part of its own (0: never)
  int heavy_workers = 0;          // heavy jobs at once (0: workers - 1, at least 1)
  double hint = 0;                // edit-rate hint of light parts (0: the executor's default)
  bool estimate = true;           // heavy pairs: hint from their shared k-mers (tsu_estimate.h)
};

struct Request;
using ReqPtr = std::shared_ptr<Request>;

// A request's pairs idx, run as (part of) a job.
struct Part {
  ReqPtr req;
  std::vector<int32_t> idx;
  bool heavy = false;
  bool alone = false;  // run as a job of its own (after a job-level failure)
  int attempts = 0;
  double hint = 0;
  uint32_t flags = 0;        // executor flags: the request's, plus kFitStart
  size_t full = 0, min = 0;  // predicted bytes alone
  int64_t pairs() const { return (int64_t)idx.size(); }
};
using PartPtr = std::shared_ptr<Part>;

struct Request {
  uint64_t id = 0;
  Pairs in;
  uint32_t flags = 0;
  enum State { kQueued, kRunning, kDone } state = kQueued;
  bool cancelled = false;
  int parts_left = 0;
  int attempts = 0;      // most attempts of any part
  int job_requests = 0;  // most parts in a job that delivered one of its parts
  int64_t job_seq = 0;   // job that started its first part
  Clock::time_point t_submit, t_start, t_done;
  bool started = false;
  std::vector<std::pair<PartPtr, Output>> done_parts;
  Output out;
};

class Server {
 public:
  Server(const Config& cfg, std::vector<std::unique_ptr<Executor>> workers, std::unique_ptr<Executor> planner)
      : cfg_(cfg), planner_(std::move(planner)) {
    const size_t nw = std::max<size_t>(1, workers.size());
    if (cfg_.resident_cap == 0) cfg_.resident_cap = cfg_.budget / (2 * nw);
    if (cfg_.heavy_workers <= 0 || cfg_.heavy_workers > (int)nw - 1) cfg_.heavy_workers = std::max(1, (int)nw - 1);
    t_reset_ = Clock::now();
    for (size_t i = 0; i < workers.size(); ++i) {
      auto w = std::make_unique<Worker>();
      w->idx = (int)i;
      w->ex = std::move(workers[i]);
      w->grant = w->ex->held();
      workers_.push_back(std::move(w));
    }
    for (auto& w : workers_) w->th = std::thread([this, p = w.get()] { worker_loop(p); });
    sched_ = std::thread([this] { sched_loop(); });
  }

  ~Server() { shutdown(); }

  // Drop queued requests, let running jobs finish, stop the threads.
  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (stopped_) return;
      stopping_ = true;
      std::vector<PartPtr> queued(light_.begin(), light_.end());
      queued.insert(queued.end(), heavy_.begin(), heavy_.end());
      for (auto& p : queued) fail_request(*p->req, TSU_EBUSY, Clock::now());  // empties the queues
    }
    cv_sched_.notify_all();
    cv_work_.notify_all();
    if (sched_.joinable()) sched_.join();
    for (auto& w : workers_)
      if (w->th.joinable()) w->th.join();
    std::lock_guard<std::mutex> lk(mu_);
    stopped_ = true;
    cv_done_.notify_all();
  }

  int submit(const tsu_batch* b, uint32_t flags, uint64_t* id) {
    if (!b || !id) return TSU_EINVAL;
    if (b->num_pairs < 0 || b->num_pairs > INT32_MAX) return TSU_EINVAL;
    if (b->num_pairs && (!b->pattern || !b->pattern_off || !b->pattern_len || !b->text || !b->text_off || !b->text_len))
      return TSU_EINVAL;
    for (int64_t i = 0; i < b->num_pairs; ++i) {
      const int32_t m = b->pattern_len[i], n = b->text_len[i];
      if (m < 0 || n < 0 || m > (1 << 26) || n > (1 << 26) || b->pattern_off[i] < 0 || b->text_off[i] < 0)
        return TSU_EINVAL;
    }
    auto r = std::make_shared<Request>();
    r->t_submit = Clock::now();
    r->flags = flags & (TSU_SCORE_ONLY | TSU_BIDIRECTIONAL);
    r->in.assign(*b);
    // parts: each heavy pair alone (longest first), then the light pairs
    std::vector<PartPtr> parts;
    auto light = std::make_shared<Part>();
    for (int32_t i = 0; i < (int32_t)r->in.n(); ++i) {
      const int32_t L = std::max(r->in.plen[(size_t)i], r->in.tlen[(size_t)i]);
      if (cfg_.heavy_len > 0 && L >= cfg_.heavy_len) {
        auto h = std::make_shared<Part>();
        h->heavy = true;
        h->idx.push_back(i);
        parts.push_back(h);
      } else {
        light->idx.push_back(i);
      }
    }
    std::stable_sort(parts.begin(), parts.end(), [&](const PartPtr& a, const PartPtr& c) {
      const int32_t i = a->idx[0], j = c->idx[0];
      return (int64_t)r->in.plen[(size_t)i] + r->in.tlen[(size_t)i] >
             (int64_t)r->in.plen[(size_t)j] + r->in.tlen[(size_t)j];
    });
    if (!light->idx.empty()) parts.push_back(light);
    for (auto& p : parts) {
      p->req = r;
      p->hint = cfg_.hint;
      p->flags = r->flags;
      if (p->heavy && cfg_.estimate) {
        const int32_t i = p->idx[0];
        const double e = estimate_edit_rate(r->in.pat.data() + r->in.poff[(size_t)i], r->in.plen[(size_t)i],
                                            r->in.txt.data() + r->in.toff[(size_t)i], r->in.tlen[(size_t)i]);
        if (e >= 0) {
          p->hint = std::min(1.0, std::max(0.02, 1.3 * e + 0.01));
          p->flags |= kFitStart;
        }
      }
      const int rc = predict_parts({p}, p->flags, p->hint, &p->full, &p->min);
      if (rc) return rc;
      // too big for the budget: CIGARs with checkpointed history instead
      // (the bidirectional mode keeps no history to checkpoint)
      if (p->min > cfg_.budget && !(p->flags & (TSU_SCORE_ONLY | TSU_BIDIRECTIONAL))) {
        size_t full2 = 0, min2 = 0;
        if (predict_parts({p}, p->flags | kLowMem, p->hint, &full2, &min2) == TSU_OK && min2 <= cfg_.budget) {
          p->flags |= kLowMem;
          p->full = full2;
          p->min = min2;
        }
      }
    }
    std::lock_guard<std::mutex> lk(mu_);
    if (stopping_) return TSU_EBUSY;
    for (auto& p : parts)
      if (p->min > cfg_.budget) {
        ++st_rejected_;
        err_ = "request needs " + std::to_string(p->min) + " B of device memory for " + std::to_string(p->pairs()) +
               " pair(s), budget " + std::to_string(cfg_.budget);
        return TSU_ENOMEM;
      }
    if (waiting_ >= cfg_.max_queue) {
      ++st_rejected_;
      err_ = "queue full";
      return TSU_EBUSY;
    }
    r->id = ++next_id_;
    *id = r->id;
    ++st_submitted_;
    reqs_[r->id] = r;
    if (parts.empty()) {  // nothing to align
      r->state = Request::kDone;
      r->t_start = r->t_done = r->t_submit;
      record_done(*r);
      cv_done_.notify_all();
      return TSU_OK;
    }
    r->parts_left = (int)parts.size();
    ++open_;
    ++waiting_;
    for (auto& p : parts) (p->heavy ? heavy_ : light_).push_back(p);
    cv_sched_.notify_one();
    return TSU_OK;
  }

  // Copy a finished request's results out and forget it.  TSU_EPENDING
  // while it is queued or running; TSU_EOVERFLOW (request kept, cigar_needed
  // set) when res->cigar_capacity is too small.  Otherwise the request's
  // status.
  int poll(uint64_t id, tsu_result* res, tsu_request_info* info) {
    std::lock_guard<std::mutex> lk(mu_);
    return take(id, res, info);
  }

  int wait(uint64_t id, double timeout_ms, tsu_result* res, tsu_request_info* info) {
    std::unique_lock<std::mutex> lk(mu_);
    const auto deadline = Clock::now() + std::chrono::microseconds((int64_t)(std::max(0.0, timeout_ms) * 1000.0));
    auto ready = [&] {
      auto it = reqs_.find(id);
      return it == reqs_.end() || it->second->state == Request::kDone;
    };
    if (timeout_ms < 0) {
      cv_done_.wait(lk, ready);
    } else if (!cv_done_.wait_until(lk, deadline, ready)) {
      return TSU_ETIMEOUT;
    }
    return take(id, res, info);
  }

  // Queued: never runs.  Running: its results are dropped.  Done: forgotten.
  int cancel(uint64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return TSU_ENOTFOUND;
    ReqPtr r = it->second;
    reqs_.erase(it);
    r->cancelled = true;
    fail_request(*r, TSU_EBUSY, Clock::now());
    ++st_cancelled_;
    cv_sched_.notify_one();
    return TSU_OK;
  }

  void stats(tsu_server_stats* s) {
    std::lock_guard<std::mutex> lk(mu_);
    *s = tsu_server_stats{};
    s->submitted = st_submitted_;
    s->completed = st_completed_;
    s->failed = st_failed_;
    s->rejected = st_rejected_;
    s->cancelled = st_cancelled_;
    s->timed_out = st_timed_out_;
    int64_t running = 0;
    for (auto& kv : reqs_) running += kv.second->state == Request::kRunning;
    s->running = running;
    s->queued = waiting_;
    s->jobs = st_jobs_;
    s->pairs_completed = st_pairs_;
    s->mean_requests_per_job = st_jobs_ ? (double)st_job_parts_ / (double)st_jobs_ : 0.0;
    std::vector<double> v = lat_;
    if (!v.empty()) {
      auto pct = [&](double q) {
        const size_t k = std::min(v.size() - 1, (size_t)(q * (double)v.size()));
        std::nth_element(v.begin(), v.begin() + (long)k, v.end());
        return v[k];
      };
      s->p50_ms = pct(0.50);
      s->p99_ms = pct(0.99);
      s->p999_ms = pct(0.999);
      double sum = 0, mx = 0;
      for (double x : v) {
        sum += x;
        mx = std::max(mx, x);
      }
      s->mean_ms = sum / (double)v.size();
      s->max_ms = mx;
    }
    s->elapsed_s = ms_between(t_reset_, Clock::now()) / 1000.0;
    s->budget_bytes = cfg_.budget;
    s->granted_bytes = granted();
    s->peak_granted_bytes = peak_granted_;
    s->workers = (int32_t)workers_.size();
    s->heavy_jobs = st_heavy_jobs_;
    s->busy_s = st_busy_ms_ / 1000.0;
    s->heavy_busy_s = st_heavy_busy_ms_ / 1000.0;
  }

  void reset_stats() {
    std::lock_guard<std::mutex> lk(mu_);
    st_submitted_ = st_completed_ = st_failed_ = st_rejected_ = st_cancelled_ = st_timed_out_ = 0;
    st_jobs_ = st_job_parts_ = st_pairs_ = st_heavy_jobs_ = 0;
    st_busy_ms_ = st_heavy_busy_ms_ = 0;
    lat_.clear();
    peak_granted_ = granted();
    t_reset_ = Clock::now();
  }

  std::string error() {
    std::lock_guard<std::mutex> lk(mu_);
    return err_;
  }

 private:
  struct Worker {
    int idx = 0;
    std::unique_ptr<Executor> ex;
    std::thread th;
    bool busy = false;   // a job is assigned
    bool heavy = false;  // the job is a heavy one
    bool stuck = false;  // the watchdog failed its requests
    size_t grant = 0;    // bytes granted to the running job, or held while idle
    double hint = 0;
    std::vector<PartPtr> job;
    Clock::time_point started;
  };

  size_t granted() const {
    size_t g = 0;
    for (auto& w : workers_) g += w->grant;
    return g;
  }

  int predict_parts(const std::vector<PartPtr>& parts, uint32_t flags, double hint, size_t* full, size_t* min) {
    std::vector<int32_t> pl, tl;
    int64_t pb = 0, tb = 0;
    for (auto& p : parts)
      for (int32_t i : p->idx) {
        const Pairs& in = p->req->in;
        pl.push_back(in.plen[(size_t)i]);
        tl.push_back(in.tlen[(size_t)i]);
        pb += in.plen[(size_t)i];
        tb += in.tlen[(size_t)i];
      }
    std::lock_guard<std::mutex> lk(plan_mu_);
    return planner_->predict((int64_t)pl.size(), pl.data(), tl.data(), pb, tb, flags, hint, full, min);
  }

  void record_done(Request& r) {
    if (r.out.status == TSU_OK) {
      ++st_completed_;
      st_pairs_ += r.in.n();
      lat_.push_back(ms_between(r.t_submit, r.t_done));
    } else if (r.out.status == TSU_ETIMEOUT) {
      ++st_timed_out_;
    } else {
      ++st_failed_;
    }
  }

  void drop_queued_parts(const Request& r) {
    for (auto* q : {&light_, &heavy_})
      q->erase(std::remove_if(q->begin(), q->end(), [&](const PartPtr& p) { return p->req.get() == &r; }), q->end());
  }

  // A request fails (mu_ held): its queued parts are dropped, running ones
  // are ignored when they return.
  void fail_request(Request& r, int status, Clock::time_point now) {
    if (r.state == Request::kDone) return;
    drop_queued_parts(r);
    --open_;
    if (!r.started) --waiting_;
    r.state = Request::kDone;
    r.out = Output{};
    r.out.status = status;
    r.done_parts.clear();
    r.t_done = now;
    if (!r.started) r.t_start = now;
    if (!r.cancelled) record_done(r);
  }

  // All parts done (mu_ held): scatter the parts' results into the
  // request's pair order.
  void assemble(Request& r) {
    const int64_t n = r.in.n();
    const bool cig = !(r.flags & TSU_SCORE_ONLY);
    r.out = Output{};
    r.out.score.assign((size_t)n, 0);
    r.out.pair_status.assign((size_t)n, -1);
    std::vector<const uint32_t*> run_ptr(cig ? (size_t)n : 0, nullptr);
    std::vector<int64_t> run_len(cig ? (size_t)n : 0, 0);
    for (auto& po : r.done_parts) {
      const Part& p = *po.first;
      const Output& o = po.second;
      for (size_t k = 0; k < p.idx.size(); ++k) {
        const size_t i = (size_t)p.idx[k];
        r.out.score[i] = o.score[k];
        r.out.pair_status[i] = o.pair_status[k];
        if (cig) {
          run_ptr[i] = o.cigar.data() + o.coff[k];
          run_len[i] = o.coff[k + 1] - o.coff[k];
        }
      }
    }
    if (cig) {
      r.out.coff.assign((size_t)n + 1, 0);
      for (int64_t i = 0; i < n; ++i) r.out.coff[(size_t)i + 1] = r.out.coff[(size_t)i] + run_len[(size_t)i];
      r.out.cigar.resize((size_t)r.out.coff[(size_t)n]);
      for (int64_t i = 0; i < n; ++i)
        if (run_len[(size_t)i])
          memcpy(r.out.cigar.data() + r.out.coff[(size_t)i], run_ptr[(size_t)i], sizeof(uint32_t) * (size_t)run_len[(size_t)i]);
    }
    r.done_parts.clear();
  }

  int take(uint64_t id, tsu_result* res, tsu_request_info* info) {
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return TSU_ENOTFOUND;
    Request& r = *it->second;
    if (r.state != Request::kDone) return TSU_EPENDING;
    const int64_t n = r.in.n();
    if (info) {
      info->num_pairs = n;
      info->queue_ms = ms_between(r.t_submit, r.t_start);
      info->latency_ms = ms_between(r.t_submit, r.t_done);
      info->job_requests = r.job_requests;
      info->attempts = r.attempts;
      info->job_seq = r.job_seq;
    }
    if (r.out.status == TSU_OK && n) {
      if (!res || !res->score) return TSU_EINVAL;
      const bool cig = !(r.flags & TSU_SCORE_ONLY);
      if (cig) {
        if (!res->cigar_offset) return TSU_EINVAL;
        const int64_t need = (int64_t)r.out.cigar.size();
        res->cigar_needed = need;
        if (need > res->cigar_capacity || (need && !res->cigar)) return TSU_EOVERFLOW;
        memcpy(res->cigar_offset, r.out.coff.data(), sizeof(int64_t) * (size_t)(n + 1));
        if (need) memcpy(res->cigar, r.out.cigar.data(), sizeof(uint32_t) * (size_t)need);
      }
      memcpy(res->score, r.out.score.data(), sizeof(int32_t) * (size_t)n);
      if (res->pair_status) memcpy(res->pair_status, r.out.pair_status.data(), sizeof(int32_t) * (size_t)n);
    } else if (r.out.status == TSU_OK && res && res->cigar_offset && !(r.flags & TSU_SCORE_ONLY)) {
      res->cigar_offset[0] = 0;
      res->cigar_needed = 0;
    }
    const int st = r.out.status;
    reqs_.erase(it);
    return st;
  }

  // ---- scheduler thread: admission and watchdog
  void sched_loop() {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      for (;;) {
        if (stopping_) break;
        const bool a = admit(light_);
        const bool b = admit(heavy_);
        if (!a && !b) break;
      }
      if (stopping_) break;
      watchdog();
      const double tick = cfg_.watchdog_ms > 0 ? std::min(50.0, std::max(1.0, cfg_.watchdog_ms / 4)) : 200.0;
      cv_sched_.wait_for(lk, std::chrono::microseconds((int64_t)(tick * 1000)));
    }
  }

  void watchdog() {
    if (cfg_.watchdog_ms <= 0) return;
    const auto now = Clock::now();
    bool any = false;
    for (auto& w : workers_) {
      if (!w->busy || w->stuck || ms_between(w->started, now) <= cfg_.watchdog_ms) continue;
      w->stuck = true;
      for (auto& p : w->job) {
        if (p->req->state == Request::kDone) continue;
        fail_request(*p->req, TSU_ETIMEOUT, now);
        any = true;
      }
      err_ = "watchdog: job on worker " + std::to_string(w->idx) + " exceeded " + std::to_string(cfg_.watchdog_ms) + " ms";
    }
    if (any) cv_done_.notify_all();
  }

  size_t avail_for(const Worker* x) const {
    size_t others = 0;
    for (auto& v : workers_)
      if (v.get() != x) others += v->grant;
    return cfg_.budget > others ? cfg_.budget - others : 0;
  }

  void trim_worker(Worker* w) {
    if (w->busy) return;
    w->ex->trim();
    w->grant = w->ex->held();
  }

  // Start the head job of queue q if possible (mu_ held).  Returns whether
  // anything changed.
  bool admit(std::deque<PartPtr>& q) {
    while (!q.empty() && q.front()->req->state == Request::kDone) q.pop_front();  // failed or cancelled
    if (q.empty()) {
      if (drain_for_ == &q) drain_for_ = nullptr;
      return false;
    }
    if (drain_for_ && drain_for_ != &q) return false;
    const bool heavy = &q == &heavy_;
    if (heavy) {
      int running = 0;
      for (auto& v : workers_) running += v->busy && v->heavy;
      if (running >= cfg_.heavy_workers) return false;
    }
    Worker* w = nullptr;
    for (auto& v : workers_)
      if (!v->busy && (!w || v->grant > w->grant)) w = v.get();  // reuse the most resident memory
    if (!w) return false;
    PartPtr head = q.front();
    const uint32_t flags = head->flags;
    size_t take = 1;
    if (!heavy && !head->alone) {
      int64_t pairs = head->pairs();
      while (take < q.size() && (int)take < cfg_.max_job_requests) {
        const PartPtr& p = q[take];
        if (p->alone || p->req->state == Request::kDone || p->flags != flags ||
            pairs + p->pairs() > cfg_.max_job_pairs)
          break;
        pairs += p->pairs();
        ++take;
      }
    }
    size_t full = 0, min = 0;
    for (;;) {
      if (take == 1) {
        full = head->full;
        min = head->min;
      } else if (predict_parts(std::vector<PartPtr>(q.begin(), q.begin() + (long)take), flags, head->hint, &full,
                               &min) != TSU_OK) {
        take = 1;
        continue;
      }
      size_t avail = avail_for(w);
      if (w->grant + full <= avail) break;
      if (full <= avail) {
        trim_worker(w);
        break;
      }
      // trim idle workers, largest first, until the job fits
      while (full > avail) {
        Worker* v = nullptr;
        for (auto& u : workers_)
          if (u.get() != w && !u->busy && u->grant > 0 && (!v || u->grant > v->grant)) v = u.get();
        if (!v) break;
        trim_worker(v);
        avail = avail_for(w);
      }
      if (w->grant + full <= avail) break;
      if (full <= avail) {
        trim_worker(w);
        break;
      }
      if (take > 1) {
        take = std::max<size_t>(1, take / 2);
        continue;
      }
      // one part that does not fit at full concurrency
      bool others_busy = false;
      for (auto& v : workers_) others_busy |= v->busy;
      if (others_busy) {
        drain_for_ = &q;  // let the device drain, then run it alone
        return false;
      }
      drain_for_ = nullptr;
      trim_worker(w);
      avail = avail_for(w);
      if (min <= avail) {
        full = avail;  // run with fewer pairs in flight
        break;
      }
      q.pop_front();  // cannot fit even in an idle device
      err_ = "request " + std::to_string(head->req->id) + " needs " + std::to_string(min) + " B, budget " +
             std::to_string(cfg_.budget);
      fail_request(*head->req, TSU_ENOMEM, Clock::now());
      cv_done_.notify_all();
      return true;
    }
    // assign
    if (drain_for_ == &q) drain_for_ = nullptr;
    const auto now = Clock::now();
    w->busy = true;
    w->heavy = heavy;
    w->stuck = false;
    w->grant = w->grant + full;
    w->hint = head->hint;
    w->started = now;
    w->job.assign(q.begin(), q.begin() + (long)take);
    q.erase(q.begin(), q.begin() + (long)take);
    ++job_seq_;
    for (auto& p : w->job) {
      Request& r = *p->req;
      ++p->attempts;
      if (!r.started) {
        r.started = true;
        --waiting_;
        r.t_start = now;
        r.job_seq = job_seq_;
        r.state = Request::kRunning;
      }
      r.attempts = std::max(r.attempts, p->attempts);
    }
    ++st_jobs_;
    st_job_parts_ += (int64_t)take;
    peak_granted_ = std::max(peak_granted_, granted());
    cv_work_.notify_all();
    return true;
  }

  // ---- worker threads
  void worker_loop(Worker* w) {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_work_.wait(lk, [&] { return stopping_ || (w->busy && !w->job.empty()); });
      if (!w->busy || w->job.empty()) {
        if (stopping_) break;
        continue;
      }
      std::vector<PartPtr> job = w->job;
      const size_t grant = w->grant;
      const double hint = w->hint;
      const uint32_t flags = job[0]->flags;
      lk.unlock();
      Pairs in;  // the requests' pairs are immutable once queued
      for (auto& p : job) in.append(p->req->in, p->idx);
      w->ex->set_budget(grant);
      Output out;
      const int rc = w->ex->run(in, flags, hint, &out);
      const size_t needed = rc == TSU_ENOMEM ? w->ex->needed() : 0;
      const std::string why = rc ? w->ex->error() : std::string();
      if (w->ex->held() > cfg_.resident_cap) w->ex->trim();
      const size_t held = w->ex->held();
      const double ran_ms = ms_between(w->started, Clock::now());
      lk.lock();
      st_busy_ms_ += ran_ms;
      if (w->heavy) {
        st_heavy_busy_ms_ += ran_ms;
        ++st_heavy_jobs_;
      }
      finish(w, job, rc, out, needed, why);
      w->busy = false;
      w->heavy = false;
      w->stuck = false;
      w->job.clear();
      w->grant = held;
      cv_sched_.notify_one();
      cv_done_.notify_all();
    }
  }

  // Hand a job's output to its parts' requests (mu_ held).
  void finish(Worker* w, std::vector<PartPtr>& job, int rc, Output& out, size_t needed, const std::string& why) {
    const auto now = Clock::now();
    const bool cig = !(job[0]->req->flags & TSU_SCORE_ONLY);
    if (rc) err_ = why;
    if (rc != TSU_OK && !stopping_ && (job.size() > 1 || rc == TSU_ENOMEM)) {
      // re-queue at the head: each part alone; a single part that ran out of
      // memory gets the reservation the engine asked for
      std::vector<PartPtr> again;
      for (auto& p : job) {
        if (p->req->state == Request::kDone) continue;
        const bool retry = job.size() > 1 || (needed > w->grant && needed <= cfg_.budget && p->attempts < 3);
        if (!retry) continue;
        if (job.size() == 1) p->full = p->min = std::max(p->full, needed);
        p->alone = true;
        again.push_back(p);
      }
      for (auto it = again.rbegin(); it != again.rend(); ++it) (job[0]->heavy ? heavy_ : light_).push_front(*it);
      if (!again.empty()) {
        job.erase(std::remove_if(job.begin(), job.end(),
                                 [&](const PartPtr& p) { return std::find(again.begin(), again.end(), p) != again.end(); }),
                  job.end());
        if (job.empty()) return;
      }
    }
    int64_t k0 = 0;
    int64_t base = 0;  // offset of this part's pairs in the job
    for (auto& p : job) {
      Request& r = *p->req;
      const int64_t n = p->pairs();
      (void)k0;
      if (r.state == Request::kDone) {  // failed, cancelled or timed out meanwhile
        base += n;
        continue;
      }
      if (rc != TSU_OK) {
        fail_request(r, rc, now);
        base += n;
        continue;
      }
      Output po;
      po.score.assign(out.score.begin() + base, out.score.begin() + base + n);
      po.pair_status.assign(out.pair_status.begin() + base, out.pair_status.begin() + base + n);
      if (cig) {
        const int64_t c0 = out.coff[(size_t)base], c1 = out.coff[(size_t)(base + n)];
        po.coff.resize((size_t)n + 1);
        for (int64_t i = 0; i <= n; ++i) po.coff[(size_t)i] = out.coff[(size_t)(base + i)] - c0;
        po.cigar.assign(out.cigar.begin() + c0, out.cigar.begin() + c1);
      }
      r.done_parts.emplace_back(p, std::move(po));
      r.job_requests = std::max(r.job_requests, (int)job.size());
      base += n;
      if (--r.parts_left == 0) {
        assemble(r);
        r.state = Request::kDone;
        r.t_done = now;
        --open_;
        record_done(r);
      }
    }
  }

  Config cfg_;
  std::unique_ptr<Executor> planner_;
  std::mutex plan_mu_;  // planner_ (taken after mu_ when both are held)
  std::vector<std::unique_ptr<Worker>> workers_;
  std::thread sched_;
  std::mutex mu_;
  std::condition_variable cv_sched_, cv_work_, cv_done_;
  std::deque<PartPtr> light_, heavy_;
  std::map<uint64_t, ReqPtr> reqs_;
  int64_t open_ = 0;     // requests not done
  int64_t waiting_ = 0;  // requests none of whose parts has started
  // a head part that needs the whole device: the other queue starts nothing
  // until it has started
  const std::deque<PartPtr>* drain_for_ = nullptr;
  uint64_t next_id_ = 0;
  int64_t job_seq_ = 0;
  bool stopping_ = false, stopped_ = false;
  std::string err_;
  // statistics since the last reset
  int64_t st_submitted_ = 0, st_completed_ = 0, st_failed_ = 0, st_rejected_ = 0, st_cancelled_ = 0,
          st_timed_out_ = 0, st_jobs_ = 0, st_job_parts_ = 0, st_pairs_ = 0, st_heavy_jobs_ = 0;
  double st_busy_ms_ = 0, st_heavy_busy_ms_ = 0;
  std::vector<double> lat_;
  size_t peak_granted_ = 0;
  Clock::time_point t_reset_;
};

}  // namespace serve
}  // namespace tsu
