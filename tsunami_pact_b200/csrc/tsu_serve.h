// tsu_serve.h -- request scheduler of the alignment server (host only, no
// CUDA).  The server's C ABI (tsu_server.cpp) runs it over engine contexts;
// the tests run it over a fake executor on the CPU.
//
// No counterpart in the reference, which aligns one file per process
// (wfa_gpu.cu:43-188).  Design:
//   * submit copies a request's pairs into the server and queues it (FIFO);
//   * a pool of workers, each an Executor with its own CUDA streams and
//     device buffers, runs jobs; a job is the head request of the queue plus
//     the requests behind it (same flags, up to max_job_pairs pairs and
//     max_job_requests requests), aligned in one engine call -- continuous
//     batching: requests that arrive while others run join the next job and
//     their kernels overlap the running jobs' kernels on the device;
//   * admission: a job starts when a worker is idle and the job's predicted
//     device bytes (Executor::predict: inputs, packed words, outputs, CIGAR
//     arena and wavefront scratch at the edit-rate hint, capped by the
//     penalty-derived score bound) fit in the budget beside what the other
//     workers were granted or still hold.  Idle workers keep their buffers
//     (resident state) until the memory is needed elsewhere, then are
//     trimmed.  A job that does not fit is shrunk to its head request; a
//     head request that cannot fit even alone in an idle device is refused
//     with TSU_ENOMEM; otherwise the head waits (strict FIFO, so large
//     requests are not starved by small ones);
//   * results are split per request and made visible to poll/wait; latency
//     is measured from submit to that moment;
//   * a job of several requests that fails is re-queued at the head as
//     single-request jobs, so a failure stays with the request that caused
//     it; a single request that ran out of memory is re-queued with the
//     reservation the engine asked for (up to 3 attempts);
//   * watchdog: a job running longer than watchdog_ms completes its
//     requests with TSU_ETIMEOUT; the worker's late results are discarded
//     and it takes no new job until it returns.
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

namespace tsu {
namespace serve {

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

  void append(const Pairs& o) {
    const int64_t pb = (int64_t)pat.size(), tb = (int64_t)txt.size();
    pat.insert(pat.end(), o.pat.begin(), o.pat.end());
    txt.insert(txt.end(), o.txt.begin(), o.txt.end());
    for (int64_t v : o.poff) poff.push_back(v + pb);
    for (int64_t v : o.toff) toff.push_back(v + tb);
    plen.insert(plen.end(), o.plen.begin(), o.plen.end());
    tlen.insert(tlen.end(), o.tlen.begin(), o.tlen.end());
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
// from one thread at a time.
class Executor {
 public:
  virtual ~Executor() = default;
  // Predicted device bytes to align `plen`/`tlen` (n pairs, pb/tb sequence
  // bytes) in one call: every pair of a band in flight (*full) or one (*min).
  virtual int predict(int64_t n, const int32_t* plen, const int32_t* tlen, int64_t pb, int64_t tb, uint32_t flags,
                      size_t* full, size_t* min) = 0;
  virtual size_t held() = 0;                 // device bytes held now
  virtual void set_budget(size_t bytes) = 0;  // for the next run
  virtual int trim() = 0;                    // release every buffer
  // Align every pair; fills out->score and out->pair_status (and CIGARs).
  virtual int run(const Pairs& in, uint32_t flags, Output* out) = 0;
  virtual size_t needed() = 0;  // after TSU_ENOMEM: the bytes the run needed (0: unknown)
  virtual std::string error() = 0;
};

struct Config {
  int workers = 4;
  size_t budget = 0;               // device bytes for all workers
  int64_t max_queue = 1 << 16;     // queued requests before submit says TSU_EBUSY
  int64_t max_job_pairs = 16384;   // pairs merged into one job
  int max_job_requests = 64;       // requests merged into one job
  double watchdog_ms = 0;          // 0: off
  size_t resident_cap = 0;         // bytes an idle worker may keep (0: budget / (2 * workers))
};

struct Request {
  uint64_t id = 0;
  Pairs in;
  uint32_t flags = 0;
  size_t full = 0, min = 0;  // predicted bytes alone
  enum State { kQueued, kRunning, kDone } state = kQueued;
  bool cancelled = false;
  bool alone = false;  // run as a job of its own (after a job-level failure)
  int attempts = 0;
  int job_requests = 0;
  int64_t job_seq = 0;
  Clock::time_point t_submit, t_start, t_done;
  Output out;
};
using ReqPtr = std::shared_ptr<Request>;

class Server {
 public:
  Server(const Config& cfg, std::vector<std::unique_ptr<Executor>> workers, std::unique_ptr<Executor> planner)
      : cfg_(cfg), planner_(std::move(planner)) {
    if (cfg_.resident_cap == 0) cfg_.resident_cap = cfg_.budget / (2 * std::max<size_t>(1, workers.size()));
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

  // Cancel queued requests, let running jobs finish, stop the threads.
  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (stopped_) return;
      stopping_ = true;
      for (auto& r : queue_) {
        r->state = Request::kDone;
        r->out.status = TSU_EBUSY;
        r->t_done = Clock::now();
      }
      queue_.clear();
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
    r->flags = flags & TSU_SCORE_ONLY;
    r->in.assign(*b);
    if (r->in.n()) {
      std::lock_guard<std::mutex> pl(plan_mu_);
      const int rc = planner_->predict(r->in.n(), r->in.plen.data(), r->in.tlen.data(), (int64_t)r->in.pat.size(),
                                       (int64_t)r->in.txt.size(), r->flags, &r->full, &r->min);
      if (rc) return rc;
    }
    std::lock_guard<std::mutex> lk(mu_);
    if (stopping_) return TSU_EBUSY;
    if (r->min > cfg_.budget) {
      ++st_rejected_;
      err_ = "request needs " + std::to_string(r->min) + " B of device memory, budget " + std::to_string(cfg_.budget);
      return TSU_ENOMEM;
    }
    if ((int64_t)queue_.size() >= cfg_.max_queue) {
      ++st_rejected_;
      err_ = "queue full";
      return TSU_EBUSY;
    }
    r->id = ++next_id_;
    *id = r->id;
    ++st_submitted_;
    reqs_[r->id] = r;
    if (r->in.n() == 0) {  // nothing to align
      r->state = Request::kDone;
      r->t_start = r->t_done = r->t_submit;
      record_done(*r);
      cv_done_.notify_all();
      return TSU_OK;
    }
    queue_.push_back(r);
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

  // Queued: removed.  Running: its results are dropped when the job ends.
  // Done: forgotten.
  int cancel(uint64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return TSU_ENOTFOUND;
    ReqPtr r = it->second;
    reqs_.erase(it);
    if (r->state == Request::kQueued) {
      queue_.erase(std::remove(queue_.begin(), queue_.end(), r), queue_.end());
      r->state = Request::kDone;
      r->out.status = TSU_EBUSY;
    }
    r->cancelled = true;
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
    s->queued = (int64_t)queue_.size();
    for (auto& w : workers_) s->running += w->busy ? (int64_t)w->job.size() : 0;
    s->jobs = st_jobs_;
    s->pairs_completed = st_pairs_;
    s->mean_requests_per_job = st_jobs_ ? (double)st_job_reqs_ / (double)st_jobs_ : 0.0;
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
  }

  void reset_stats() {
    std::lock_guard<std::mutex> lk(mu_);
    st_submitted_ = st_completed_ = st_failed_ = st_rejected_ = st_cancelled_ = st_timed_out_ = 0;
    st_jobs_ = st_job_reqs_ = st_pairs_ = 0;
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
    bool stuck = false;  // the watchdog completed its requests
    size_t grant = 0;    // bytes granted to the running job, or held while idle
    std::vector<ReqPtr> job;
    Clock::time_point started;
  };

  size_t granted() const {
    size_t g = 0;
    for (auto& w : workers_) g += w->grant;
    return g;
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
      while (!stopping_ && admit_one()) {
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
      for (auto& r : w->job) {
        if (r->state == Request::kDone) continue;
        r->state = Request::kDone;
        r->out = Output{};
        r->out.status = TSU_ETIMEOUT;
        r->t_done = now;
        record_done(*r);
        any = true;
      }
      err_ = "watchdog: job on worker " + std::to_string(w->idx) + " exceeded " + std::to_string(cfg_.watchdog_ms) + " ms";
    }
    if (any) cv_done_.notify_all();
  }

  // Start one job if possible (mu_ held).  Returns whether anything changed.
  bool admit_one() {
    while (!queue_.empty() && queue_.front()->cancelled) queue_.pop_front();
    if (queue_.empty()) return false;
    Worker* w = nullptr;
    for (auto& v : workers_)
      if (!v->busy && (!w || v->grant > w->grant)) w = v.get();  // reuse the most resident memory
    if (!w) return false;
    ReqPtr head = queue_.front();
    // candidate job: the head and the requests behind it
    size_t take = 1;
    if (!head->alone) {
      int64_t pairs = head->in.n();
      while (take < queue_.size() && (int)take < cfg_.max_job_requests) {
        const ReqPtr& r = queue_[take];
        if (r->alone || r->cancelled || r->flags != head->flags || pairs + r->in.n() > cfg_.max_job_pairs) break;
        pairs += r->in.n();
        ++take;
      }
    }
    auto avail_for = [&](Worker* x) {
      size_t others = 0;
      for (auto& v : workers_)
        if (v.get() != x) others += v->grant;
      return cfg_.budget > others ? cfg_.budget - others : 0;
    };
    size_t full = 0, min = 0;
    for (;;) {
      if (take == 1) {
        full = head->full;
        min = head->min;
      } else if (!predict_job(take, &full, &min)) {
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
      // the head alone does not fit at full concurrency
      bool others_busy = false;
      for (auto& v : workers_) others_busy |= v->busy;
      if (!others_busy) {
        trim_worker(w);
        avail = avail_for(w);
        if (min <= avail) {
          full = avail;  // run with fewer pairs in flight
          break;
        }
        // cannot fit even in an idle device
        queue_.pop_front();
        head->state = Request::kDone;
        head->out = Output{};
        head->out.status = TSU_ENOMEM;
        head->t_start = head->t_done = Clock::now();
        record_done(*head);
        err_ = "request " + std::to_string(head->id) + " needs " + std::to_string(min) + " B, budget " +
               std::to_string(cfg_.budget);
        cv_done_.notify_all();
        return true;
      }
      return false;  // wait for running jobs to finish
    }
    // assign
    const auto now = Clock::now();
    w->busy = true;
    w->stuck = false;
    w->grant = w->grant + full;
    w->started = now;
    w->job.assign(queue_.begin(), queue_.begin() + (long)take);
    queue_.erase(queue_.begin(), queue_.begin() + (long)take);
    ++job_seq_;
    for (auto& r : w->job) {
      r->state = Request::kRunning;
      r->t_start = now;
      r->job_requests = (int)take;
      r->job_seq = job_seq_;
      ++r->attempts;
    }
    ++st_jobs_;
    st_job_reqs_ += (int64_t)take;
    peak_granted_ = std::max(peak_granted_, granted());
    cv_work_.notify_all();
    return true;
  }

  bool predict_job(size_t take, size_t* full, size_t* min) {
    std::vector<int32_t> pl, tl;
    int64_t pb = 0, tb = 0;
    for (size_t i = 0; i < take; ++i) {
      const Pairs& p = queue_[i]->in;
      pl.insert(pl.end(), p.plen.begin(), p.plen.end());
      tl.insert(tl.end(), p.tlen.begin(), p.tlen.end());
      pb += (int64_t)p.pat.size();
      tb += (int64_t)p.txt.size();
    }
    std::lock_guard<std::mutex> pl_lk(plan_mu_);
    return planner_->predict((int64_t)pl.size(), pl.data(), tl.data(), pb, tb, queue_.front()->flags, full, min) ==
           TSU_OK;
  }

  void trim_worker(Worker* w) {
    if (w->busy) return;
    w->ex->trim();
    w->grant = w->ex->held();
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
      std::vector<ReqPtr> job = w->job;
      const size_t grant = w->grant;
      lk.unlock();
      Pairs merged;
      const Pairs* in = &job[0]->in;
      if (job.size() > 1) {
        for (auto& r : job) merged.append(r->in);
        in = &merged;
      }
      w->ex->set_budget(grant);
      Output out;
      const int rc = w->ex->run(*in, job[0]->flags, &out);
      const size_t needed = rc == TSU_ENOMEM ? w->ex->needed() : 0;
      const std::string why = rc ? w->ex->error() : std::string();
      if (w->ex->held() > cfg_.resident_cap) w->ex->trim();
      const size_t held = w->ex->held();
      lk.lock();
      finish(w, job, rc, out, needed, why);
      w->busy = false;
      w->stuck = false;
      w->job.clear();
      w->grant = held;
      cv_sched_.notify_one();
      cv_done_.notify_all();
    }
  }

  // Split a job's output per request (mu_ held).
  void finish(Worker* w, std::vector<ReqPtr>& job, int rc, Output& out, size_t needed, const std::string& why) {
    const auto now = Clock::now();
    const bool cig = !(job[0]->flags & TSU_SCORE_ONLY);
    if (rc) err_ = why;
    if (rc != TSU_OK && !stopping_ && (job.size() > 1 || rc == TSU_ENOMEM)) {
      // re-queue at the head, each request alone, so a failure stays with
      // the request that caused it; a single request that ran out of memory
      // gets the reservation the engine asked for
      std::vector<ReqPtr> again;
      for (auto& r : job) {
        if (r->cancelled || r->state == Request::kDone) continue;
        const bool retry = job.size() > 1 || (needed > w->grant && needed <= cfg_.budget && r->attempts < 3);
        if (!retry) continue;
        if (job.size() == 1) r->full = r->min = std::max(r->full, needed);
        r->alone = true;
        r->state = Request::kQueued;
        again.push_back(r);
      }
      for (auto it = again.rbegin(); it != again.rend(); ++it) queue_.push_front(*it);
    }
    int64_t p0 = 0;
    for (auto& rp : job) {
      Request& r = *rp;
      const int64_t n = r.in.n();
      const int64_t p1 = p0 + n;
      if (r.state == Request::kQueued || r.cancelled || r.state == Request::kDone) {
        p0 = p1;
        continue;  // re-queued, cancelled, or completed by the watchdog
      }
      r.out = Output{};
      if (rc == TSU_OK) {
        r.out.score.assign(out.score.begin() + p0, out.score.begin() + p1);
        r.out.pair_status.assign(out.pair_status.begin() + p0, out.pair_status.begin() + p1);
        if (cig) {
          const int64_t c0 = out.coff[(size_t)p0], c1 = out.coff[(size_t)p1];
          r.out.coff.resize((size_t)n + 1);
          for (int64_t i = 0; i <= n; ++i) r.out.coff[(size_t)i] = out.coff[(size_t)(p0 + i)] - c0;
          r.out.cigar.assign(out.cigar.begin() + c0, out.cigar.begin() + c1);
        }
      } else {
        r.out.status = rc;
      }
      r.state = Request::kDone;
      r.t_done = now;
      record_done(r);
      p0 = p1;
    }
    (void)w;
  }

  Config cfg_;
  std::unique_ptr<Executor> planner_;
  std::mutex plan_mu_;  // planner_ (taken after mu_ when both are held)
  std::vector<std::unique_ptr<Worker>> workers_;
  std::thread sched_;
  std::mutex mu_;
  std::condition_variable cv_sched_, cv_work_, cv_done_;
  std::deque<ReqPtr> queue_;
  std::map<uint64_t, ReqPtr> reqs_;
  uint64_t next_id_ = 0;
  int64_t job_seq_ = 0;
  bool stopping_ = false, stopped_ = false;
  std::string err_;
  // statistics since the last reset
  int64_t st_submitted_ = 0, st_completed_ = 0, st_failed_ = 0, st_rejected_ = 0, st_cancelled_ = 0,
          st_timed_out_ = 0, st_jobs_ = 0, st_job_reqs_ = 0, st_pairs_ = 0;
  std::vector<double> lat_;
  size_t peak_granted_ = 0;
  Clock::time_point t_reset_;
};

}  // namespace serve
}  // namespace tsu
