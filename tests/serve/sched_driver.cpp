// sched_driver.cpp -- the request scheduler (tsunami_pact_b200/csrc/tsu_serve.h)
// over a fake executor, on the CPU, for tests/test_serve_host.py.
//
// The fake "aligns" a pair by a checksum of its two sequences (score) and a
// few runs derived from it (CIGAR), after a delay the pattern's first byte
// encodes; it predicts memory from the sequence bytes and, like the engine,
// holds at most its budget while it runs and keeps its buffers afterwards.
// Every scenario checks the scheduler's invariants: each request's results
// are those of its own pairs, the fakes never hold more than the server's
// budget together, and requests start in submission order (job numbers).
//
// usage: sched_driver <scenario>   -> prints "ok <scenario>" and exits 0
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../tsunami_pact_b200/csrc/tsu_serve.h"

using namespace tsu::serve;

namespace {

std::atomic<int64_t> g_held_total{0};  // bytes all fakes hold
std::atomic<int64_t> g_held_peak{0};
std::atomic<int> g_running{0};
std::atomic<int> g_running_peak{0};
std::atomic<int> g_runs{0};
std::atomic<int> g_heavy_running{0};
std::atomic<int> g_heavy_peak{0};
size_t g_budget = 0;
std::mutex g_log_mu;
std::vector<int> g_run_log;  // request tags of the pairs each run saw

[[noreturn]] void fail(const std::string& why) {
  fprintf(stderr, "FAIL: %s\n", why.c_str());
  fflush(stderr);
  std::_Exit(1);
}
#define CHECK(c)                                                   \
  do {                                                             \
    if (!(c)) fail(std::string(#c) + " at line " + std::to_string(__LINE__)); \
  } while (0)

uint32_t checksum(const char* p, int32_t m, const char* t, int32_t n) {
  uint32_t h = 2166136261u;
  for (int32_t i = 0; i < m; ++i) h = (h ^ (uint8_t)p[i]) * 16777619u;
  h = (h ^ 0xffu) * 16777619u;
  for (int32_t i = 0; i < n; ++i) h = (h ^ (uint8_t)t[i]) * 16777619u;
  return h;
}
int32_t fake_score(uint32_t h) { return (int32_t)(h & 0x7fffffff); }
int fake_runs(uint32_t h) { return 1 + (int)(h % 3); }

struct FakeOpts {
  double bytes_per_base = 10.0;
  size_t fixed = 1000;
  double min_frac = 0.25;
  int delay_unit_us = 200;  // per unit of the pattern's first byte - 'A'
  bool fail_on_bang = true;  // a pattern starting with '!' fails the run
  double merged_factor = 1.0;  // memory a run of several requests needs, x its prediction
  int32_t heavy_len = 1 << 30;  // runs with a pair this long count as heavy
};
FakeOpts g_opts;
std::atomic<int> g_lowmem_runs{0};

class Fake final : public Executor {
 public:
  int predict(int64_t n, const int32_t* plen, const int32_t* tlen, int64_t pb, int64_t tb, uint32_t flags, double,
              size_t* full, size_t* min) override {
    (void)n;
    (void)plen;
    (void)tlen;
    *full = g_opts.fixed + (size_t)(g_opts.bytes_per_base * (double)(pb + tb));
    if (flags & kLowMem) *full /= 8;  // checkpointed history: an eighth
    *min = (size_t)((double)*full * g_opts.min_frac);
    return TSU_OK;
  }
  size_t held() override { return held_; }
  void set_budget(size_t b) override { budget_ = b; }
  int trim() override {
    hold(0);
    return TSU_OK;
  }
  size_t needed() override { return needed_; }
  std::string error() override { return "fake error"; }

  int run(const Pairs& in, uint32_t flags, double hint, Output* out) override {
    const int64_t n = in.n();
    size_t full = 0, min = 0;
    predict(n, in.plen.data(), in.tlen.data(), (int64_t)in.pat.size(), (int64_t)in.txt.size(), flags, hint, &full, &min);
    int tags = 0;
    for (int64_t i = 0; i < n; ++i) tags += in.plen[(size_t)i] >= 2 && in.pat[(size_t)in.poff[(size_t)i] + 1] == '#';
    if (tags > 1) {
      full = (size_t)((double)full * g_opts.merged_factor);
      min = (size_t)((double)min * g_opts.merged_factor);
    }
    needed_ = 0;
    if (min > budget_) {
      needed_ = min;
      return TSU_ENOMEM;
    }
    hold(std::max(held_, std::min(full, budget_)));
    if (held_ > budget_) fail("fake holds more than its budget");
    const int r = ++g_running;
    int pk = g_running_peak.load();
    while (r > pk && !g_running_peak.compare_exchange_weak(pk, r)) {
    }
    bool heavy = false;
    for (int64_t i = 0; i < n; ++i) heavy |= std::max(in.plen[(size_t)i], in.tlen[(size_t)i]) >= g_opts.heavy_len;
    if (heavy) {
      if (n != 1) fail("a heavy pair shares a job");
      const int h = ++g_heavy_running;
      int hp = g_heavy_peak.load();
      while (h > hp && !g_heavy_peak.compare_exchange_weak(hp, h)) {
      }
    }
    ++g_runs;
    if (flags & kLowMem) ++g_lowmem_runs;
    {
      std::lock_guard<std::mutex> lk(g_log_mu);
      for (int64_t i = 0; i < n; ++i)
        if (in.plen[(size_t)i] >= 2 && in.pat[(size_t)in.poff[(size_t)i] + 1] == '#') {
          // pair tagged with its request number: "?#<tag>..."
          g_run_log.push_back(atoi(in.pat.data() + in.poff[(size_t)i] + 2));
        }
    }
    int delay = 0;
    bool bad = false;
    for (int64_t i = 0; i < n; ++i) {
      if (in.plen[(size_t)i] == 0) continue;
      const char c = in.pat[(size_t)in.poff[(size_t)i]];
      if (c == '!' && g_opts.fail_on_bang) bad = true;
      if (c >= 'A' && c <= 'Z') delay = std::max(delay, (c - 'A') * g_opts.delay_unit_us);
    }
    std::this_thread::sleep_for(std::chrono::microseconds(delay));
    --g_running;
    if (heavy) --g_heavy_running;
    if (bad) return TSU_EINTERNAL;
    out->score.resize((size_t)n);
    out->pair_status.assign((size_t)n, 0);
    const bool cig = !(flags & TSU_SCORE_ONLY);
    if (cig) out->coff.assign((size_t)n + 1, 0);
    out->cigar.clear();
    for (int64_t i = 0; i < n; ++i) {
      const uint32_t h = checksum(in.pat.data() + in.poff[(size_t)i], in.plen[(size_t)i],
                                  in.txt.data() + in.toff[(size_t)i], in.tlen[(size_t)i]);
      out->score[(size_t)i] = fake_score(h);
      if (cig) {
        for (int k = 0; k < fake_runs(h); ++k) out->cigar.push_back((h >> k) & 0xffffu);
        out->coff[(size_t)i + 1] = (int64_t)out->cigar.size();
      }
    }
    return TSU_OK;
  }

  ~Fake() override { hold(0); }

 private:
  void hold(size_t b) {
    g_held_total += (int64_t)b - (int64_t)held_;
    held_ = b;
    const int64_t t = g_held_total.load();
    int64_t pk = g_held_peak.load();
    while (t > pk && !g_held_peak.compare_exchange_weak(pk, t)) {
    }
    if (g_budget && t > (int64_t)g_budget) fail("fakes hold " + std::to_string(t) + " B > budget " + std::to_string(g_budget));
  }
  size_t budget_ = 0, held_ = 0, needed_ = 0;
};

std::unique_ptr<Server> make_server(Config c) {
  g_budget = c.budget;
  std::vector<std::unique_ptr<Executor>> ws;
  for (int i = 0; i < c.workers; ++i) ws.emplace_back(new Fake());
  return std::make_unique<Server>(c, std::move(ws), std::unique_ptr<Executor>(new Fake()));
}

// A request: n pairs; the first pair's pattern is "<delay>#<tag>" padded.
struct Req {
  std::vector<std::string> p, t;
  std::string ps, ts;
  std::vector<int64_t> po, to;
  std::vector<int32_t> pl, tl;
  tsu_batch b{};
  void build() {
    ps.clear();
    ts.clear();
    po.clear();
    to.clear();
    pl.clear();
    tl.clear();
    for (size_t i = 0; i < p.size(); ++i) {
      po.push_back((int64_t)ps.size());
      to.push_back((int64_t)ts.size());
      ps += p[i];
      ts += t[i];
      pl.push_back((int32_t)p[i].size());
      tl.push_back((int32_t)t[i].size());
    }
  }
  // the batch view, with pointers into this object as it is now
  const tsu_batch* bp() {
    b = tsu_batch{(int64_t)p.size(), ps.data(), po.data(), pl.data(), ts.data(), to.data(), tl.data()};
    return &b;
  }
};

Req make_req(std::mt19937& rng, int tag, int npairs, char delay = 'A', int len = 20) {
  Req r;
  for (int i = 0; i < npairs; ++i) {
    std::string a, b;
    for (int k = 0; k < len; ++k) a += "ACGT"[rng() % 4];
    for (int k = 0; k < len; ++k) b += "ACGT"[rng() % 4];
    if (i == 0) {
      std::string head = std::string(1, delay) + "#" + std::to_string(tag) + ".";
      a = head + a;
    }
    r.p.push_back(a);
    r.t.push_back(b);
  }
  r.build();
  return r;
}

// A request of short pairs with long ones (len_long) at positions `longs`;
// every pair's pattern starts with the delay letter.
Req make_mixed(std::mt19937& rng, int tag, int npairs, const std::vector<int>& longs, int len_long, char delay) {
  Req r = make_req(rng, tag, npairs, delay, 20);
  for (int i : longs) {
    std::string a(1, delay), b;
    for (int k = 1; k < len_long; ++k) a += "ACGT"[rng() % 4];
    for (int k = 0; k < len_long; ++k) b += "ACGT"[rng() % 4];
    r.p[(size_t)i] = a;
    r.t[(size_t)i] = b;
  }
  r.build();
  return r;
}

// Wait for id and check its results against its own pairs.
int check_result(Server& s, uint64_t id, const Req& r, bool cigar, double timeout_ms = 20000,
                 tsu_request_info* info_out = nullptr) {
  const int64_t n = (int64_t)r.p.size();
  std::vector<int32_t> sc((size_t)n, -1), ps((size_t)n, -1);
  std::vector<int64_t> co((size_t)n + 1, -1);
  std::vector<uint32_t> cg(4 * (size_t)n + 1);
  tsu_result res{sc.data(), cg.data(), (int64_t)cg.size(), co.data(), 0, ps.data()};
  tsu_request_info info{};
  const int rc = s.wait(id, timeout_ms, &res, &info);
  if (info_out) *info_out = info;
  if (rc != TSU_OK) return rc;
  CHECK(info.num_pairs == n);
  CHECK(info.latency_ms >= info.queue_ms);
  std::vector<uint32_t> want;
  for (int64_t i = 0; i < n; ++i) {
    const uint32_t h = checksum(r.p[(size_t)i].data(), (int32_t)r.p[(size_t)i].size(), r.t[(size_t)i].data(),
                                (int32_t)r.t[(size_t)i].size());
    CHECK(sc[(size_t)i] == fake_score(h));
    CHECK(ps[(size_t)i] == 0);
    if (cigar) {
      CHECK(co[(size_t)i] == (int64_t)want.size());
      for (int k = 0; k < fake_runs(h); ++k) want.push_back((h >> k) & 0xffffu);
    }
  }
  if (cigar) {
    CHECK(co[(size_t)n] == (int64_t)want.size());
    CHECK(res.cigar_needed == (int64_t)want.size());
    for (size_t k = 0; k < want.size(); ++k) CHECK(cg[k] == want[k]);
  }
  return TSU_OK;
}

// Requests given in submission order start in that order.
void check_fifo(const std::vector<tsu_request_info>& infos) {
  for (size_t i = 1; i < infos.size(); ++i)
    if (infos[i].job_seq < infos[i - 1].job_seq)
      fail("request " + std::to_string(i) + " started before request " + std::to_string(i - 1));
}

// Wait for every request, check it, check FIFO.
void check_all(Server& s, const std::vector<uint64_t>& ids, const std::vector<Req>& rs, bool cigar) {
  std::vector<tsu_request_info> infos(ids.size());
  for (size_t i = 0; i < rs.size(); ++i) CHECK(check_result(s, ids[i], rs[i], cigar, 20000, &infos[i]) == TSU_OK);
  check_fifo(infos);
}

// ---- scenarios
void basic() {
  std::mt19937 rng(1);
  Config c;
  c.workers = 3;
  c.budget = 1 << 30;
  auto s = make_server(c);
  std::vector<Req> rs;
  std::vector<uint64_t> ids;
  for (int i = 0; i < 60; ++i) rs.push_back(make_req(rng, i, 1 + (int)(rng() % 40), 'F'));
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  check_all(*s, ids, rs, true);
  tsu_server_stats st{};
  s->stats(&st);
  CHECK(st.completed == 60 && st.failed == 0 && st.pairs_completed > 0);
  CHECK(st.jobs < 60);  // requests that queued behind a running job were merged
  CHECK(st.mean_requests_per_job > 1.0);
  CHECK(st.p50_ms <= st.p99_ms && st.p99_ms <= st.p999_ms && st.p999_ms <= st.max_ms);
  CHECK(s->poll(ids[0], nullptr, nullptr) == TSU_ENOTFOUND);  // taken
}

void score_only() {
  std::mt19937 rng(2);
  Config c;
  c.workers = 2;
  c.budget = 1 << 30;
  auto s = make_server(c);
  std::vector<Req> rs;
  std::vector<uint64_t> ids;
  for (int i = 0; i < 20; ++i) rs.push_back(make_req(rng, i, 5));
  for (size_t i = 0; i < rs.size(); ++i) {
    uint64_t id = 0;
    CHECK(s->submit(rs[i].bp(), i % 2 ? TSU_SCORE_ONLY : 0, &id) == TSU_OK);  // mixed flags never share a job
    ids.push_back(id);
  }
  for (size_t i = 0; i < rs.size(); ++i) CHECK(check_result(*s, ids[i], rs[i], i % 2 == 0) == TSU_OK);
}

void admission() {
  // each request predicts ~60% of the budget: never two at once
  std::mt19937 rng(3);
  Config c;
  c.workers = 4;
  Req probe = make_req(rng, 0, 8, 'F', 100);
  size_t full = g_opts.fixed + (size_t)(g_opts.bytes_per_base * (double)(probe.ps.size() + probe.ts.size()));
  c.budget = (size_t)((double)full / 0.6);
  c.max_job_requests = 1;
  auto s = make_server(c);
  std::vector<Req> rs;
  std::vector<uint64_t> ids;
  for (int i = 0; i < 10; ++i) rs.push_back(make_req(rng, i, 8, 'F', 100));
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  check_all(*s, ids, rs, true);
  CHECK(g_running_peak.load() == 1);
  CHECK(g_held_peak.load() <= (int64_t)c.budget);
  tsu_server_stats st{};
  s->stats(&st);
  CHECK(st.peak_granted_bytes <= c.budget);
}

void concurrency() {
  // small requests, roomy budget: jobs overlap
  std::mt19937 rng(4);
  Config c;
  c.workers = 4;
  c.budget = 1 << 30;
  c.max_job_requests = 1;
  auto s = make_server(c);
  std::vector<Req> rs;
  std::vector<uint64_t> ids;
  for (int i = 0; i < 16; ++i) rs.push_back(make_req(rng, i, 2, 'K'));
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  for (size_t i = 0; i < rs.size(); ++i) CHECK(check_result(*s, ids[i], rs[i], true) == TSU_OK);
  CHECK(g_running_peak.load() >= 2);
}

void reject() {
  std::mt19937 rng(5);
  Config c;
  c.workers = 2;
  c.budget = 2000;
  auto s = make_server(c);
  Req big = make_req(rng, 0, 50, 'A', 100);  // min ~ 0.25 * 10 * 10000 B > budget
  uint64_t id = 0;
  CHECK(s->submit(big.bp(), 0, &id) == TSU_ENOMEM);
  Req small = make_req(rng, 1, 1, 'A', 5);
  CHECK(s->submit(small.bp(), 0, &id) == TSU_OK);
  CHECK(check_result(*s, id, small, true) == TSU_OK);
  tsu_server_stats st{};
  s->stats(&st);
  CHECK(st.rejected == 1 && st.completed == 1);
  // bad input
  Req bad = make_req(rng, 2, 2);
  bad.pl[1] = -3;
  CHECK(s->submit(bad.bp(), 0, &id) == TSU_EINVAL);
  CHECK(s->submit(nullptr, 0, &id) == TSU_EINVAL);
}

void degraded() {
  // a request whose full prediction exceeds the budget but whose minimum
  // fits runs alone with the whole budget
  std::mt19937 rng(6);
  Config c;
  c.workers = 2;
  Req r = make_req(rng, 0, 4, 'B', 100);
  const size_t full = g_opts.fixed + (size_t)(g_opts.bytes_per_base * (double)(r.ps.size() + r.ts.size()));
  c.budget = full / 2;
  auto s = make_server(c);
  uint64_t id = 0;
  CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
  CHECK(check_result(*s, id, r, true) == TSU_OK);
  CHECK(g_held_peak.load() <= (int64_t)c.budget);
}

void lowmem() {
  // a CIGAR request whose smallest footprint exceeds the budget runs in
  // low-memory mode (its footprint an eighth) instead of failing; the same
  // request score-only has no such mode and is rejected
  std::mt19937 rng(19);
  Config c;
  c.workers = 2;
  Req r = make_req(rng, 0, 4, 'B', 100);
  const size_t full = g_opts.fixed + (size_t)(g_opts.bytes_per_base * (double)(r.ps.size() + r.ts.size()));
  c.budget = (size_t)((double)full * g_opts.min_frac / 2);
  auto s = make_server(c);
  uint64_t id = 0;
  CHECK(s->submit(r.bp(), TSU_SCORE_ONLY, &id) == TSU_ENOMEM);
  CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
  CHECK(check_result(*s, id, r, true) == TSU_OK);
  CHECK(g_lowmem_runs.load() >= 1);
  CHECK(g_held_peak.load() <= (int64_t)c.budget);
}

void fifo() {
  // a large head request waits for memory; the small ones behind it do not
  // overtake it
  std::mt19937 rng(7);
  Config c;
  c.workers = 4;
  c.max_job_requests = 1;
  Req big = make_req(rng, 1, 4, 'D', 200);
  const size_t big_full = g_opts.fixed + (size_t)(g_opts.bytes_per_base * (double)(big.ps.size() + big.ts.size()));
  c.budget = big_full + big_full / 10;
  auto s = make_server(c);
  std::vector<Req> rs;
  rs.push_back(make_req(rng, 0, 4, 'T', 40));  // long-running, holds memory
  rs.push_back(big);
  for (int i = 2; i < 12; ++i) rs.push_back(make_req(rng, i, 1, 'B', 10));
  std::vector<uint64_t> ids;
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  check_all(*s, ids, rs, true);
}

void cancel() {
  std::mt19937 rng(8);
  Config c;
  c.workers = 1;
  c.budget = 1 << 30;
  c.max_job_requests = 1;
  g_opts.delay_unit_us = 2000;  // 'Z' = 50 ms
  auto s = make_server(c);
  Req slow = make_req(rng, 0, 1, 'Z');
  Req q1 = make_req(rng, 1, 1), q2 = make_req(rng, 2, 1);
  uint64_t a = 0, b = 0, d = 0;
  CHECK(s->submit(slow.bp(), 0, &a) == TSU_OK);
  std::this_thread::sleep_for(std::chrono::milliseconds(1));
  CHECK(s->submit(q1.bp(), 0, &b) == TSU_OK);
  CHECK(s->submit(q2.bp(), 0, &d) == TSU_OK);
  CHECK(s->cancel(b) == TSU_OK);  // queued: never runs
  CHECK(s->cancel(b) == TSU_ENOTFOUND);
  CHECK(s->poll(b, nullptr, nullptr) == TSU_ENOTFOUND);
  CHECK(check_result(*s, a, slow, true) == TSU_OK);
  CHECK(check_result(*s, d, q2, true) == TSU_OK);
  {
    std::lock_guard<std::mutex> lk(g_log_mu);
    for (int tag : g_run_log) CHECK(tag != 1);
  }
  // cancel while running: result dropped
  Req slow2 = make_req(rng, 3, 1, 'Z');
  CHECK(s->submit(slow2.bp(), 0, &a) == TSU_OK);
  std::this_thread::sleep_for(std::chrono::milliseconds(10));
  CHECK(s->cancel(a) == TSU_OK);
  CHECK(s->wait(a, 1000, nullptr, nullptr) == TSU_ENOTFOUND);
  tsu_server_stats st{};
  s->stats(&st);
  CHECK(st.cancelled == 2);
}

void pending() {
  std::mt19937 rng(9);
  Config c;
  c.workers = 1;
  c.budget = 1 << 30;
  auto s = make_server(c);
  Req slow = make_req(rng, 0, 1, 'Z');
  uint64_t a = 0;
  CHECK(s->submit(slow.bp(), 0, &a) == TSU_OK);
  std::vector<int32_t> sc(1);
  std::vector<int64_t> co(2);
  std::vector<uint32_t> cg(1);
  tsu_result res{sc.data(), cg.data(), 0, co.data(), 0, nullptr};
  CHECK(s->poll(a, &res, nullptr) == TSU_EPENDING);
  CHECK(s->wait(a, 0.5, &res, nullptr) == TSU_ETIMEOUT);
  // too small a CIGAR buffer: overflow, request kept
  CHECK(s->wait(a, 20000, &res, nullptr) == TSU_EOVERFLOW);
  CHECK(res.cigar_needed > 0);
  CHECK(check_result(*s, a, slow, true) == TSU_OK);
}

void watchdog() {
  std::mt19937 rng(10);
  g_opts.delay_unit_us = 12000;  // 'Z' = 300 ms
  Config c;
  c.workers = 2;
  c.budget = 1 << 30;
  c.watchdog_ms = 40;
  c.max_job_requests = 1;
  auto s = make_server(c);
  Req hang = make_req(rng, 0, 1, 'Z');
  Req quick = make_req(rng, 1, 1, 'A');
  uint64_t a = 0, b = 0;
  CHECK(s->submit(hang.bp(), 0, &a) == TSU_OK);
  CHECK(s->submit(quick.bp(), 0, &b) == TSU_OK);
  const auto t0 = Clock::now();
  CHECK(s->wait(a, 5000, nullptr, nullptr) == TSU_ETIMEOUT);  // the request's status
  CHECK(ms_between(t0, Clock::now()) < 250);                  // before the job returned
  CHECK(check_result(*s, b, quick, true) == TSU_OK);          // the other worker serves on
  tsu_server_stats st{};
  s->stats(&st);
  CHECK(st.timed_out == 1);
  CHECK(s->error().find("watchdog") != std::string::npos);
}

void nomem_retry() {
  // merged jobs that fail on memory are re-run request by request
  std::mt19937 rng(11);
  g_opts.min_frac = 1.0;       // the fake fails below its full prediction
  g_opts.merged_factor = 2.0;  // and a merged job needs twice what was predicted
  Config c;
  c.workers = 1;
  auto s_probe = make_req(rng, 0, 3, 'A', 50);
  const size_t full = g_opts.fixed + (size_t)(g_opts.bytes_per_base * (double)(s_probe.ps.size() + s_probe.ts.size()));
  c.budget = 4 * full;
  auto s = make_server(c);
  std::vector<Req> rs;
  std::vector<uint64_t> ids;
  Req blocker = make_req(rng, 100, 1, 'Q');
  uint64_t bid = 0;
  CHECK(s->submit(blocker.bp(), 0, &bid) == TSU_OK);
  for (int i = 0; i < 6; ++i) rs.push_back(make_req(rng, i, 3, 'A', 50));
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  CHECK(check_result(*s, bid, blocker, true) == TSU_OK);
  int retried = 0;
  for (size_t i = 0; i < rs.size(); ++i) {
    tsu_request_info info{};
    CHECK(check_result(*s, ids[i], rs[i], true, 20000, &info) == TSU_OK);
    retried += info.attempts > 1;
    CHECK(info.attempts == 1 || info.job_requests == 1);  // a retry runs alone
  }
  CHECK(retried > 0);
}

void failure_isolation() {
  // a request whose job fails is re-run alone; only it fails
  std::mt19937 rng(12);
  Config c;
  c.workers = 1;
  c.budget = 1 << 30;
  auto s = make_server(c);
  Req blocker = make_req(rng, 100, 1, 'Q');
  uint64_t bid = 0;
  CHECK(s->submit(blocker.bp(), 0, &bid) == TSU_OK);
  std::vector<Req> rs;
  std::vector<uint64_t> ids;
  for (int i = 0; i < 5; ++i) rs.push_back(make_req(rng, i, 2));
  rs[2].p[1][0] = '!';  // poisoned pair
  rs[2].build();
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  CHECK(check_result(*s, bid, blocker, true) == TSU_OK);
  for (size_t i = 0; i < rs.size(); ++i) {
    tsu_request_info info{};
    const int rc = check_result(*s, ids[i], rs[i], true, 20000, &info);
    if (i == 2) {
      CHECK(rc == TSU_EINTERNAL);
    } else {
      CHECK(rc == TSU_OK);
    }
  }
  tsu_server_stats st{};
  s->stats(&st);
  CHECK(st.failed == 1);
}

void queue_full() {
  std::mt19937 rng(13);
  Config c;
  c.workers = 1;
  c.budget = 1 << 30;
  c.max_queue = 2;
  c.max_job_requests = 1;
  g_opts.delay_unit_us = 4000;  // 'Z' = 100 ms
  auto s = make_server(c);
  Req slow = make_req(rng, 0, 1, 'Z');
  uint64_t id = 0;
  CHECK(s->submit(slow.bp(), 0, &id) == TSU_OK);
  std::this_thread::sleep_for(std::chrono::milliseconds(20));  // running, off the queue
  Req a = make_req(rng, 1, 1), b = make_req(rng, 2, 1), d = make_req(rng, 3, 1);
  uint64_t i1 = 0, i2 = 0, i3 = 0;
  CHECK(s->submit(a.bp(), 0, &i1) == TSU_OK);
  CHECK(s->submit(b.bp(), 0, &i2) == TSU_OK);
  CHECK(s->submit(d.bp(), 0, &i3) == TSU_EBUSY);
  CHECK(check_result(*s, id, slow, true) == TSU_OK);
  CHECK(check_result(*s, i1, a, true) == TSU_OK);
  CHECK(check_result(*s, i2, b, true) == TSU_OK);
}

void stress() {
  // 8 client threads submitting and waiting at once
  Config c;
  c.workers = 4;
  c.budget = 200000;
  auto s = make_server(c);
  std::vector<std::thread> th;
  std::atomic<int> done{0};
  for (int t = 0; t < 8; ++t)
    th.emplace_back([&, t] {
      std::mt19937 rng(100 + t);
      for (int i = 0; i < 60; ++i) {
        Req r = make_req(rng, 1000 * t + i, 1 + (int)(rng() % 20), "ABC"[rng() % 3], 10 + (int)(rng() % 60));
        uint64_t id = 0;
        const uint32_t fl = rng() % 4 == 0 ? TSU_SCORE_ONLY : 0;
        CHECK(s->submit(r.bp(), fl, &id) == TSU_OK);
        if (rng() % 8 == 0) {
          s->cancel(id);
        } else {
          CHECK(check_result(*s, id, r, fl == 0) == TSU_OK);
        }
        ++done;
      }
    });
  for (auto& x : th) x.join();
  CHECK(done.load() == 480);
  CHECK(g_held_peak.load() <= (int64_t)c.budget);
}

void heavy_split() {
  // long pairs run as jobs of their own, at most heavy_workers at once; each
  // request's results come back in its own pair order
  std::mt19937 rng(15);
  g_opts.heavy_len = 100;
  Config c;
  c.workers = 5;
  c.heavy_workers = 2;
  c.heavy_len = 100;
  c.budget = 1 << 30;
  auto s = make_server(c);
  std::vector<Req> rs;
  std::vector<uint64_t> ids;
  for (int i = 0; i < 30; ++i) {
    std::vector<int> longs;
    const int n = 2 + (int)(rng() % 12);
    for (int k = 0; k < n; ++k)
      if (rng() % 4 == 0) longs.push_back(k);
    rs.push_back(make_mixed(rng, i, n, longs, 150 + (int)(rng() % 100), "BCD"[rng() % 3]));
  }
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  for (size_t i = 0; i < rs.size(); ++i) CHECK(check_result(*s, ids[i], rs[i], true) == TSU_OK);
  CHECK(g_heavy_peak.load() >= 1 && g_heavy_peak.load() <= 2);
  tsu_server_stats st{};
  s->stats(&st);
  CHECK(st.completed == 30 && st.failed == 0);
}

void heavy_fail() {
  // a failing long pair fails its request only; the request's other parts
  // are dropped or ignored
  std::mt19937 rng(16);
  g_opts.heavy_len = 100;
  Config c;
  c.workers = 3;
  c.heavy_len = 100;
  c.budget = 1 << 30;
  auto s = make_server(c);
  std::vector<Req> rs;
  for (int i = 0; i < 6; ++i) rs.push_back(make_mixed(rng, i, 6, {1, 4}, 200, 'C'));
  rs[3].p[4][0] = '!';
  rs[3].build();
  std::vector<uint64_t> ids;
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  for (size_t i = 0; i < rs.size(); ++i) CHECK(check_result(*s, ids[i], rs[i], true) == (i == 3 ? TSU_EINTERNAL : TSU_OK));
  tsu_server_stats st{};
  s->stats(&st);
  CHECK(st.failed == 1 && st.completed == 5);
}

void estimate() {
  // the k-mer edit-rate estimate that sizes long pairs' memory
  std::mt19937 rng(17);
  const double rates[] = {0.01, 0.05, 0.10, 0.15, 0.20};
  for (int L : {16384, 30000, 50000})
    for (double r : rates) {
      std::string p, t;
      for (int k = 0; k < L; ++k) p += "ACGT"[rng() % 4];
      // a third each of substitutions, insertions, deletions at random places
      for (int k = 0; k < L; ++k) {
        const double u = std::uniform_real_distribution<double>(0, 1)(rng);
        if (u < r / 3) {
          t += "ACGT"[(tsu::base2(p[k]) + 1 + rng() % 3) % 4];
        } else if (u < 2 * r / 3) {
          t += p[k];
          t += "ACGT"[rng() % 4];
        } else if (u < r) {
          // deleted
        } else {
          t += p[k];
        }
      }
      const double e = tsu::estimate_edit_rate(p.data(), (int32_t)p.size(), t.data(), (int32_t)t.size());
      if (std::fabs(e - r) > 0.02 + 0.1 * r)
        fail("estimate " + std::to_string(e) + " for rate " + std::to_string(r) + " at " + std::to_string(L));
    }
  // too short or not ACGT: no estimate
  CHECK(tsu::estimate_edit_rate("ACGT", 4, "ACGT", 4) < 0);
  std::string n(20000, 'N');
  CHECK(tsu::estimate_edit_rate(n.data(), 20000, n.data(), 20000) < 0);
}

void shutdown_busy() {
  std::mt19937 rng(14);
  Config c;
  c.workers = 1;
  c.budget = 1 << 30;
  c.max_job_requests = 1;
  auto s = make_server(c);
  std::vector<Req> rs;
  for (int i = 0; i < 5; ++i) rs.push_back(make_req(rng, i, 1, 'M'));
  std::vector<uint64_t> ids;
  for (auto& r : rs) {
    uint64_t id = 0;
    CHECK(s->submit(r.bp(), 0, &id) == TSU_OK);
    ids.push_back(id);
  }
  s->shutdown();  // queued ones dropped, the running one finishes
  uint64_t id = 0;
  CHECK(s->submit(rs[0].bp(), 0, &id) == TSU_EBUSY);
  int ok = 0, dropped = 0;
  for (auto x : ids) {
    const int rc = s->wait(x, 1000, nullptr, nullptr);
    ok += rc == TSU_OK || rc == TSU_EINVAL;  // EINVAL: done, no result buffer given
    dropped += rc == TSU_EBUSY;
  }
  CHECK(ok + dropped == 5 && dropped >= 1);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: sched_driver <scenario>\n");
    return 2;
  }
  const std::string sc = argv[1];
  struct {
    const char* name;
    void (*fn)();
  } table[] = {{"basic", basic},           {"score_only", score_only}, {"admission", admission},
               {"concurrency", concurrency}, {"reject", reject},       {"degraded", degraded},
               {"fifo", fifo},             {"cancel", cancel},         {"pending", pending},
               {"watchdog", watchdog},     {"nomem_retry", nomem_retry}, {"failure_isolation", failure_isolation},
               {"queue_full", queue_full}, {"stress", stress},         {"shutdown", shutdown_busy},
               {"heavy_split", heavy_split}, {"heavy_fail", heavy_fail}, {"estimate", estimate},
               {"lowmem", lowmem}};
  for (auto& e : table)
    if (sc == e.name) {
      e.fn();
      printf("ok %s\n", e.name);
      return 0;
    }
  fprintf(stderr, "unknown scenario %s\n", sc.c_str());
  return 2;
}
