// emu_driver.cpp -- host-side replica of the engine's batch flow
// (tsu_engine.cu run_device) driving the real kernels through the CPU warp
// emulator.  Test infrastructure: compiled by tests/test_kernel_emu.py with
// AddressSanitizer, it checks the kernels' indexing and outputs on the CPU.
//
// Input (stdin):  x o e o2 e2 pbf pef tbf tef lowmem cigar hint first_mode first_gw N
//                 then N records "m n\n<pattern>\n<text>\n"
//   o2 < 0: one gap piece; else dual gap-affine (the kModelDual kernels);
//   o < 0: gap-linear with mismatch x and gap e per base (kModelLinear);
//   pbf pef tbf tef: free ends (all 0: end-to-end); lowmem: checkpoint
//   interval of the low-memory mode (0 off, < 0 chosen by the planner)
//   first_mode 1 = shared ring, 0 = global ring; first_gw = warps per pair
//   of the first pass (1, 2, 4, 8, 16).  Retry passes follow the engine's
//   ladder (tsu_plan.h next_pass).
// Output (stdout): per pair "score<TAB>ops" (ops = WFA2 operation string),
//                 then a line "passes <k> retried <r> gws <g1,g2,...>".
#include "warp_emu.h"
// clang-format off
#include "../../tsunami_pact_b200/csrc/tsu_kernels.cuh"
#include "../../tsunami_pact_b200/csrc/tsu_plan.h"
// clang-format on

#include <cstdio>
#include <iostream>
#include <numeric>
#include <string>

template <class T>
struct Buf {  // exact-size heap block
  T* p = nullptr;
  size_t n = 0;
  explicit Buf(size_t count = 0) { resize(count); }
  void resize(size_t count) {
    std::free(p);
    n = count;
    p = count ? static_cast<T*>(std::malloc(sizeof(T) * count)) : nullptr;
    if (p) std::memset((void*)p, 0, sizeof(T) * count);
  }
  ~Buf() { std::free(p); }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
};

// The align passes of each penalty model (emu_model.cpp, compiled once per
// model).
void run_pass_affine(bool cigar, int mode, int gw, int threads, size_t smem, const tsu::AlignArgs& a, bool lowmem);
void run_pass_dual(bool cigar, int mode, int gw, int threads, size_t smem, const tsu::AlignArgs& a, bool lowmem);
void run_pass_linear(bool cigar, int mode, int gw, int threads, size_t smem, const tsu::AlignArgs& a, bool lowmem);

int main() {
  int X, O, E, O2, E2, PBF, PEF, TBF, TEF, LOWMEM, cigar, first_mode, first_gw;
  double hint;
  int64_t N;
  if (!(std::cin >> X >> O >> E >> O2 >> E2 >> PBF >> PEF >> TBF >> TEF >> LOWMEM >> cigar >> hint >> first_mode >>
        first_gw >> N))
    return 2;
  std::vector<std::string> pats(N), txts(N);
  for (int64_t i = 0; i < N; ++i) {
    int m, n;
    std::cin >> m >> n;
    std::cin.get();
    pats[i].resize(m);
    std::cin.read(&pats[i][0], m);
    std::cin.get();
    txts[i].resize(n);
    std::cin.read(&txts[i][0], n);
    std::cin.get();
  }
  int g = 1;
  const tsu::Pen rp = O < 0 ? tsu::reduce_linear(X, E, &g) : tsu::reduce_penalties(X, O, E, O2, E2, &g);
  const int smem_optin = 232448;
  // sequences: exact-size buffers (pattern i, text i concatenated)
  int64_t ptot = 0, ttot = 0;
  for (auto& s : pats) ptot += (int64_t)s.size();
  for (auto& s : txts) ttot += (int64_t)s.size();
  Buf<uint8_t> pb(std::max<int64_t>(ptot, 1)), tb(std::max<int64_t>(ttot, 1));
  Buf<int64_t> po(N), to(N);
  Buf<int32_t> pl(N), tl(N);
  int32_t max_m = 0, max_n = 0;
  {
    int64_t a = 0, b = 0;
    for (int64_t i = 0; i < N; ++i) {
      po.p[i] = a;
      pl.p[i] = (int32_t)pats[i].size();
      std::memcpy(pb.p + a, pats[i].data(), pats[i].size());
      a += pats[i].size();
      to.p[i] = b;
      tl.p[i] = (int32_t)txts[i].size();
      std::memcpy(tb.p + b, txts[i].data(), txts[i].size());
      b += txts[i].size();
      max_m = std::max(max_m, pl.p[i]);
      max_n = std::max(max_n, tl.p[i]);
    }
  }
  tsu::SeqView sv{N, pb.p, po.p, pl.p, tb.p, to.p, tl.p};
  // word counts + exclusive scan (the engine does this with CUB)
  Buf<int64_t> wcnt(std::max<int64_t>(2 * N, 1)), woff(std::max<int64_t>(2 * N, 1));
  emu::launch(1, 64, 0, [&] { tsu::word_count_kernel(N, pl.p, tl.p, wcnt.p); });
  int64_t total = 0;
  for (int64_t j = 0; j < 2 * N; ++j) {
    woff.p[j] = total;
    total += wcnt.p[j];
  }
  Buf<uint64_t> words(std::max<int64_t>(total, 1));
  Buf<uint8_t> nonacgt(std::max<int64_t>(2 * N, 1));
  tsu::PackView pk{words.p, woff.p, nonacgt.p};
  emu::launch(1, 64, 0, [&] { tsu::pack_kernel(sv, pk); });

  Buf<int32_t> score(std::max<int64_t>(N, 1)), status(std::max<int64_t>(N, 1));
  Buf<int64_t> cpos(std::max<int64_t>(N, 1));
  Buf<int32_t> clen(std::max<int64_t>(N, 1)), retry(std::max<int64_t>(N, 1)), order(std::max<int64_t>(N, 1));
  Buf<unsigned long long> counters(8);  // [0]: queue (u32) + retry count (u32), [2]: cursor, [3..4]: work
  int64_t arena_cap = tsu::arena_runs(rp, N, max_m, max_n, hint);
  Buf<uint32_t> arena(arena_cap);
  const bool want_cigar = cigar != 0;
  int64_t n_order = N;
  const int32_t* ord = nullptr;
  int passes = 0;
  int64_t retried = 0;
  double h = hint;
  unsigned* queue = reinterpret_cast<unsigned*>(counters.p);
  unsigned* retry_cnt = queue + 1;
  unsigned long long* cursor = counters.p + 2;
  tsu::PassChoice pc{first_mode ? tsu::kModeShared : tsu::kModeGlobal, first_gw};
  int32_t pm = max_m, pn = max_n;
  std::string gws;
  for (;;) {
    const tsu::PassGeom geo = tsu::plan_geometry(rp, pm, pn, pc.mode, pc.gw, h, want_cigar, smem_optin, LOWMEM);
    const int groups = geo.groups_per_cta;  // one block
    Buf<int32_t> ring(geo.mode == tsu::kModeGlobal ? (size_t)groups * geo.ring_ints : 0);
    Buf<uint32_t> hist(want_cigar ? (size_t)groups * geo.hist_cap : 0);
    Buf<int2> table(want_cigar ? (size_t)groups * geo.table_cap : 0);
    Buf<uint8_t> ckpt(geo.ckpt_k > 0 ? (size_t)groups * geo.ckpt_cap * geo.ckpt_bytes : 0);
    tsu::AlignArgs a{};
    a.seq = sv;
    a.pk = pk;
    a.order = ord;
    a.n_order = n_order;
    a.pen = rp;
    a.g = g;
    a.ring_w = geo.ring_w;
    a.seq_cap = geo.seq_cap;
    a.ring_global = ring.p;
    a.ring_stride = geo.ring_ints;
    a.hist = hist.p;
    a.hist_cap = geo.hist_cap;
    a.table = table.p;
    a.table_cap = geo.table_cap;
    a.score = score.p;
    a.status = status.p;
    a.arena = arena.p;
    a.arena_cursor = cursor;
    a.arena_cap = arena_cap;
    a.cig_pos = cpos.p;
    a.cig_len = clen.p;
    a.queue = queue;
    a.retry = retry.p;
    a.retry_count = retry_cnt;
    a.work = counters.p + 3;
    a.ef_pb = PBF;
    a.ef_pe = PEF;
    a.ef_tb = TBF;
    a.ef_te = TEF;
    a.ckpt = ckpt.p;
    a.ckpt_k = geo.ckpt_k;
    a.ckpt_cap = geo.ckpt_cap;
    a.ckpt_bytes = (int32_t)geo.ckpt_bytes;
    a.ckpt_stride = (int64_t)geo.ckpt_cap * geo.ckpt_bytes;
    const size_t smem = (size_t)groups * geo.group_smem;
    const int threads = geo.cta_threads;
    gws += (gws.empty() ? "" : ",") + std::string(geo.mode == tsu::kModeShared ? "s" : "g") + std::to_string(geo.gw);
    const bool lowmem = geo.ckpt_k > 0;
    if (rp.linear())
      run_pass_linear(want_cigar, geo.mode, geo.gw, threads, smem, a, lowmem);
    else if (rp.dual())
      run_pass_dual(want_cigar, geo.mode, geo.gw, threads, smem, a, lowmem);
    else
      run_pass_affine(want_cigar, geo.mode, geo.gw, threads, smem, a, lowmem);
    ++passes;
    const unsigned nretry = *retry_cnt;
    if (nretry == 0) break;
    retried += nretry;
    if (passes > 16) {
      std::fprintf(stderr, "pairs still fail after %d passes\n", passes);
      return 3;
    }
    if (geo.mode == tsu::kModeGlobal && h >= tsu::kHintCeiling) {
      std::fprintf(stderr, "pairs exceed the scratch ceiling\n");
      return 3;
    }
    std::vector<int32_t> rl(retry.p, retry.p + nretry);
    pm = pn = 0;
    for (int32_t i : rl) {
      pm = std::max(pm, pl.p[i]);
      pn = std::max(pn, tl.p[i]);
    }
    std::sort(rl.begin(), rl.end(), [&](int32_t u, int32_t v) { return pl.p[u] + tl.p[u] > pl.p[v] + tl.p[v]; });
    std::memcpy(order.p, rl.data(), sizeof(int32_t) * nretry);
    ord = order.p;
    n_order = nretry;
    h = tsu::next_hint(h, geo.mode == tsu::kModeGlobal);
    // the ladder's global step at 8 warps: emulating 16-warp groups (one
    // host thread per lane) is slow; the 16-warp global kernel has its own
    // test (test_warp_groups)
    pc = tsu::next_pass(pc, rp, pm, pn, smem_optin, 8);
    if (want_cigar) {
      const unsigned long long used = *cursor;
      const int64_t maxlen = std::max(pm, pn);
      const int64_t need =
          (int64_t)used + (int64_t)nretry * (2 * tsu::hint_score(rp, maxlen, h) / rp.min_pen() + 1);
      if (need > arena_cap) {
        Buf<uint32_t> nb(need);
        std::memcpy(nb.p, arena.p, sizeof(uint32_t) * (size_t)std::min<int64_t>((int64_t)used, arena_cap));
        std::swap(arena.p, nb.p);
        std::swap(arena.n, nb.n);
        arena_cap = need;
      }
    }
    queue[0] = 0;
    queue[1] = 0;
  }
  for (int64_t i = 0; i < N; ++i) {
    if (status.p[i] != tsu::kPairOk) {
      std::fprintf(stderr, "pair %lld status %d\n", (long long)i, status.p[i]);
      return 4;
    }
  }
  // compaction: lengths -> scan -> compact_kernel
  Buf<int64_t> len64(N + 1), off(N + 1);
  emu::launch(1, 64, 0, [&] { tsu::cig_len64_kernel(N, clen.p, status.p, len64.p); });
  len64.p[N] = 0;
  int64_t acc = 0;
  for (int64_t i = 0; i <= N; ++i) {
    off.p[i] = acc;
    acc += len64.p[i];
  }
  Buf<uint32_t> out(std::max<int64_t>(acc, 1));
  if (want_cigar) emu::launch(1, 64, 0, [&] { tsu::compact_kernel(N, arena.p, cpos.p, off.p, out.p); });
  static const char code2c[16] = {'M', 'I', 'D', '?', '?', '?', '?', '?', 'X', '?', '?', '?', '?', '?', '?', '?'};
  std::string line;
  for (int64_t i = 0; i < N; ++i) {
    line = std::to_string(score.p[i]);
    line += '\t';
    if (want_cigar)
      for (int64_t r = off.p[i]; r < off.p[i + 1]; ++r) line.append(out.p[r] >> 4, code2c[out.p[r] & 15]);
    line += '\n';
    std::fwrite(line.data(), 1, line.size(), stdout);
  }
  std::printf("passes %d retried %lld gws %s\n", passes, (long long)retried, gws.c_str());
  return 0;
}
