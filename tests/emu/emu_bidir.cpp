// emu_bidir.cpp -- runs the BiWFA kernels (tsu_bidir.cuh, tsu_segment.cuh)
// through the CPU warp emulator.  Test infrastructure: compiled by
// tests/test_bidir_kernel.py with AddressSanitizer; every segment's crossing
// total, component, diagonal and cut are compared with the CPU oracle's
// two-ring search (ora_crossing_split), and every base-case segment's
// operations with the oracle's segment alignment (ora_align_segment).
//
// Input (stdin):  x o e gw N [step_cap], then N records
//                 "m n begin end\n<pattern>\n<text>\n" (each record is one
//                 pair; its segment is the whole pair, or with
//                 "S v0 h0 sm sn" after begin end, a sub-range)
// Output (stdout): gw 1, 4, 16 (breakpoint kernel): per segment
//                  "T comp k h" (T in penalty units, -1: none); gw 0 or -1
//                  (segment kernel with int16 or int32 history, one block
//                  of 4 warps, step_cap steps):
//                  per segment "status ops" (ops '-' when empty), then
//                  "retries K": segments that found the (deliberately
//                  small) run arena full and ran again
#include "warp_emu.h"
// clang-format off
#include "../../tsunami_pact_b200/csrc/tsu_kernels.cuh"
#include "../../tsunami_pact_b200/csrc/tsu_segment.cuh"
// clang-format on

#include <cstdio>
#include <iostream>
#include <string>

template <class T>
struct Buf {  // exact-size heap block
  T* p = nullptr;
  explicit Buf(size_t count) {
    p = count ? static_cast<T*>(std::malloc(sizeof(T) * count)) : nullptr;
    if (p) std::memset((void*)p, 0, sizeof(T) * count);
  }
  ~Buf() { std::free(p); }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
};

int main() {
  int X, O, E, GW;
  int64_t N;
  if (!(std::cin >> X >> O >> E >> GW >> N)) return 2;
  int step_cap = 0;
  if (GW <= 0 && !(std::cin >> step_cap)) return 2;
  const bool h32 = GW < 0;  // segment kernel with int32 history (gw -1)
  if (GW < 0) GW = 0;
  std::vector<std::string> pats(N), txts(N);
  std::vector<tsu::BidirSeg> segs(N);
  for (int64_t i = 0; i < N; ++i) {
    int m, n;
    char b, e;
    std::cin >> m >> n >> b >> e;
    tsu::BidirSeg sg{(int32_t)i, 0, 0, m, n, b, e};
    if (std::cin.peek() == ' ') {
      char S;
      std::cin >> S >> sg.v0 >> sg.h0 >> sg.m >> sg.n;
    }
    std::cin.get();
    pats[i].resize(m);
    std::cin.read(&pats[i][0], m);
    std::cin.get();
    txts[i].resize(n);
    std::cin.read(&txts[i][0], n);
    std::cin.get();
    segs[i] = sg;
  }
  int g = 1;
  const tsu::Pen rp = tsu::reduce_penalties(X, O, E, -1, 0, &g);
  // forward and reversed byte sequences, exact size
  int64_t ptot = 0, ttot = 0;
  for (auto& s : pats) ptot += (int64_t)s.size();
  for (auto& s : txts) ttot += (int64_t)s.size();
  Buf<uint8_t> pb(std::max<int64_t>(ptot, 1)), tb(std::max<int64_t>(ttot, 1));
  Buf<uint8_t> rpb(std::max<int64_t>(ptot, 1)), rtb(std::max<int64_t>(ttot, 1));
  Buf<int64_t> po(N), to(N);
  Buf<int32_t> pl(N), tl(N);
  int ring_w = 3;
  {
    int64_t a = 0, b = 0;
    for (int64_t i = 0; i < N; ++i) {
      const int m = (int)pats[i].size(), n = (int)txts[i].size();
      po.p[i] = a;
      pl.p[i] = m;
      to.p[i] = b;
      tl.p[i] = n;
      for (int j = 0; j < m; ++j) pb.p[a + j] = pats[i][j], rpb.p[a + j] = pats[i][m - 1 - j];
      for (int j = 0; j < n; ++j) tb.p[b + j] = txts[i][j], rtb.p[b + j] = txts[i][n - 1 - j];
      a += m;
      b += n;
      ring_w = std::max(ring_w, segs[i].m + segs[i].n + 3);
    }
  }
  tsu::SeqView sv{N, pb.p, po.p, pl.p, tb.p, to.p, tl.p};
  tsu::SeqView rsv{N, rpb.p, po.p, pl.p, rtb.p, to.p, tl.p};
  Buf<int64_t> wcnt(std::max<int64_t>(2 * N, 1)), woff(std::max<int64_t>(2 * N, 1));
  emu::launch(1, 64, 0, [&] { tsu::word_count_kernel(N, pl.p, tl.p, wcnt.p); });
  int64_t total = 0;
  for (int64_t j = 0; j < 2 * N; ++j) {
    woff.p[j] = total;
    total += wcnt.p[j];
  }
  Buf<uint64_t> words(std::max<int64_t>(total, 1)), rwords(std::max<int64_t>(total, 1));
  Buf<uint8_t> nonacgt(std::max<int64_t>(2 * N, 1)), rnonacgt(std::max<int64_t>(2 * N, 1));
  tsu::PackView pk{words.p, woff.p, nonacgt.p};
  tsu::PackView pkr{rwords.p, woff.p, rnonacgt.p};
  emu::launch(1, 64, 0, [&] { tsu::pack_kernel(sv, pk); });
  emu::launch(1, 64, 0, [&] { tsu::pack_kernel<true>(sv, pkr); });
  // the reversed packing equals packing the reversed bytes
  {
    Buf<uint64_t> chk(std::max<int64_t>(total, 1));
    Buf<uint8_t> chk_na(std::max<int64_t>(2 * N, 1));
    tsu::PackView pkc{chk.p, woff.p, chk_na.p};
    emu::launch(1, 64, 0, [&] { tsu::pack_kernel(rsv, pkc); });
    if (std::memcmp(chk.p, rwords.p, sizeof(uint64_t) * total)) {
      std::fprintf(stderr, "reversed packing differs\n");
      return 4;
    }
  }

  if (GW == 0) {
    // segment kernel: one block of kSegThreads, each warp with its own
    // history of exactly seg_hist_cap cells and step table
    const int warps = tsu::kSegThreads / 32;
    int32_t bases = 0;
    for (auto& sg : segs) bases = std::max(bases, sg.m + sg.n);
    const int64_t hcap = tsu::seg_hist_cap(step_cap, bases);
    const int64_t wcap = tsu::seg_run_cap(rp, bases, step_cap);
    Buf<char> hist((size_t)(warps * 3 * hcap) * (h32 ? 4 : 2));
    Buf<int32_t> table((size_t)warps * 9 * step_cap);
    Buf<uint32_t> wruns((size_t)(warps * wcap));
    // an arena too small for every segment's runs at once: some segments
    // report kPairArena (2) and run again with a larger one
    int64_t rtot = 0;
    for (int64_t i = 0; i < N; ++i) rtot += tsu::seg_run_cap(rp, (int64_t)segs[i].m + segs[i].n, step_cap);
    const int64_t small_cap = std::min<int64_t>(rtot, 24);
    Buf<uint32_t> runs(std::max<int64_t>(rtot, 1));
    Buf<int64_t> roff(N);
    Buf<int32_t> rlen(N), sst(N);
    Buf<unsigned> queue(1);
    Buf<unsigned long long> cursor(1);
    int64_t retries = 0;
    Buf<tsu::BidirSeg> dsegs(N);
    std::memcpy(dsegs.p, segs.data(), sizeof(tsu::BidirSeg) * N);
    tsu::SegArgs a{};
    a.seq = sv;
    a.pk = pk;
    a.pkr = pkr;
    a.segs = dsegs.p;
    a.n_segs = N;
    a.pen = rp;
    a.g = g;
    a.hist = hist.p;
    a.hist_cap = hcap;
    a.table = table.p;
    a.step_cap = step_cap;
    a.wruns = wruns.p;
    a.wruns_cap = wcap;
    a.runs = runs.p;
    a.runs_cap = small_cap;
    a.cursor = cursor.p;
    a.run_off = roff.p;
    a.run_len = rlen.p;
    a.status = sst.p;
    a.queue = queue.p;
    auto seg = [&](const tsu::SegArgs& x) {
      const size_t sm = tsu::seg_smem_bytes(rp);
      if (h32)
        emu::launch(1, tsu::kSegThreads, sm, [&] { tsu::segment_kernel<int32_t>(x); });
      else
        emu::launch(1, tsu::kSegThreads, sm, [&] { tsu::segment_kernel<int16_t>(x); });
    };
    seg(a);
    // the segments that found the arena full, again with room for all
    {
      std::vector<int64_t> again;
      for (int64_t i = 0; i < N; ++i)
        if (sst.p[i] == tsu::kPairArena) again.push_back(i);
      retries = (int64_t)again.size();
      if (!again.empty()) {
        Buf<tsu::BidirSeg> rsegs(again.size());
        for (size_t j = 0; j < again.size(); ++j) rsegs.p[j] = segs[(size_t)again[j]];
        Buf<int64_t> roff2(again.size());
        Buf<int32_t> rlen2(again.size()), sst2(again.size());
        queue.p[0] = 0;
        cursor.p[0] = std::min<unsigned long long>(cursor.p[0], (unsigned long long)small_cap);
        tsu::SegArgs b = a;
        b.segs = rsegs.p;
        b.n_segs = (int64_t)again.size();
        b.runs_cap = rtot;
        b.run_off = roff2.p;
        b.run_len = rlen2.p;
        b.status = sst2.p;
        seg(b);
        for (size_t j = 0; j < again.size(); ++j) {
          roff.p[again[j]] = roff2.p[j];
          rlen.p[again[j]] = rlen2.p[j];
          sst.p[again[j]] = sst2.p[j];
        }
      }
    }
    for (int64_t i = 0; i < N; ++i) {
      std::string ops;
      if (sst.p[i] == tsu::kPairOk) {
        for (int r = 0; r < rlen.p[i]; ++r) {
          const uint32_t u = runs.p[roff.p[i] + r];
          const uint32_t op = u & 15u;
          ops.append(u >> 4, op == tsu::kOpM ? 'M' : op == tsu::kOpX ? 'X' : op == tsu::kOpI ? 'I' : 'D');
        }
      }
      std::printf("%d %s\n", sst.p[i], ops.empty() ? "-" : ops.c_str());
    }
    std::printf("retries %lld\n", (long long)retries);
    return 0;
  }
  const int threads = GW <= 4 ? 128 : 32 * GW;
  const int groups = threads / (32 * GW);
  const int64_t ring_stride = (int64_t)2 * rp.rm * 4 * ring_w;  // elements (int16 below 16 warps)
  Buf<char> ring((size_t)groups * ring_stride * tsu::bidir_ring_bytes(GW));
  Buf<int32_t> oT(N), oc(N), ok(N), oh(N), ost(N);
  Buf<unsigned> queue(2);
  Buf<unsigned long long> work(2);
  Buf<tsu::BidirSeg> dsegs(N);
  std::memcpy(dsegs.p, segs.data(), sizeof(tsu::BidirSeg) * N);
  tsu::BidirArgs a{};
  a.seq = sv;
  a.pk = pk;
  a.pkr = pkr;
  a.segs = dsegs.p;
  a.n_segs = N;
  a.pen = rp;
  a.ring_w = ring_w;
  a.ring = ring.p;
  a.ring_stride = ring_stride;
  a.out_T = oT.p;
  a.out_comp = oc.p;
  a.out_k = ok.p;
  a.out_h = oh.p;
  a.status = ost.p;
  a.queue = queue.p;
  a.work = work.p;
  const size_t smem = (size_t)groups * tsu::bidir_group_smem(rp, GW);
  switch (GW) {
    case 1: emu::launch(1, threads, smem, [&] { tsu::bidir_kernel<1>(a); }); break;
    case 4: emu::launch(1, threads, smem, [&] { tsu::bidir_kernel<4>(a); }); break;
    case 16: emu::launch(1, threads, smem, [&] { tsu::bidir_kernel<16>(a); }); break;
    default: return 3;
  }
  for (int64_t i = 0; i < N; ++i)
    std::printf("%d %c %d %d\n", oT.p[i] < 0 ? -1 : oT.p[i] * g, (char)oc.p[i], ok.p[i], oh.p[i]);
  return 0;
}
