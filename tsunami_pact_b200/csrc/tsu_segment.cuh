// tsu_segment.cuh -- the base case of bidirectional WFA on the GPU: one
// small segment aligned by the forward WFA with its begin and end
// components, every wavefront kept, and its CIGAR runs by backtrace.
//
// A segment (BidirSeg) that must end in M runs forward on the sequences,
// starting in its begin component (offset 0 in I or D at score 0).  One that
// must end in a gap runs on the reversed sequences instead, forced to open
// that gap first (a seed at score o + e), free to end in its begin gap at a
// discount of o, and its operations come out in reverse.  The wavefronts
// are the breakpoint kernel's (tsu_bidir.cuh: out-of-bounds cells null in
// every component, M kept before and after extension).  The end is the
// lowest score whose M reaches offset n on diagonal n - m, or whose free end
// gap does (cost s - o); the search stops once no later score can be lower.
// The backtrace recomputes each cell's source from the kept wavefronts and
// takes the largest (offset, code), the codes in the order of the
// reference's bt_type_t (common.h:67-77): mismatch 9 > D extend 6 > D open 5
// > I extend 2 > I open 1; the forced first gap opens from the empty origin.
//
// One warp per segment, persistent over a work queue.  Per warp in device
// memory: the history (hist_cap cells of 3 int32: M, I, D; the backtrace
// never reads M before extension, so it is not kept) and the step table
// (step_cap rows: lo, hi, first history cell, and the first / last present
// diagonal of M, I, D).  A segment that needs more
// steps or cells than the launch gives gets status kPairScratch and runs
// again in a launch with more.  The backtrace writes its runs (length << 4 |
// kOp*; at most seg_run_cap of them) into the warp's own area, then the warp
// takes their exact count from the run arena (an atomic cursor) and copies
// them there; a segment that finds the arena full gets status kPairArena.
#pragma once

#include "tsu_bidir.cuh"

namespace tsu {

// HT: the history's element type -- int16 when every segment of the launch
// has both sides below 32,767 (offsets fit; half the history traffic),
// int32 otherwise.  Negative stored values are absent cells.
template <typename HT>
__global__ void __launch_bounds__(kSegThreads, 6) segment_kernel(SegArgs a) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int hM = 0, hI = 1, hD = 2;  // components of a history cell
  constexpr HT kHNull = (HT)(sizeof(HT) == 2 ? -16384 : kBNull);
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const Pen pen = a.pen;
  const int x = pen.x, go = pen.go, ge = pen.ge, oo = pen.go - pen.ge;
  HT* const hist = static_cast<HT*>(a.hist) + gwarp * a.hist_cap * 3;
  int32_t* const tab = a.table + gwarp * (int64_t)a.step_cap * 9;
  // the last rm rows of the step table in shared memory, slot s mod rm (the
  // steps read them; the backtrace reads the table in device memory)
#ifdef TSU_WARP_EMU
  int* const rt = reinterpret_cast<int*>(emu::dyn_smem()) + (threadIdx.x >> 5) * pen.rm * 9;
#else
  extern __shared__ int seg_smem[];
  int* const rt = seg_smem + (threadIdx.x >> 5) * pen.rm * 9;
#endif
  const int rm = pen.rm;
  auto slot_back = [&](int sl, int b) -> int { return sl - b + (sl < b ? rm : 0); };  // slot b steps before (b < rm)
  for (;;) {
    unsigned q = 0;
    if (lane == 0) q = atomicAdd(a.queue, 1u);
    q = __shfl_sync(FULL, q, 0);
    if ((int64_t)q >= a.n_segs) break;
    const BidirSeg sg = a.segs[q];
    const int m = sg.m, n = sg.n, k_end = n - m;
    const int64_t pair = sg.pair;
    const bool bytes = a.pk.nonacgt[pair] | a.pk.nonacgt[a.seq.n + pair];
    const bool fwd = sg.end == 'M';
    const int start = fwd ? sg.begin : 'M';
    const int forced = fwd ? 'M' : sg.end;
    const int free_end = fwd ? 'M' : sg.begin;
    const int M_full = a.seq.pat_len[pair], N_full = a.seq.txt_len[pair];
    const PackView& pw = fwd ? a.pk : a.pkr;
    const uint32_t* pwp = reinterpret_cast<const uint32_t*>(pw.words + pw.woff[pair]);
    const uint32_t* twp = reinterpret_cast<const uint32_t*>(pw.words + pw.woff[a.seq.n + pair]);
    const uint8_t* pb = a.seq.pat + a.seq.pat_off[pair];
    const uint8_t* tb = a.seq.txt + a.seq.txt_off[pair];
    // position of the (possibly reversed) segment's base 0: packed forward
    // (v0, h0) or reversed (M - v0 - m, N - h0 - n); bytes forward (v0, h0)
    // or, read backwards, the segment's last bases (v0 + m - 1, h0 + n - 1)
    const int pv0 = fwd ? sg.v0 : (bytes ? sg.v0 + m - 1 : M_full - sg.v0 - m);
    const int ph0 = fwd ? sg.h0 : (bytes ? sg.h0 + n - 1 : N_full - sg.h0 - n);
    const bool back = !fwd && bytes;
    auto lcp = [&](int v, int h, int rem) -> int {
      if (rem <= 0) return 0;
      return bidir_lcp(bytes, !back, pwp, twp, pb, tb, back ? pv0 - v : pv0 + v, back ? ph0 - h : ph0 + h, rem);
    };
    auto inb = [&](int32_t off, int k) -> bool {
      return ((uint32_t)off <= (uint32_t)n) & ((uint32_t)(off - k) <= (uint32_t)m);
    };
    auto get = [&](int s, int c, int k) -> int32_t {
      if (s < 0) return kBNull;
      const int32_t* t = tab + (int64_t)s * 9;
      if (k < t[0] || k > t[1]) return kBNull;
      const int32_t v = hist[((int64_t)t[2] + (k - t[0])) * 3 + c];
      return v < 0 ? kBNull : v;
    };
    int st = kPairOk;
    int64_t used = 0;  // history cells in use
    int have = 0, best = 0, s_end = 0, state = 'M';
    int n_steps = 0;
    const int64_t smax = (int64_t)(m + n) * (pen.rm - 1) + 2 * go;
    for (int s = 0, sl = 0; s <= smax; ++s, sl = sl + 1 == rm ? 0 : sl + 1) {
      if (have && s - (free_end != 'M' ? oo : 0) > best) break;
      if (s >= a.step_cap) {
        st = kPairScratch;
        break;
      }
      const bool seed_i = forced == 'I' && s == go && inb(1, 1);
      const bool seed_d = forced == 'D' && s == go && inb(0, -1);
      int lo, hi;
      if (s == 0) {
        lo = forced == 'M' ? 0 : 1;
        hi = 0;
      } else {
        lo = INT_MAX, hi = INT_MIN;
        auto widen = [&](int b, int c) {  // present range of component c, b steps back
          if (s < b) return;
          const int* u = rt + slot_back(sl, b) * 9 + 3 + 2 * c;
          if (u[0] > u[1]) return;
          lo = min(lo, u[0] - 1);
          hi = max(hi, u[1] + 1);
        };
        widen(x, 0);
        widen(go, 0);
        widen(ge, 1);
        widen(ge, 2);
        if (seed_i) lo = min(lo, 1), hi = max(hi, 1);
        if (seed_d) lo = min(lo, -1), hi = max(hi, -1);
        if (lo > hi) lo = 1, hi = 0;
      }
      const int width = hi - lo + 1;  // 0 when empty
      if (used + width > a.hist_cap) {
        st = kPairScratch;
        break;
      }
      HT* row = hist + used * 3;
      int pm0 = INT_MAX, pm1 = INT_MIN, pi0 = INT_MAX, pi1 = INT_MIN, pd0 = INT_MAX, pd1 = INT_MIN;
      // the source rows (s - x, s - o - e, s - e), resolved once per step
      struct Row {
        const HT* base;  // cell of diagonal k at base + 3 (k - lo)
        int lo, hi;
      };
      auto row_of = [&](int b) -> Row {  // b steps back
        if (s < b || s == 0) return Row{hist, 1, 0};
        const int* t = rt + slot_back(sl, b) * 9;
        return Row{hist + (int64_t)t[2] * 3, t[0], t[1]};
      };
      const Row RX = row_of(x), RG = row_of(go), RE = row_of(ge);
      int32_t eM = kBNull, eI = kBNull, eD = kBNull;  // this step's cells on the end diagonal
      auto rd = [&](const Row& R, int c, int k) -> int32_t {
        if (k < R.lo || k > R.hi) return kBNull;
        const int32_t v = R.base[(int64_t)(k - R.lo) * 3 + c];
        return v < 0 ? kBNull : v;
      };
      for (int k = lo + lane; k <= hi; k += 32) {
        int32_t cm = kBNull, ci = kBNull, cd = kBNull;
        if (s == 0) {
          cm = lcp(0, 0, min(m, n));
          ci = start == 'I' ? 0 : kBNull;
          cd = start == 'D' ? 0 : kBNull;
        } else {
          int32_t ins = max(rd(RG, hM, k - 1), rd(RE, hI, k - 1)) + 1;
          if (seed_i && k == 1) ins = max(ins, 1);
          int32_t del = max(rd(RG, hM, k + 1), rd(RE, hD, k + 1));
          if (seed_d && k == -1) del = max(del, 0);
          const int32_t mis = rd(RX, hM, k) + 1;
          if (inb(ins, k)) ci = ins;
          if (inb(del, k)) cd = del;
          const int32_t pv = max(mis, max(ins, del));
          if (inb(pv, k)) {
            const int vv = pv - k;
            cm = pv + lcp(vv, pv, min(m - vv, n - pv));
          }
        }
        HT* cell = row + (int64_t)(k - lo) * 3;
        cell[hM] = cm < 0 ? kHNull : (HT)cm;
        cell[hI] = ci < 0 ? kHNull : (HT)ci;
        cell[hD] = cd < 0 ? kHNull : (HT)cd;
        if (k == k_end) eM = cm, eI = ci, eD = cd;
        if (cm != kBNull) pm0 = min(pm0, k), pm1 = k;
        if (ci != kBNull) pi0 = min(pi0, k), pi1 = k;
        if (cd != kBNull) pd0 = min(pd0, k), pd1 = k;
      }
      pm0 = __reduce_min_sync(FULL, pm0);
      pm1 = __reduce_max_sync(FULL, pm1);
      pi0 = __reduce_min_sync(FULL, pi0);
      pi1 = __reduce_max_sync(FULL, pi1);
      pd0 = __reduce_min_sync(FULL, pd0);
      pd1 = __reduce_max_sync(FULL, pd1);
      eM = __reduce_max_sync(FULL, eM);
      eI = __reduce_max_sync(FULL, eI);
      eD = __reduce_max_sync(FULL, eD);
      if (lane == 0) {
        const int32_t row9[9] = {lo, hi, (int32_t)used, pm0 <= pm1 ? pm0 : 1, pm0 <= pm1 ? pm1 : 0,
                                 pi0 <= pi1 ? pi0 : 1, pi0 <= pi1 ? pi1 : 0, pd0 <= pd1 ? pd0 : 1,
                                 pd0 <= pd1 ? pd1 : 0};
        int32_t* t = tab + (int64_t)s * 9;
        int* r = rt + sl * 9;
        for (int i = 0; i < 9; ++i) t[i] = row9[i], r[i] = row9[i];
      }
      __syncwarp();
      used += width;
      ++n_steps;
      if (eM >= n && (!have || s < best)) have = 1, best = s, s_end = s, state = 'M';
      if (free_end == 'I' || free_end == 'D') {
        const int32_t gv = free_end == 'I' ? eI : eD;
        if (gv == n && (!have || s - oo < best)) have = 1, best = s - oo, s_end = s, state = free_end;
      }
    }
    if (st == kPairOk && !have) st = kPairInternal;
    int64_t nr = 0;                // runs of the backtrace
    const int64_t cap = min(seg_run_cap(pen, (int64_t)m + n, a.step_cap), a.wruns_cap);
    uint32_t* const out = a.wruns + gwarp * a.wruns_cap;
    if (lane == 0 && st == kPairOk) {
      // backtrace from the end; runs written backwards from the area's
      // end (forward pass: the segment's last operation comes first), or
      // forwards from its start (reversed pass: its first comes first)
      uint32_t cop = 0;
      int64_t clen = 0;
      bool bad = false;
      auto flush = [&]() {
        if (clen == 0) return;
        if (nr >= cap || clen >= (1 << 28)) {
          bad = true;
          return;
        }
        out[fwd ? cap - 1 - nr : nr] = (uint32_t)clen << 4 | cop;
        ++nr;
        clen = 0;
      };
      auto put = [&](uint32_t op, int64_t cnt) {
        if (cnt <= 0) return;
        if (op != cop) flush(), cop = op;
        clen += cnt;
      };
      auto bsrc = [&](int ss, int c, int k, int delta, int code) -> long long {
        const int32_t v = get(ss, c, k);
        if (v == kBNull) return LLONG_MIN / 4;
        return (long long)(v + delta) * 16 + code;
      };
      int s2 = s_end, k = k_end;
      int32_t off = get(s_end, state == 'M' ? hM : (state == 'I' ? hI : hD), k_end);
      int v = off - k, h = off;
      while (v > 0 && h > 0 && s2 > 0) {
        long long io = bsrc(s2 - go, hM, k - 1, 1, 1);
        const long long ix = bsrc(s2 - ge, hI, k - 1, 1, 2);
        long long dop = bsrc(s2 - go, hM, k + 1, 0, 5);
        const long long dx = bsrc(s2 - ge, hD, k + 1, 0, 6);
        if (forced == 'I' && s2 == go && k == 1) io = max(io, 1ll * 16 + 1);
        if (forced == 'D' && s2 == go && k == -1) dop = max(dop, 0ll * 16 + 5);
        long long b;
        if (state == 'M')
          b = max(bsrc(s2 - x, hM, k, 1, 9), max(max(io, ix), max(dop, dx)));
        else if (state == 'I')
          b = max(io, ix);
        else
          b = max(dop, dx);
        if (b < 0) {
          bad = true;
          break;
        }
        if (state == 'M') {
          const int32_t moff = (int32_t)(b / 16);
          put(kOpM, off - moff);
          off = moff;
          v = off - k;
          h = off;
          if (v <= 0 || h <= 0) break;
        }
        switch ((int)(b % 16)) {
          case 9: s2 -= x; state = 'M'; put(kOpX, 1); off--; break;
          case 1: s2 -= go; state = 'M'; put(kOpI, 1); k--; off--; break;
          case 2: s2 -= ge; state = 'I'; put(kOpI, 1); k--; off--; break;
          case 5: s2 -= go; state = 'M'; put(kOpD, 1); k++; break;
          default: s2 -= ge; state = 'D'; put(kOpD, 1); k++; break;
        }
        v = off - k;
        h = off;
      }
      if (!bad && v > 0 && h > 0) {
        const int nm = v < h ? v : h;
        put(kOpM, nm);
        v -= nm;
        h -= nm;
      }
      if (!bad) put(kOpD, v);
      if (!bad) put(kOpI, h);
      if (!bad) flush();
      if (bad) st = kPairInternal;
    }
    st = __shfl_sync(FULL, st, 0);
    nr = __shfl_sync(FULL, nr, 0);
    if (st == kPairOk) {
      // the runs' place in the arena, then a warp-wide copy
      unsigned long long pos = 0;
      if (lane == 0) pos = atomicAdd(a.cursor, (unsigned long long)nr);
      pos = __shfl_sync(FULL, pos, 0);
      if ((int64_t)pos + nr > a.runs_cap) {
        st = kPairArena;
      } else {
        const uint32_t* src = fwd ? out + cap - nr : out;
        for (int64_t i = lane; i < nr; i += 32) a.runs[pos + i] = src[i];
        if (lane == 0) {
          a.run_off[q] = (int64_t)pos;
          a.run_len[q] = (int32_t)nr;
          if (a.pair_score) a.pair_score[pair] = best * a.g;
        }
      }
    }
    if (lane == 0) {
      a.status[q] = st;
      if (a.work) {
        atomicAdd(a.work, (unsigned long long)used);
        atomicAdd(a.work + 1, (unsigned long long)n_steps);
      }
    }
    __syncwarp();
  }
}

// Runs of each pair from its leaves, in alignment order: the one leaf of the
// whole-pair launch when pre_st[i] is OK (at pre_off[i], pre_len[i] runs),
// else the recursion's leaves first[i] .. first[i + 1] (at run_off[j],
// run_len[j]); runs of the same operation that meet at a cut merge.
// count: out_len[i] = the pair's run count (0 unless status[i] is OK);
// write: the runs at out[out_off[i]...].  One thread per pair.
template <bool kWrite>
__global__ void seg_runs_kernel(int64_t n, const int32_t* __restrict__ pre_st, const int64_t* __restrict__ pre_off,
                                const int32_t* __restrict__ pre_len, const int64_t* __restrict__ first,
                                const int64_t* __restrict__ run_off, const int32_t* __restrict__ run_len,
                                const uint32_t* __restrict__ runs, const int32_t* __restrict__ status,
                                int64_t* __restrict__ out_len, const int64_t* __restrict__ out_off,
                                uint32_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (status[i] != kPairOk) {
      if (!kWrite) out_len[i] = 0;
      continue;
    }
    int64_t cnt = 0, w = kWrite ? out_off[i] : 0;
    uint32_t cur = 0;
    bool open = false;
    auto leaf = [&](const uint32_t* r, int len) {
      for (int t = 0; t < len; ++t) {
        const uint32_t u = r[t];
        if (open && (u & 15u) == (cur & 15u)) {
          cur += u & ~15u;
        } else {
          if (kWrite && open) out[w++] = cur;
          cur = u;
          open = true;
          ++cnt;
        }
      }
    };
    if (pre_st[i] == kPairOk)
      leaf(runs + pre_off[i], pre_len[i]);
    else
      for (int64_t j = first[i]; j < first[i + 1]; ++j) leaf(runs + run_off[j], run_len[j]);
    if (kWrite) {
      if (open) out[w] = cur;
    } else {
      out_len[i] = cnt;
    }
  }
}

// Whole pairs as segments, free at both ends.
__global__ void whole_pairs_kernel(int64_t n, const int32_t* __restrict__ plen, const int32_t* __restrict__ tlen,
                                   BidirSeg* __restrict__ segs) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    segs[i] = BidirSeg{(int32_t)i, 0, 0, plen[i], tlen[i], 'M', 'M'};
}

}  // namespace tsu
