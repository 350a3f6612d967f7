// tsu_bidir.cuh -- the breakpoint search of bidirectional WFA (BiWFA) on the
// GPU: forward and reverse wavefronts of a segment, two rings, in turns.
//
// A segment is a pattern range [v0, v0 + m) and a text range [h0, h0 + n) of
// one pair, with a begin component (the forward pass starts in M, or inside
// an I or D gap continued from the left: offset 0 in that component at score
// 0) and an end component (the reverse pass, on the reversed sequences, is
// forced to open that gap first: a seed at score o + e).  Wavefronts follow
// the segment semantics of the CPU BiWFA model (out-of-bounds cells are null
// in every component; offset = text position h on diagonal k = h - v, the
// recurrences of the reference kernel, wfa_gpu.cu:616-626):
//   I[s][k]  = max(M[s-o-e][k-1], I[s-e][k-1]) + 1
//   D[s][k]  = max(M[s-o-e][k+1], D[s-e][k+1])
//   M'[s][k] = max(M[s-x][k] + 1, I[s][k], D[s][k])   (pre-extension, kept)
//   M[s][k]  = M'[s][k] extended along the diagonal
// each kept only in bounds.  A pass's wavefront at score s spans the
// present cells of its sources widened by one diagonal on each side.
//
// Search (the two-ring rule): forward and reverse advance in turns, the
// lower score first (forward on ties); each new wavefront is checked against
// the other side's last max(x, o+e) + 1 scores -- the ring depth -- for a
// diagonal where forward and reverse offsets cross (forward + reverse >= n;
// M, I, D in turn, forward diagonals ascending; a gap crossing counts its
// opening once).  The strictly lowest total is kept, the first found among
// equals; the search stops when no later crossing can be lower.  An M
// crossing is cut at max(forward pre-extension offset, n - reverse offset),
// a gap crossing at the forward gap cell.  For a segment free at both ends
// the total is the optimal score.
//
// A forward cell (k, hf) and the reverse cell on the same diagonal (kd - k,
// hr) cross exactly when their anti-diagonals 2 hf - k and 2 hr - (kd - k)
// add up to m + n or more.  Each slot keeps the furthest anti-diagonal of
// its present cells per component, so a pair of wavefronts whose maxima add
// up to less is not scanned: before the two passes meet, no check reads a
// cell.
//
// One group of GW warps per segment, persistent over a work queue.  The
// rings of both directions live in global memory (indexed by diagonal:
// k + m + 1), of RT: int16 for groups of 1 and 4 warps (segments whose
// longer side is below 16,384, so every offset fits; half the DRAM traffic
// of int32, which bounds these groups on long segments), int32 for 16-warp
// groups; negative values are absent cells.  Each slot's limits and
// per-component present ranges live in shared memory.  The reverse pass's
// M before extension is not stored (the cut reads only the forward one).
// Scores run in units of g = gcd(x, o, e).
#pragma once

#include <climits>
#include <type_traits>

#include "tsu_common.cuh"
#include "tsu_extend.cuh"

namespace tsu {

constexpr int32_t kBNull = -(1 << 30);  // an absent cell
enum : int { kCM = 0, kCMP = 1, kCI = 2, kCD = 3 };

struct BidirSeg {
  int32_t pair;       // pair of the batch whose sequences hold the segment
  int32_t v0, h0;     // segment start in the pattern and the text
  int32_t m, n;       // segment lengths
  int32_t begin, end; // 'M', 'I', 'D'
};

struct BidirArgs {
  SeqView seq;           // the batch's byte sequences
  PackView pk;           // packed words of the sequences
  PackView pkr;          // packed words of the reversed sequences (same offsets)
  const BidirSeg* segs;
  int64_t n_segs;
  Pen pen;               // reduced penalties (one gap piece)
  int ring_w;            // diagonals per ring slot (>= m + n + 3 of every segment)
  void* ring;            // per group: [2][rm][4][ring_w] of the kernel's ring type
  int64_t ring_stride;   // ring elements per group
  int32_t* out_T;        // per segment: lowest crossing total (score units), -1 none
  int32_t* out_comp;     // 'M', 'I', 'D'
  int32_t* out_k;        // forward diagonal of the cut
  int32_t* out_h;        // cut offset (text position)
  int32_t* status;       // per segment: kPairOk / kPairInternal
  unsigned int* queue;
  unsigned long long* work;  // [2]: wavefront cells computed, score steps (nullable)
};

// Shared memory of a group: limits [2][rm][kBLim] (lo, hi, then first /
// last present diagonal of M, I, D, then the furthest anti-diagonal 2 h - k
// of the present cells of M, I, D), warp partials [GW][kBLim], broadcast
// words [8].
constexpr int kBLim = 12;
__host__ __device__ inline int bidir_group_smem(const Pen& p, int gw) {
  return (2 * p.rm * kBLim + gw * kBLim + 8) * 4;
}

template <int GW>
constexpr int bidir_cta_threads() {
  return GW <= 4 ? 128 : 32 * GW;
}

template <int GW>
__device__ __forceinline__ void bidir_sync(int gid) {
  if constexpr (GW == 1) {
    __syncwarp();
  } else {
#ifdef TSU_WARP_EMU
    emu::named_bar(1 + gid, 32 * GW);
#else
    asm volatile("bar.sync %0, %1;" ::"r"(1 + gid), "r"(32 * GW) : "memory");
#endif
  }
}

// Longest common prefix of pattern[v..] and text[h..] (at most rem), in the
// forward or reversed packed words, or byte by byte for pairs with bytes
// outside ACGT (fwd: at pat[v], txt[h]; reversed: backwards from pat[v],
// txt[h]).
__device__ __forceinline__ int bidir_lcp(bool bytes, bool fwd, const uint32_t* pw, const uint32_t* tw,
                                         const uint8_t* pb, const uint8_t* tb, int v, int h, int rem) {
  if (!bytes) {
    const GlobalSeq P{pw}, T{tw};
    return lcp16(P, v, T, h, rem);
  }
  int l = 0;
  if (fwd) {
    while (l < rem && pb[v + l] == tb[h + l]) ++l;
  } else {
    while (l < rem && pb[v - l] == tb[h - l]) ++l;
  }
  return l;
}

// 128-thread blocks (1- and 4-warp groups): at least 5 per SM (96 registers,
// no spills; 20 warps per SM).
// Ring element type of a group of GW warps (int16 below 16 warps).
template <int GW>
using bidir_ring_t = typename std::conditional<(GW < 16), int16_t, int32_t>::type;
__host__ __device__ inline int bidir_ring_bytes(int gw) { return gw < 16 ? 2 : 4; }

template <int GW>
__global__ void __launch_bounds__(bidir_cta_threads<GW>(), GW <= 4 ? 5 : 1) bidir_kernel(BidirArgs a) {
  using RT = bidir_ring_t<GW>;
  constexpr RT kRNull = (RT)(sizeof(RT) == 2 ? -16384 : kBNull);  // stored absent cell
#ifdef TSU_WARP_EMU
  unsigned char* smem_raw = emu::dyn_smem();
#else
  extern __shared__ __align__(16) unsigned char smem_raw[];
#endif
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int GT = 32 * GW;
  const int tid = threadIdx.x;
  const int gid = tid / GT;
  const int gt = tid - gid * GT;
  const int lane = tid & 31;
  const int wig = gt >> 5;
  const int gpb = blockDim.x / GT;
  const int64_t ggroup = (int64_t)blockIdx.x * gpb + gid;
  const Pen pen = a.pen;
  const int rm = pen.rm;
  const int mx = rm - 1;                 // deepest source, and the check window
  const int x = pen.x, go = pen.go, ge = pen.ge, oo = pen.go - pen.ge;  // oo: the gap opening alone
  int* lim = reinterpret_cast<int*>(smem_raw + (size_t)gid * bidir_group_smem(pen, GW));
  int* part = lim + 2 * rm * kBLim;
  int* bc = part + GW * kBLim;
  RT* const ring = static_cast<RT*>(a.ring) + ggroup * a.ring_stride;
  const int W = a.ring_w;

  for (;;) {
    unsigned qi;
    if (gt == 0) bc[0] = (int)atomicAdd(a.queue, 1u);
    bidir_sync<GW>(gid);
    qi = (unsigned)bc[0];
    bidir_sync<GW>(gid);
    if ((int64_t)qi >= a.n_segs) break;
    const BidirSeg sg = a.segs[qi];
    const int m = sg.m, n = sg.n, kd = n - m, koff = m + 1;
    const int64_t pair = sg.pair;
    const bool bytes = a.pk.nonacgt[pair] | a.pk.nonacgt[a.seq.n + pair];
    const int M_full = a.seq.pat_len[pair], N_full = a.seq.txt_len[pair];
    // forward words and positions; the reversed segment starts at
    // M_full - v0 - m in the reversed pattern (N_full - h0 - n in the text)
    const uint32_t* fpw = reinterpret_cast<const uint32_t*>(a.pk.words + a.pk.woff[pair]);
    const uint32_t* ftw = reinterpret_cast<const uint32_t*>(a.pk.words + a.pk.woff[a.seq.n + pair]);
    const uint32_t* rpw = reinterpret_cast<const uint32_t*>(a.pkr.words + a.pkr.woff[pair]);
    const uint32_t* rtw = reinterpret_cast<const uint32_t*>(a.pkr.words + a.pkr.woff[a.seq.n + pair]);
    const uint8_t* pb = a.seq.pat + a.seq.pat_off[pair];
    const uint8_t* tb = a.seq.txt + a.seq.txt_off[pair];
    const int rv0 = M_full - sg.v0 - m, rh0 = N_full - sg.h0 - n;
    // the CPU model's step bound, (m + n) max(x, o + e) + 2 (o + e) + 2, in
    // score units
    const int64_t smax = (int64_t)(m + n) * mx + 2 * go + 2;
    unsigned long long n_cells = 0, n_steps = 0;

    auto L = [&](int d, int s) -> int* { return lim + (d * rm + s % rm) * kBLim; };
    // slots by index (0..rm-1): the callers keep each direction's current
    // slot and step back from it, so the hot paths divide by rm nowhere
    auto LS = [&](int d, int sl) -> int* { return lim + (d * rm + sl) * kBLim; };
    auto CS = [&](int d, int sl, int c) -> RT* { return ring + ((int64_t)(d * rm + sl) * 4 + c) * W + koff; };
    // a stored cell as an offset, kBNull when absent
    auto ld = [&](const RT* p, int64_t i) -> int32_t {
      const int32_t v = p[i];
      return v < 0 ? kBNull : v;
    };
    auto sv = [&](int32_t v) -> RT { return v < 0 ? kRNull : (RT)v; };
    auto back = [&](int sl, int b) -> int { return sl - b + (sl < b ? rm : 0); };  // slot of b scores before (b < rm)
    auto cells = [&](int d, int s, int c) -> RT* {
      return ring + ((int64_t)(d * rm + s % rm) * 4 + c) * W + koff;
    };
    auto get = [&](int d, int s, int c, int k) -> int32_t {
      if (s < 0) return kBNull;
      const int* l = L(d, s);
      if (k < l[0] || k > l[1]) return kBNull;
      return ld(cells(d, s, c), k);
    };
    auto inb = [&](int32_t off, int k) -> bool {
      return ((uint32_t)off <= (uint32_t)n) & ((uint32_t)(off - k) <= (uint32_t)m);
    };

    // One wavefront of direction d (0 forward, 1 reverse) at score s, in
    // ring slot sl (= s mod rm).
    auto compute = [&](int d, int s, int sl) {
      const int start = d == 0 ? sg.begin : 'M';
      const int forced = d == 0 ? 'M' : sg.end;
      int* out = LS(d, sl);
      RT* cM = CS(d, sl, kCM);
      RT* cMP = CS(d, sl, kCMP);
      RT* cI = CS(d, sl, kCI);
      RT* cD = CS(d, sl, kCD);
      if (s == 0) {
        if (gt == 0) {
          if (forced == 'M') {
            const int rem = min(m, n);
            const int lx = d == 0 ? bidir_lcp(bytes, true, fpw, ftw, pb, tb, sg.v0, sg.h0, rem)
                                  : bidir_lcp(bytes, false, rpw, rtw, pb, tb, bytes ? sg.v0 + m - 1 : rv0,
                                              bytes ? sg.h0 + n - 1 : rh0, rem);
            cMP[0] = 0;
            cM[0] = sv(lx);
            cI[0] = start == 'I' ? 0 : kRNull;
            cD[0] = start == 'D' ? 0 : kRNull;
            out[0] = 0, out[1] = 0;
            out[2] = 0, out[3] = 0;
            out[4] = start == 'I' ? 0 : 1, out[5] = 0;
            out[6] = start == 'D' ? 0 : 1, out[7] = 0;
            out[8] = 2 * lx;
            out[9] = start == 'I' ? 0 : kBNull;
            out[10] = start == 'D' ? 0 : kBNull;
          } else {
            out[0] = 1, out[1] = 0;
            out[2] = 1, out[3] = 0, out[4] = 1, out[5] = 0, out[6] = 1, out[7] = 0;
            out[8] = out[9] = out[10] = kBNull;
          }
        }
        bidir_sync<GW>(gid);
        return;
      }
      // envelope of the present sources, widened by one diagonal
      int lo = INT_MAX, hi = INT_MIN;
      auto widen = [&](int ss, int c) {
        if (ss < 0) return;
        const int* l = LS(d, back(sl, s - ss));
        const int plo = l[2 + 2 * c], phi = l[3 + 2 * c];
        if (plo > phi) return;
        lo = min(lo, plo - 1);
        hi = max(hi, phi + 1);
      };
      widen(s - x, 0);
      widen(s - go, 0);
      widen(s - ge, 1);
      widen(s - ge, 2);
      const bool seed_i = forced == 'I' && s == go && inb(1, 1);
      const bool seed_d = forced == 'D' && s == go && inb(0, -1);
      if (seed_i) lo = min(lo, 1), hi = max(hi, 1);
      if (seed_d) lo = min(lo, -1), hi = max(hi, -1);
      if (lo > hi) lo = 1, hi = 0;
      int pm0 = INT_MAX, pm1 = INT_MIN, pi0 = INT_MAX, pi1 = INT_MIN, pd0 = INT_MAX, pd1 = INT_MIN;
      int am = kBNull, ai = kBNull, ad = kBNull;  // furthest anti-diagonals
      // the three source slots (s - x, s - o - e, s - e), resolved once per
      // step: cells of component c on diagonal k at base[c W + k] when k is
      // in [lo, hi]
      struct Src {
        const RT* base;
        int lo, hi;
      };
      auto src = [&](int ss) -> Src {
        if (ss < 0) return Src{ring, 1, 0};
        const int b = back(sl, s - ss);
        const int* l = LS(d, b);
        return Src{CS(d, b, 0), l[0], l[1]};
      };
      const Src SX = src(s - x), SG = src(s - go), SE = src(s - ge);
      auto rd = [&](const Src& S, int c, int k) -> int32_t {
        return (k < S.lo || k > S.hi) ? kBNull : ld(S.base, (int64_t)c * W + k);
      };
      // this direction's words and the position of its base 0 (packed:
      // forward (v0, h0), reversed (rv0, rh0); bytes: read forwards from
      // (v0, h0) or backwards from (v0 + m - 1, h0 + n - 1))
      const uint32_t* dpw = d == 0 ? fpw : rpw;
      const uint32_t* dtw = d == 0 ? ftw : rtw;
      const int dv0 = d == 0 ? sg.v0 : (bytes ? sg.v0 + m - 1 : rv0);
      const int dh0 = d == 0 ? sg.h0 : (bytes ? sg.h0 + n - 1 : rh0);
      const int dir = d == 0 || !bytes ? 1 : -1;
      for (int k = lo + gt; k <= hi; k += GT) {
        int32_t ins = max(rd(SG, kCM, k - 1), rd(SE, kCI, k - 1)) + 1;
        if (seed_i && k == 1) ins = max(ins, 1);
        int32_t del = max(rd(SG, kCM, k + 1), rd(SE, kCD, k + 1));
        if (seed_d && k == -1) del = max(del, 0);
        const int32_t mis = rd(SX, kCM, k) + 1;
        const bool vi = inb(ins, k), vd = inb(del, k);
        cI[k] = vi ? (RT)ins : kRNull;
        cD[k] = vd ? (RT)del : kRNull;
        if (vi) pi0 = min(pi0, k), pi1 = k, ai = max(ai, 2 * ins - k);
        if (vd) pd0 = min(pd0, k), pd1 = k, ad = max(ad, 2 * del - k);
        const int32_t pv = max(mis, max(ins, del));
        if (inb(pv, k)) {
          const int vv = pv - k;
          const int rem = min(m - vv, n - pv);
          const int lx = bidir_lcp(bytes, dir > 0, dpw, dtw, pb, tb, dv0 + dir * vv, dh0 + dir * pv, rem);
          if (d == 0) cMP[k] = (RT)pv;
          cM[k] = (RT)(pv + lx);
          pm0 = min(pm0, k), pm1 = k;
          am = max(am, 2 * (pv + lx) - k);
        } else {
          if (d == 0) cMP[k] = kRNull;
          cM[k] = kRNull;
        }
      }
      pm0 = __reduce_min_sync(FULL, pm0);
      pm1 = __reduce_max_sync(FULL, pm1);
      pi0 = __reduce_min_sync(FULL, pi0);
      pi1 = __reduce_max_sync(FULL, pi1);
      pd0 = __reduce_min_sync(FULL, pd0);
      pd1 = __reduce_max_sync(FULL, pd1);
      am = __reduce_max_sync(FULL, am);
      ai = __reduce_max_sync(FULL, ai);
      ad = __reduce_max_sync(FULL, ad);
      if constexpr (GW > 1) {
        if (lane == 0) {
          int* pp = part + wig * kBLim;
          pp[0] = pm0, pp[1] = pm1, pp[2] = pi0, pp[3] = pi1, pp[4] = pd0, pp[5] = pd1;
          pp[6] = am, pp[7] = ai, pp[8] = ad;
        }
        bidir_sync<GW>(gid);
        int q0 = INT_MAX, q1 = INT_MIN, q2 = INT_MAX, q3 = INT_MIN, q4 = INT_MAX, q5 = INT_MIN;
        int q6 = kBNull, q7 = kBNull, q8 = kBNull;
        if (lane < GW) {
          const int* pp = part + lane * kBLim;
          q0 = pp[0], q1 = pp[1], q2 = pp[2], q3 = pp[3], q4 = pp[4], q5 = pp[5];
          q6 = pp[6], q7 = pp[7], q8 = pp[8];
        }
        pm0 = __reduce_min_sync(FULL, q0);
        pm1 = __reduce_max_sync(FULL, q1);
        pi0 = __reduce_min_sync(FULL, q2);
        pi1 = __reduce_max_sync(FULL, q3);
        pd0 = __reduce_min_sync(FULL, q4);
        pd1 = __reduce_max_sync(FULL, q5);
        am = __reduce_max_sync(FULL, q6);
        ai = __reduce_max_sync(FULL, q7);
        ad = __reduce_max_sync(FULL, q8);
      }
      bidir_sync<GW>(gid);  // every thread has read the sources' limits and partials
      if (gt == 0) {
        out[0] = lo, out[1] = hi;
        out[2] = pm0 <= pm1 ? pm0 : 1, out[3] = pm0 <= pm1 ? pm1 : 0;
        out[4] = pi0 <= pi1 ? pi0 : 1, out[5] = pi0 <= pi1 ? pi1 : 0;
        out[6] = pd0 <= pd1 ? pd0 : 1, out[7] = pd0 <= pd1 ? pd1 : 0;
        out[8] = am, out[9] = ai, out[10] = ad;
      }
      n_cells += (unsigned long long)(hi - lo + 1);
      ++n_steps;
      bidir_sync<GW>(gid);  // the new limits and cells are visible
    };

    // Crossing checks of one turn: the new wavefront (direction d_new at
    // s_new) against the other side's scores s_lo..s_hi, in ascending order;
    // candidates keyed (total, check, component, diagonal), the lowest kept.
    int have = 0, bT = 0, bC = 'M', bK = 0, bH = 0;
    // The new best: decode the check, component and diagonal of the key, and
    // read the cut from the rings.
    auto record = [&](unsigned long long key, int total, int d_new, int s_new, int s_lo) {
      const int j = (int)((key >> 34) & 63), ci = (int)((key >> 32) & 3);
      const int k = (int)(uint32_t)(key & 0xffffffffu) - koff;
      const int s2 = s_lo + j;
      const int sf = d_new == 0 ? s_new : s2, sr = d_new == 0 ? s2 : s_new;
      have = 1;
      bT = total;
      bK = k;
      if (ci == 0) {
        bC = 'M';
        const int32_t pre = ld(cells(0, sf, kCMP), k), hr = get(1, sr, kCM, kd - k);
        bH = max(pre, n - hr);
      } else {
        bC = ci == 1 ? 'I' : 'D';
        bH = ld(cells(0, sf, ci == 1 ? kCI : kCD), k);
      }
    };

    // sl_new: slot of s_new; sl_hi: the other side's slot of s_hi.
    auto check = [&](int d_new, int s_new, int sl_new, int s_lo, int s_hi, int sl_hi) {
      unsigned long long key = ~0ull;
      for (int s2 = s_lo; s2 <= s_hi; ++s2) {
        const int sf = d_new == 0 ? s_new : s2, sr = d_new == 0 ? s2 : s_new;
        const int sl2 = back(sl_hi, s_hi - s2);
        const int slf = d_new == 0 ? sl_new : sl2, slr = d_new == 0 ? sl2 : sl_new;
        const int* lf = LS(0, slf);
        const int* lr = LS(1, slr);
        for (int ci = 0; ci < 3; ++ci) {
          // nothing crosses below an anti-diagonal sum of m + n
          if (lf[8 + ci] + lr[8 + ci] < m + n) continue;
          const int plo = lf[2 + 2 * ci], phi = lf[3 + 2 * ci];
          const int c = ci == 0 ? kCM : (ci == 1 ? kCI : kCD);
          const RT* fc = CS(0, slf, c);
          const RT* rc = CS(1, slr, c);
          const int rlo = lr[0], rhi = lr[1];
          for (int k = plo + gt; k <= phi; k += GT) {
            const int32_t hf = fc[k];
            if (hf < 0) continue;
            const int kr = kd - k;
            const int32_t hr = (kr < rlo || kr > rhi) ? -1 : (int32_t)rc[kr];
            if (hr < 0 || hf + hr < n) continue;
            const int total = sf + sr - (ci == 0 ? 0 : oo);
            const unsigned long long kk = ((unsigned long long)(uint32_t)total << 40) |
                                          ((unsigned long long)(s2 - s_lo) << 34) | ((unsigned long long)ci << 32) |
                                          (unsigned long long)(uint32_t)(k + koff);
            key = kk < key ? kk : key;
          }
        }
      }
      // group minimum of the 64-bit keys (butterflies: every lane ends with
      // it; a warp whose lanes found nothing keeps ~0 without them)
      if (__any_sync(FULL, key != ~0ull))
        for (int sh = 16; sh > 0; sh >>= 1) {
          const unsigned long long o2 = __shfl_xor_sync(FULL, key, sh);
          key = o2 < key ? o2 : key;
        }
      if constexpr (GW > 1) {
        unsigned long long* kp = reinterpret_cast<unsigned long long*>(part);  // GW words (part holds kBLim GW ints)
        bidir_sync<GW>(gid);
        if (lane == 0) kp[wig] = key;
        bidir_sync<GW>(gid);
        key = lane < GW ? kp[lane] : ~0ull;
        for (int sh = 16; sh > 0; sh >>= 1) {
          const unsigned long long o2 = __shfl_xor_sync(FULL, key, sh);
          key = o2 < key ? o2 : key;
        }
        bidir_sync<GW>(gid);
      }
      const int total = (int)(key >> 40);
      if (key != ~0ull && (!have || total < bT)) record(key, total, d_new, s_new, s_lo);
      // the cut was read from the rings: no lane may overwrite them before
      bidir_sync<GW>(gid);
    };
    int st = kPairOk;
    compute(0, 0, 0);
    compute(1, 0, 0);
    check(0, 0, 0, 0, 0, 0);
    int sf = 0, sr = 0, slf = 0, slr = 0;  // scores and their ring slots
    while (sf <= smax) {
      if (have && sf + sr - 2 * mx - oo > bT) break;
      if (sf <= sr) {
        ++sf;
        slf = slf + 1 == rm ? 0 : slf + 1;
        compute(0, sf, slf);
        check(0, sf, slf, max(0, sr - mx), sr, slr);
      } else {
        ++sr;
        slr = slr + 1 == rm ? 0 : slr + 1;
        compute(1, sr, slr);
        check(1, sr, slr, max(0, sf - mx), sf, slf);
      }
    }
    if (!have) st = kPairInternal;
    if (gt == 0) {
      a.out_T[qi] = have ? bT : -1;
      a.out_comp[qi] = bC;
      a.out_k[qi] = bK;
      a.out_h[qi] = bH;
      a.status[qi] = st;
      if (a.work) {
        atomicAdd(a.work, n_cells);
        atomicAdd(a.work + 1, n_steps);
      }
    }
    bidir_sync<GW>(gid);
  }
}

// Base score of the recursion (score units): a segment whose crossing
// total is at most max(2 max(x, o + e), TSU_BIDIR_BASE_MIN) is aligned whole
// by the segment kernel.  Larger bases mean fewer recursion levels of
// small segments and more history per leaf warp (about 16 B x base^2):
// on 1,000,000 pairs of 1 kbp at 5 % a base of 256 took 834 ms against
// 2,656 ms at 32, on 20,000 pairs of 10 kbp at 15 % 5,313 against 6,150 ms.
#ifndef TSU_BIDIR_BASE_MIN
#define TSU_BIDIR_BASE_MIN 256
#endif
__host__ __device__ inline int bidir_base(const Pen& p) {
  const int b = 2 * (p.rm - 1);
  return b > TSU_BIDIR_BASE_MIN ? b : TSU_BIDIR_BASE_MIN;
}

// Arguments of the base-case segment kernel (tsu_segment.cuh).
struct SegArgs {
  SeqView seq;
  PackView pk, pkr;       // forward and reversed packed words
  const BidirSeg* segs;
  int64_t n_segs;
  Pen pen;
  int g;                  // score unit
  void* hist;             // per warp: hist_cap x 3 (M, I, D) of the launch's history type
  int64_t hist_cap;
  int32_t* table;         // per warp: step_cap x 9 int32
  int32_t step_cap;
  uint32_t* wruns;        // per warp: wruns_cap runs, where the backtrace writes
  int64_t wruns_cap;
  uint32_t* runs;         // run arena: each leaf's runs at run_off, packed
  int64_t runs_cap;
  unsigned long long* cursor;  // arena cursor (runs handed out)
  int64_t* run_off;       // per segment: first run in the arena
  int32_t* run_len;       // per segment: runs
  int32_t* status;        // per segment: kPairOk, kPairScratch (more steps or
                          // history), kPairArena (arena full), kPairInternal
  int32_t* pair_score;    // nullable: per pair, the segment's score (penalty units)
  unsigned int* queue;
  unsigned long long* work;  // nullable: [2] wavefront cells computed, score steps
};

constexpr int kSegThreads = 128;
// Shared memory of a segment-kernel block: per warp the last rm rows of the
// step table (9 int each).
__host__ __device__ inline size_t seg_smem_bytes(const Pen& p) {
  return (size_t)(kSegThreads / 32) * (size_t)p.rm * 9 * sizeof(int);
}

// Runs a segment of m + n bases can need when it ends below step_cap: each
// mismatch run costs at least x and each gap run at least o + e, except a
// gap continued from the segment's begin or left free at its end (one each),
// and M runs lie between them.
__host__ __device__ inline int64_t seg_run_cap(const Pen& p, int64_t bases, int step_cap) {
  const int minrun = p.x < p.go ? p.x : p.go;
  const int64_t b = 2 * ((int64_t)step_cap / minrun) + 5;
  return bases < b ? (bases > 0 ? bases : 1) : b;
}

// History cells (3 int32 each) a warp needs for step_cap steps of segments
// whose m + n is at most bases: the wavefront at score s spans at most
// 2 s + 1 diagonals, and never more than m + n + 3.
__host__ __device__ inline int64_t seg_hist_cap(int step_cap, int64_t bases) {
  int64_t c = 0;
  for (int s = 0; s < step_cap; ++s) c += (2 * (int64_t)s + 3 < bases + 3) ? 2 * (int64_t)s + 3 : bases + 3;
  return c;
}

#ifndef TSU_WARP_EMU
// Instantiations (tsu_bidir.cu): groups of 1, 4 or 16 warps.
cudaError_t bidir_occupancy(int gw, int threads, size_t smem, int* occ);
void launch_bidir(int gw, int blocks, int threads, size_t smem, cudaStream_t st, const BidirArgs& a);
// The base-case kernels (tsu_segment.cuh), launched from tsu_bidir.cu.
cudaError_t segment_occupancy(const Pen& pen, int* blocks_per_sm);  // the lower of the two history types
void launch_segment(bool int16_history, int blocks, int threads, cudaStream_t st, const SegArgs& a);
void launch_seg_runs(bool write, int blocks, cudaStream_t st, int64_t n, const int32_t* pre_st, const int64_t* pre_off,
                     const int32_t* pre_len, const int64_t* first, const int64_t* run_off, const int32_t* run_len,
                     const uint32_t* runs, const int32_t* status, int64_t* out_len, const int64_t* out_off,
                     uint32_t* out);
void launch_whole_pairs(int blocks, cudaStream_t st, int64_t n, const int32_t* plen, const int32_t* tlen,
                        BidirSeg* segs);
#endif

}  // namespace tsu
