// tsu_align.cuh -- the persistent gap-affine WFA kernel.
//
// Re-design of the reference kernel wfa_dispatcher (wfa_gpu.cu:191-722):
//   * persistent grid; each group of GW warps pulls pairs from a device work
//     queue (the reference launched one 32-thread block per pair,
//     wfa_gpu.cu:113).  GW = 1 for short pairs (four independent warps per
//     block); GW = 2..16 lets one long pair use several warps;
//   * score steps s = 0, 1, ... in units of g = gcd(x, o, e);
//   * one fused pass per step: thread t of the group owns diagonals
//     k = lo + t + 32*GW*j and computes I, D and M of score s from the ring
//     slots of scores s - x, s - o - e and s - e (wfa_gpu.cu:610-631),
//     nullifies an out-of-bounds M (wfa_gpu.cu:628-629), extends M along its
//     diagonal (wfa_gpu.cu:257-287), checks the end point (wfa_gpu.cu:288-338)
//     and, with kCigar, streams one backtrace word per (score, diagonal) to
//     HBM; the ends of M, I and D are trimmed with warp min/max reductions
//     combined across the group's warps (wfa_gpu.cu:636-719);
//   * kModeShared: the ring of the last max(x, o+e)+1 scores is int16 in
//     shared memory (offsets clamped to [null, n+1], which changes no valid
//     cell: validity depends only on the value and the diagonal, so a clamped
//     out-of-bounds candidate still loses every max to -- or stays invalid
//     against -- any valid one) and the pair's packed sequences are staged
//     in shared memory.  Pairs wider than the ring or longer than the staging
//     area are handed back for a kModeGlobal pass (int32 ring in global
//     memory, sequences read through the read-only cache).
// Synchronisation of a group (GW > 1): one named barrier per step, after the
// cell loop; warp partial reductions are double-buffered by step parity and
// every thread writes the (identical) slot limits itself, so the next step
// reads them without a second barrier.  Null steps, which read slot limits
// and then overwrite one, take a barrier in between.
// Thread 0 of the group walks the backtrace once the end is reached
// (tsu_backtrace.cuh).
// kModel = kModelDual: dual gap-affine (a gap of length L costs
// min(o1 + e1 L, o2 + e2 L)), the I2 / D2 components the reference declares
// (common.h:52-58,67-77,80-87): two more gap components with their own ring
// slots (s - o2 - e2, s - e2), M = max(mismatch, D2, D1, I2, I1) with ties in
// that (piggyback) order, and a backtrace word with a 3-bit M source and four
// extension bits.
// kModel = kModelLinear: gap-linear (a gap costs e per base; edit and indel
// distance): the M component alone, M = max(M[s-x][k] + 1, M[s-e][k-1] + 1,
// M[s-e][k+1]), ties mismatch > deletion > insertion; no I/D ring slots.
#pragma once

#include <type_traits>

#include "tsu_backtrace.cuh"
#include "tsu_common.cuh"
#include "tsu_extend.cuh"

namespace tsu {

template <int GW>
__device__ __forceinline__ void group_sync(int gid) {
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

template <int GW>
constexpr int cta_threads() {
  return GW <= 4 ? 128 : 32 * GW;
}
template <int kMode, int GW>
constexpr int cta_min_blocks() {
  return kMode == kModeShared ? (GW == 1 ? 7 : (GW <= 4 ? 6 : (GW == 8 ? 3 : 1))) : (GW <= 4 ? 4 : (GW == 8 ? 2 : 1));
}

template <bool kCigar, int kMode, int GW, int kModel = kModelAffine>
__global__ void __launch_bounds__(cta_threads<GW>(), (cta_min_blocks<kMode, GW>())) align_kernel(AlignArgs a) {
  static_assert(GW == 1 || GW == 2 || GW == 4 || GW == 8 || GW == 16 || GW == 32, "warps per pair");
  constexpr bool kDual = (kModel & 7) == kModelDual;
  constexpr bool kLin = (kModel & 7) == kModelLinear;
  constexpr bool kLowMem = kCigar && (kModel & kLowMemFlag) != 0;
  // Groups of 2 to 16 warps (wide wavefronts) read the sources of a warp's
  // block of diagonals without range tests where all of them lie inside
  // their trimmed ranges, and extend and track the trimmed ends with selects
  // instead of divergent branches (measured: 10 kbp at 15 %, 16 warps, -5 %).
  // The one-warp kernel runs at 72 registers with its ALU pipe the busiest,
  // and the 32-warp kernels at 64 registers: there the selects and the extra
  // registers cost more than the branches (+8 % at 1 kbp), so they keep the
  // branches.
  constexpr bool kWide = GW > 1 && GW < 32;
  static_assert(!(kModel & kLowMemFlag) || kCigar, "low-memory: CIGAR kernels");
  using RT = typename std::conditional<kMode == kModeShared, int16_t, int32_t>::type;
  // null of a source read outside its slot's trimmed range: the int16 ring's
  // null in shared mode, so that every value the cell loop computes stays
  // within int16 and needs no lower clamp when stored
  constexpr int32_t NUL = kMode == kModeShared ? (int32_t)kNull16 : kNull;
  // Global-ring groups of up to 16 warps stage the pair's packed words in
  // shared memory; the 32-warp groups run at 64 registers, where the staging
  // state costs spills, and read the words from global memory.
  constexpr bool kStage = kMode == kModeGlobal && GW < 32;
  using S = typename std::conditional<kMode == kModeShared, SharedSeq,
                                      typename std::conditional<kStage, AnySeq, GlobalSeq>::type>::type;
#ifdef TSU_WARP_EMU
  unsigned char* smem_raw = emu::dyn_smem();  // CPU warp emulation of the tests
#else
  extern __shared__ __align__(16) unsigned char smem_raw[];
#endif
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int GT = 32 * GW;  // threads per group
  const int tid = threadIdx.x;
  const int gid = tid / GT;  // group within the block
  const int gt = tid - gid * GT;
  const int lane = tid & 31;
  const int wig = gt >> 5;  // warp within the group
  const int gpb = blockDim.x / GT;
  const int64_t ggroup = (int64_t)blockIdx.x * gpb + gid;
  constexpr int PW = kDual ? 16 : 8;  // partial words per warp and step parity
  const int ns = a.pen.slots();
  const int W = a.ring_w;
  const int rm = a.pen.rm, re = a.pen.re;
  unsigned char* gsm = smem_raw + (size_t)gid * group_smem_bytes(a.pen, W, kMode, a.seq_cap, GW);
  int* s_lo = reinterpret_cast<int*>(gsm);
  int* s_hi = s_lo + ns;
  int* s_alo = s_hi + ns;
  int* part = s_alo + ns;                      // [2][GW][PW] warp partials (GW > 1)
  int* bc = part + (GW > 1 ? 2 * PW * GW : 0);  // broadcast words
  unsigned char* tail = reinterpret_cast<unsigned char*>(bc + 4);
  RT* ring;
  uint32_t* sseq = nullptr;
  if constexpr (kMode == kModeShared) {
    ring = reinterpret_cast<RT*>(tail);
    sseq = reinterpret_cast<uint32_t*>(tail + ((ns * W * 2 + 15) & ~15));
  } else {
    ring = reinterpret_cast<RT*>(a.ring_global + ggroup * a.ring_stride);
    if (kStage && a.seq_cap > 0) sseq = reinterpret_cast<uint32_t*>(gsm + ((tail - gsm + 15) & ~15) + 16);
  }
  uint32_t* const hist = kCigar ? a.hist + ggroup * a.hist_cap : nullptr;
  int2* const table = kCigar ? a.table + ggroup * (int64_t)a.table_cap : nullptr;

  for (;;) {
    unsigned qi;
    if constexpr (GW == 1) {
      unsigned q = 0;
      if (lane == 0) q = atomicAdd(a.queue, 1u);
      qi = __shfl_sync(FULL, q, 0);
    } else {
      if (gt == 0) bc[0] = (int)atomicAdd(a.queue, 1u);
      group_sync<GW>(gid);
      qi = (unsigned)bc[0];
    }
    if ((int64_t)qi >= a.n_order) break;
    const int64_t pair = a.order ? a.order[qi] : (int64_t)qi;
    const int m = a.seq.pat_len[pair];
    const int n = a.seq.txt_len[pair];
    const bool bytemode = a.pk.nonacgt[pair] | a.pk.nonacgt[a.seq.n + pair];
    const uint32_t* gpw = reinterpret_cast<const uint32_t*>(a.pk.words + a.pk.woff[pair]);
    const uint32_t* gtw = reinterpret_cast<const uint32_t*>(a.pk.words + a.pk.woff[a.seq.n + pair]);
    const uint8_t* pb = a.seq.pat + a.seq.pat_off[pair];
    const uint8_t* tb = a.seq.txt + a.seq.txt_off[pair];
    const int k_end = n - m;
    const int64_t s_max = score_bound(m, n, a.pen);
    const int pwn = 2 * (int)packed_words(m);  // uint32 words
    const int twn = 2 * (int)packed_words(n);

    int32_t st = kPairOk;
    if constexpr (kMode == kModeShared) {
      // bytes outside ACGT, lengths beyond int16 or sequences beyond the
      // staging area: handled by the global variant
      if (bytemode || m > 32000 || n > 32000 || pwn + twn > a.seq_cap) st = kPairScratch;
    }
    if constexpr (kDual) {
      if (m > kDualMaxLen || n > kDualMaxLen) st = kPairInternal;  // beyond the backtrace word
    }
    int s_end = -1;
    int k_fin = k_end;  // end diagonal (free ends: the lowest that ends)
    constexpr bool lowmem = kLowMem;  // checkpointed history (low-memory mode)
    const int K = a.ckpt_k;
    int32_t lm_len = 0;  // the low-memory walk's CIGAR (thread 0 of the group)
    int64_t lm_pos = 0;
    int64_t hbase = 0;
    unsigned long long n_cells = 0, n_steps = 0;
    uint32_t n_ext = 0;  // bases matched by this thread's extend steps

    if (st == kPairOk) {
      const uint32_t* pws;
      const uint32_t* tws;
      if constexpr (kMode == kModeShared) {
        for (int i = gt; i < pwn; i += GT) sseq[i] = __ldg(gpw + i);
        for (int i = gt; i < twn; i += GT) sseq[pwn + i] = __ldg(gtw + i);
        pws = sseq;
        tws = sseq + pwn;
      } else if (kStage && a.seq_cap > 0 && pwn + twn <= a.seq_cap) {
        // stage the pair's words in shared memory with plain loads (measured
        // on one B200 against two bulk copies completing on an mbarrier:
        // 10 kbp pairs at 15 % on 16-warp groups 3.30 s vs 3.38 s, 1 kbp
        // pairs on 8-warp groups 0.751 s vs 0.759 s)
        for (int i = gt; i < pwn; i += GT) sseq[i] = __ldg(gpw + i);
        for (int i = gt; i < twn; i += GT) sseq[pwn + i] = __ldg(gtw + i);
        group_sync<GW>(gid);
        pws = sseq;
        tws = sseq + pwn;
      } else {
        pws = gpw;
        tws = gtw;
      }
      const S P{pws}, T{tws};
      for (int i = gt; i < ns; i += GT) {
        s_lo[i] = 1;
        s_hi[i] = 0;
        s_alo[i] = 0;
      }
      group_sync<GW>(gid);
      // int16 ring: values above n + 1 are stored as n + 1 and values below
      // kNull16 as kNull16.  A stored value in (kNull16, 0) can only come from
      // an I chain of +1 per step that moves one diagonal per step inside the
      // component's trimmed range, at most ring_w (< 16,384) diagonals wide,
      // so it stays negative: every clamped value keeps its validity and its
      // order against any valid offset.
      auto store = [&](int idx, int32_t v) {
        if constexpr (kMode == kModeShared)
          ring[idx] = (RT)max(min(v, n + 1), (int32_t)kNull16);
        else
          ring[idx] = v;
      };
      // The cell loop's stores (sources read as NUL outside their ranges):
      // an extended M is a valid offset (<= n) or NUL; a D value is the
      // largest of its sources (M and D values one diagonal over), so at
      // most n and at least kNull16; an I value is its largest source + 1, at
      // least kNull16 + 1 and at most n + 2, clamped to n + 1.  A negative I
      // value climbs one per diagonal it moves, as under store(), so every
      // stored value keeps its validity and its order against any valid
      // offset.
      auto store_md = [&](int idx, int32_t v) { ring[idx] = (RT)v; };
      auto store_i = [&](int idx, int32_t v) {
        if constexpr (kMode == kModeShared)
          ring[idx] = (RT)min(v, n + 1);
        else
          ring[idx] = v;
      };
      // ---- score 0: M[0] = {k = 0: offset 0}, extended (wfa_gpu.cu:239-242)
      const int lo0 = -min(a.ef_pb, m), hi0 = min(a.ef_tb, n);
      if (lo0 == hi0) {
        if (gt == 0) {
          const int rem = m < n ? m : n;
          const int32_t o0 =
              (kMode == kModeGlobal && bytemode) ? lcp8(pb, m, 0, tb, n, 0, rem) : lcp16(P, 0, T, 0, rem);
          store(0, o0);
          s_lo[0] = 0;
          s_hi[0] = 0;
          s_alo[0] = 0;
          bc[1] = o0;
          if (kCigar) {
            table[0] = make_int2(0, 0);
            hist[0] = 0u;
          }
        }
        group_sync<GW>(gid);
        const int32_t o0 = bc[1];
        hbase = 1;
        n_cells = n_steps = 1;
        if (o0 >= n && (k_end == 0 || (a.ef_pe >= m - o0))) {
          s_end = 0;
          k_fin = 0;
        } else if (a.ef_te > 0 && o0 >= m && o0 >= n - a.ef_te) {
          s_end = 0;
          k_fin = 0;
        }
      } else if (hi0 - lo0 + 1 > W || (kCigar && hi0 - lo0 + 1 > a.hist_cap)) {
        st = kPairScratch;
      } else {
        // free beginnings: diagonals -pattern_begin_free..text_begin_free at
        // offset max(k, 0), each extended; the lowest ending diagonal wins
        int fk = INT_MAX;
        for (int k = lo0 + gt; k <= hi0; k += GT) {
          const int32_t p0 = k > 0 ? k : 0;
          const int vv = p0 - k;
          const int rem = min(m - vv, n - p0);
          const int32_t om =
              p0 + ((kMode == kModeGlobal && bytemode) ? lcp8(pb, m, vv, tb, n, p0, rem) : lcp16(P, vv, T, p0, rem));
          store(k - lo0, om);
          if (kCigar) hist[k - lo0] = (uint32_t)p0 << (kDual ? 8 : 4);
          const int ov = om - k;
          if (fk == INT_MAX && ((om >= n && ov >= m - a.ef_pe) || (ov >= m && om >= n - a.ef_te))) fk = k;
        }
        fk = __reduce_min_sync(FULL, fk);
        if constexpr (GW > 1) {
          if (lane == 0) part[wig * PW + 6] = fk;
          group_sync<GW>(gid);
          fk = __reduce_min_sync(FULL, lane < GW ? part[lane * PW + 6] : INT_MAX);
        }
        s_lo[0] = lo0;
        s_hi[0] = hi0;
        s_alo[0] = lo0;
        if (kCigar && gt == 0) table[0] = make_int2(lo0, 0);
        hbase = hi0 - lo0 + 1;
        n_cells = (unsigned long long)(hi0 - lo0 + 1);
        n_steps = 1;
        if (fk != INT_MAX) {
          s_end = 0;
          k_fin = fk;
        }
        if constexpr (GW == 1) __syncwarp();
      }

      int s = 0;
      int slm = 0, sli = 0, sli2 = 0;  // s mod rm, s mod re, s mod re2
      // ends of free-ended alignments: text consumed with at most ef_pe
      // pattern characters left (k <= k_end + ef_pe), or the pattern with at
      // most ef_te text characters left; end-to-end: k_end at offset n
      const int k_hi = k_end + a.ef_pe;
      const bool free_te = a.ef_te > 0;
      const int n_te = n - a.ef_te;
      // End-to-end alignments end on diagonal k_end alone: the cell loop
      // skips the end test, and after it the thread that computed k_end
      // reads that M value back from the ring (its own store: a valid
      // offset or the null, so >= n only at the end point).
      const bool ends_free = a.ef_pe > 0 || free_te;
      // One score step: the wavefronts of score s + 1 from the ring.  kH (a
      // compile-time tag): write the step's backtrace words and step-table
      // entry; detect: test for the end (not while recomputing history).
      auto step = [&](auto hist_tag, bool detect) {
        constexpr bool kH = kCigar && decltype(hist_tag)::value;
          ++s;
          if (++slm == rm) slm = 0;
          if constexpr (!kLin) {
            if (++sli == re) sli = 0;
          }
          if constexpr (kDual) {
            if (++sli2 == a.pen.re2) sli2 = 0;
          }
          if (s > s_max) {  // the end is reachable by s_max: inconsistency
            st = kPairInternal;
            return;
          }
          int q;
          q = slm - a.pen.x;
          if (q < 0) q += rm;
          const int slot_mm = q;
          q = slm - a.pen.go;
          if (q < 0) q += rm;
          const int slot_mo = q;
          q = sli - a.pen.ge;
          if (q < 0) q += re;
          const int slot_ie = rm + q;  // (unused by kLin)
          const int slot_de = rm + re + q;
          // sources: first diagonal, cell count (0 = null), ring index of lo.
          // Slot limits are either a trimmed range inside the slot's compute
          // range or the empty range (1, 0); the count is taken by comparison.
          int lo_mm = 0, c_mm = 0, b_mm = 0, lo_mo = 0, c_mo = 0, b_mo = 0;
          int lo_ie = 0, c_ie = 0, b_ie = 0, lo_de = 0, c_de = 0, b_de = 0;
          auto src = [&](int slot, int& lo_x, int& c_x, int& b_x) {
            const int l = s_lo[slot], h = s_hi[slot];
            if (h >= l) {
              lo_x = l;
              c_x = h - l + 1;
              b_x = slot * W + l - s_alo[slot];
            }
          };
          if (s - a.pen.x >= 0) src(slot_mm, lo_mm, c_mm, b_mm);
          if (s - a.pen.go >= 0) src(slot_mo, lo_mo, c_mo, b_mo);
          if (!kLin && s - a.pen.ge >= 0) {
            src(slot_ie, lo_ie, c_ie, b_ie);
            src(slot_de, lo_de, c_de, b_de);
          }
          // second gap piece (kDual): M at s - o2 - e2, I2 / D2 at s - e2
          int lo_mo2 = 0, c_mo2 = 0, b_mo2 = 0, lo_ie2 = 0, c_ie2 = 0, b_ie2 = 0, lo_de2 = 0, c_de2 = 0, b_de2 = 0;
          int out_i2 = 0, out_d2 = 0;
          if constexpr (kDual) {
            const int re2 = a.pen.re2;
            q = slm - a.pen.go2;
            if (q < 0) q += rm;
            if (s - a.pen.go2 >= 0) src(q, lo_mo2, c_mo2, b_mo2);
            q = sli2 - a.pen.ge2;
            if (q < 0) q += re2;
            if (s - a.pen.ge2 >= 0) {
              src(rm + 2 * re + q, lo_ie2, c_ie2, b_ie2);
              src(rm + 2 * re + re2 + q, lo_de2, c_de2, b_de2);
            }
            out_i2 = rm + 2 * re + sli2;
            out_d2 = rm + 2 * re + re2 + sli2;
          }
          const int out_m = slm, out_i = rm + sli, out_d = rm + re + sli;
          if ((c_mm | c_mo | c_ie | c_de | c_mo2 | c_ie2 | c_de2) == 0) {  // null step (wfa_gpu.cu:417-422)
            group_sync<GW>(gid);  // everyone has read the slot limits
            s_lo[out_m] = 1; s_hi[out_m] = 0;
            if constexpr (!kLin) {
              s_lo[out_i] = 1; s_hi[out_i] = 0;
              s_lo[out_d] = 1; s_hi[out_d] = 0;
            }
            if constexpr (kDual) {
              s_lo[out_i2] = 1; s_hi[out_i2] = 0;
              s_lo[out_d2] = 1; s_hi[out_d2] = 0;
            }
            if constexpr (GW == 1) __syncwarp();
            return;
          }
          int lo = INT_MAX, hi = INT_MIN;  // envelope of the sources (wfa_gpu.cu:429-439)
          if (c_mm) { lo = lo_mm; hi = lo_mm + c_mm - 1; }
          if (c_mo) { lo = min(lo, lo_mo - 1); hi = max(hi, lo_mo + c_mo); }
          if (c_ie) { lo = min(lo, lo_ie + 1); hi = max(hi, lo_ie + c_ie); }
          if (c_de) { lo = min(lo, lo_de - 1); hi = max(hi, lo_de + c_de - 2); }
          if constexpr (kDual) {
            if (c_mo2) { lo = min(lo, lo_mo2 - 1); hi = max(hi, lo_mo2 + c_mo2); }
            if (c_ie2) { lo = min(lo, lo_ie2 + 1); hi = max(hi, lo_ie2 + c_ie2); }
            if (c_de2) { lo = min(lo, lo_de2 - 1); hi = max(hi, lo_de2 + c_de2 - 2); }
          }
          const int width = hi - lo + 1;
          const bool i_present = !kLin && (c_mo || c_ie);
          const bool d_present = !kLin && (c_mo || c_de);
          const bool i2_present = kDual && (c_mo2 || c_ie2);
          const bool d2_present = kDual && (c_mo2 || c_de2);
          if (width > W || (kH && (s >= a.table_cap || hbase + width > a.hist_cap))) {
            st = kPairScratch;
            return;
          }
          const int w_m = out_m * W - lo, w_i = out_i * W - lo, w_d = out_d * W - lo;
          const int w_i2 = out_i2 * W - lo, w_d2 = out_d2 * W - lo;
          uint32_t* hrow = kH ? hist + hbase - lo : nullptr;
          int fm = INT_MAX, lm = INT_MIN, fi = INT_MAX, li = INT_MIN, fd = INT_MAX, ld = INT_MIN;
          int fi2 = INT_MAX, li2 = INT_MIN, fd2 = INT_MAX, ld2 = INT_MIN;
          int fk = INT_MAX;  // lowest ending diagonal of this thread
          // Where every one-piece source is present, the diagonals kA..kB
          // read all of them inside their trimmed ranges; a warp whose block
          // of 32 diagonals (k - lane .. + 31, the same for all its lanes)
          // lies there reads without range tests.
          int kA = INT_MAX, kB = INT_MIN;
          if (kWide && !kDual && c_mm && c_mo && (kLin || (c_ie && c_de))) {
            kA = max(lo_mm, lo_mo + 1);
            kB = min(lo_mm + c_mm - 1, lo_mo + c_mo - 2);
            if constexpr (!kLin) {
              kA = max(kA, max(lo_ie + 1, lo_de - 1));
              kB = min(kB, min(lo_ie + c_ie, lo_de + c_de - 2));
            }
            kB -= 31;  // block start bound
          }
          for (int k = lo + gt; k <= hi; k += GT) {
            int32_t ins_o, ins_e = NUL, del_o, del_e = NUL, mis;
            const int kb = k - lane;
            if (kWide && kb >= kA && kb <= kB) {
              ins_o = ring[b_mo - 1 - lo_mo + k];
              del_o = ring[b_mo + 1 - lo_mo + k];
              mis = (int32_t)ring[b_mm - lo_mm + k] + 1;
              if constexpr (!kLin) {
                ins_e = ring[b_ie - 1 - lo_ie + k];
                del_e = ring[b_de + 1 - lo_de + k];
              }
            } else {
              int j;
              j = k - 1 - lo_mo;
              ins_o = ((unsigned)j < (unsigned)c_mo) ? (int32_t)ring[b_mo + j] : NUL;
              j = k + 1 - lo_mo;
              del_o = ((unsigned)j < (unsigned)c_mo) ? (int32_t)ring[b_mo + j] : NUL;
              j = k - lo_mm;
              mis = (((unsigned)j < (unsigned)c_mm) ? (int32_t)ring[b_mm + j] : NUL) + 1;
              if constexpr (!kLin) {
                j = k - 1 - lo_ie;
                ins_e = ((unsigned)j < (unsigned)c_ie) ? (int32_t)ring[b_ie + j] : NUL;
                j = k + 1 - lo_de;
                del_e = ((unsigned)j < (unsigned)c_de) ? (int32_t)ring[b_de + j] : NUL;
              }
            }
            int j;
            const int32_t ins = max(ins_o, ins_e) + 1;
            const int32_t del = max(del_o, del_e);
            int32_t ins2 = NUL, del2 = NUL;
            uint32_t bits;
            int32_t p;
            if constexpr (kDual) {
              j = k - 1 - lo_mo2;
              const int32_t ins2_o = ((unsigned)j < (unsigned)c_mo2) ? (int32_t)ring[b_mo2 + j] : NUL;
              j = k - 1 - lo_ie2;
              const int32_t ins2_e = ((unsigned)j < (unsigned)c_ie2) ? (int32_t)ring[b_ie2 + j] : NUL;
              j = k + 1 - lo_mo2;
              const int32_t del2_o = ((unsigned)j < (unsigned)c_mo2) ? (int32_t)ring[b_mo2 + j] : NUL;
              j = k + 1 - lo_de2;
              const int32_t del2_e = ((unsigned)j < (unsigned)c_de2) ? (int32_t)ring[b_de2 + j] : NUL;
              ins2 = max(ins2_o, ins2_e) + 1;
              del2 = max(del2_o, del2_e);
              // M = max(mismatch, D2, D1, I2, I1), ties in that order
              // (piggyback codes 9 > 8,7 > 6,5 > 4,3 > 2,1)
              p = ins;
              bits = kSrcIns;
              if (ins2 >= p) { p = ins2; bits = kSrcIns2; }
              if (del >= p) { p = del; bits = kSrcDel; }
              if (del2 >= p) { p = del2; bits = kSrcDel2; }
              if (mis >= p) { p = mis; bits = kSrcMis; }
              if (ins_e >= ins_o) bits |= kI1Ext2;
              if (del_e >= del_o) bits |= kD1Ext2;
              if (ins2_e >= ins2_o) bits |= kI2Ext2;
              if (del2_e >= del2_o) bits |= kD2Ext2;
            } else {
              // M = max(D, mismatch, I); ties: mismatch > D > I (piggyback order)
              p = ins;
              bits = kSrcIns;
              if (del >= p) { p = del; bits = kSrcDel; }
              if (mis >= p) { p = mis; bits = kSrcMis; }
              if constexpr (!kLin) {
                if (ins_e >= ins_o) bits |= kIExt;
                if (del_e >= del_o) bits |= kDExt;
              }
            }
            int32_t om = NUL;
            if constexpr (kWide) {
              // Extend M (wfa_gpu.cu:257-287) without a divergent region
              // around it: every lane compares its first 16-base window (an
              // invalid cell at position 0, a valid one at v <= m and h <= n:
              // both inside the staged words and their padding word), and
              // only lanes whose window matches entirely continue in a loop.
              const bool vm = in_bounds_sel(p, k, m, n);
              const int vv = vm ? p - k : 0, hh = vm ? p : 0;
              const int rem = vm ? min(m - vv, n - p) : 0;
              int lx;
              if (kMode == kModeGlobal && bytemode) {
                lx = lcp8(pb, m, vv, tb, n, hh, rem);
              } else {
                const uint32_t d0 = win16(P, vv) ^ win16(T, hh);
                lx = d0 ? (__ffs(d0) - 1) >> 1 : 16;
                if (!d0 && rem > 16) lx = 16 + lcp16(P, vv + 16, T, hh + 16, rem - 16);
                lx = min(lx, rem);
              }
              om = vm ? p + lx : NUL;
              n_ext += (uint32_t)lx;
              fm = vm ? min(fm, k) : fm;
              lm = vm ? k : lm;
              if (ends_free) {
                bool ends = vm & (om >= n) & (k <= k_hi);
                if (free_te) ends |= vm & ((om - k) >= m) & (om >= n_te);
                fk = ends ? min(fk, k) : fk;
              }
            } else if (in_bounds(p, k, m, n)) {
              const int vv = p - k;
              const int rem = min(m - vv, n - p);
              const int lx = (kMode == kModeGlobal && bytemode) ? lcp8(pb, m, vv, tb, n, p, rem) : lcp16(P, vv, T, p, rem);
              om = p + lx;
              n_ext += (uint32_t)lx;
              fm = min(fm, k);
              lm = k;
              if (ends_free) {
                bool ends = (om >= n) & (k <= k_hi);
                if (free_te) ends |= ((om - k) >= m) & (om >= n_te);
                if (ends) fk = min(fk, k);
              }
            }
            store_md(w_m + k, om);
            if (i_present) {
              store_i(w_i + k, ins);
              if constexpr (kWide) {
                const bool vi = in_bounds_sel(ins, k, m, n);
                fi = vi ? min(fi, k) : fi;
                li = vi ? k : li;
              } else if (in_bounds(ins, k, m, n)) {
                fi = min(fi, k);
                li = k;
              }
            }
            if (d_present) {
              store_md(w_d + k, del);
              if constexpr (kWide) {
                const bool vd = in_bounds_sel(del, k, m, n);
                fd = vd ? min(fd, k) : fd;
                ld = vd ? k : ld;
              } else if (in_bounds(del, k, m, n)) {
                fd = min(fd, k);
                ld = k;
              }
            }
            if constexpr (kDual) {
              if (i2_present) {
                store_i(w_i2 + k, ins2);
                const bool vi2 = in_bounds_sel(ins2, k, m, n);
                fi2 = vi2 ? min(fi2, k) : fi2;
                li2 = vi2 ? k : li2;
              }
              if (d2_present) {
                store_md(w_d2 + k, del2);
                const bool vd2 = in_bounds_sel(del2, k, m, n);
                fd2 = vd2 ? min(fd2, k) : fd2;
                ld2 = vd2 ? k : ld2;
              }
            }
            if constexpr (kH) hrow[k] = ((uint32_t)p << (kDual ? 8 : 4)) | bits;
          }
          if (!ends_free && k_end >= lo && k_end <= hi && ((k_end - lo) & (GT - 1)) == gt &&
              (int32_t)ring[w_m + k_end] >= n)
            fk = k_end;
          fm = __reduce_min_sync(FULL, fm);
          lm = __reduce_max_sync(FULL, lm);
          fi = __reduce_min_sync(FULL, fi);
          li = __reduce_max_sync(FULL, li);
          fd = __reduce_min_sync(FULL, fd);
          ld = __reduce_max_sync(FULL, ld);
          fk = __reduce_min_sync(FULL, fk);
          if constexpr (kDual) {
            fi2 = __reduce_min_sync(FULL, fi2);
            li2 = __reduce_max_sync(FULL, li2);
            fd2 = __reduce_min_sync(FULL, fd2);
            ld2 = __reduce_max_sync(FULL, ld2);
          }
          if constexpr (GW > 1) {
            int* pp = part + ((s & 1) * GW + wig) * PW;
            if (lane == 0) {
              pp[0] = fm; pp[1] = lm; pp[2] = fi; pp[3] = li; pp[4] = fd; pp[5] = ld; pp[6] = fk;
              if constexpr (kDual) {
                pp[7] = fi2; pp[8] = li2; pp[9] = fd2; pp[10] = ld2;
              }
            }
            group_sync<GW>(gid);  // the step's ring writes and partials are complete
            // lane w takes warp w's partials; warp reductions combine them
            // (7 loads and 7 reductions per thread instead of 7 * GW)
            int p0 = INT_MAX, p1 = INT_MIN, p2 = INT_MAX, p3 = INT_MIN, p4 = INT_MAX, p5 = INT_MIN, p6 = INT_MAX;
            int p7 = INT_MAX, p8 = INT_MIN, p9 = INT_MAX, p10 = INT_MIN;
            if (lane < GW) {
              const int* qw = part + ((s & 1) * GW + lane) * PW;
              p0 = qw[0]; p1 = qw[1]; p2 = qw[2]; p3 = qw[3]; p4 = qw[4]; p5 = qw[5]; p6 = qw[6];
              if constexpr (kDual) {
                p7 = qw[7]; p8 = qw[8]; p9 = qw[9]; p10 = qw[10];
              }
            }
            fm = __reduce_min_sync(FULL, p0);
            lm = __reduce_max_sync(FULL, p1);
            fi = __reduce_min_sync(FULL, p2);
            li = __reduce_max_sync(FULL, p3);
            fd = __reduce_min_sync(FULL, p4);
            ld = __reduce_max_sync(FULL, p5);
            fk = __reduce_min_sync(FULL, p6);
            if constexpr (kDual) {
              fi2 = __reduce_min_sync(FULL, p7);
              li2 = __reduce_max_sync(FULL, p8);
              fd2 = __reduce_min_sync(FULL, p9);
              ld2 = __reduce_max_sync(FULL, p10);
            }
          }
          {
            // trimmed limits (wfa_gpu.cu:636-719), written by every thread
            // (identical values); no in-bounds cell (first > last) stores the
            // empty range (1, 0)
            const bool em = fm > lm, ei = !i_present || fi > li, ed = !d_present || fd > ld;
            s_lo[out_m] = em ? 1 : fm; s_hi[out_m] = em ? 0 : lm; s_alo[out_m] = lo;
            if constexpr (!kLin) {
              s_lo[out_i] = ei ? 1 : fi; s_hi[out_i] = ei ? 0 : li; s_alo[out_i] = lo;
              s_lo[out_d] = ed ? 1 : fd; s_hi[out_d] = ed ? 0 : ld; s_alo[out_d] = lo;
            }
            if constexpr (kDual) {
              const bool ei2 = !i2_present || fi2 > li2, ed2 = !d2_present || fd2 > ld2;
              s_lo[out_i2] = ei2 ? 1 : fi2; s_hi[out_i2] = ei2 ? 0 : li2; s_alo[out_i2] = lo;
              s_lo[out_d2] = ed2 ? 1 : fd2; s_hi[out_d2] = ed2 ? 0 : ld2; s_alo[out_d2] = lo;
            }
            if (kH && gt == 0) table[s] = make_int2(lo, (int)hbase);
          }
          if constexpr (kH) hbase += width;
          n_cells += (unsigned long long)width;
          ++n_steps;
          if constexpr (GW == 1) __syncwarp();
          if (detect && fk != INT_MAX) {
            s_end = s;
            k_fin = fk;
          }
      };

      // Low-memory mode (a.ckpt_k = K > 0, CIGAR kernels): the score pass
      // keeps no history; it saves the ring every K scores (each slot's
      // limits and trimmed values) in the group's checkpoint area.  The
      // backtrace then takes the segments (jK, (j+1)K] from the last to the
      // first: restore checkpoint j, recompute the segment with history, walk
      // down to score jK.  The recomputed words are the ones the full pass
      // writes, so the CIGAR is the same.
      uint8_t* const ck = lowmem ? a.ckpt + ggroup * a.ckpt_stride : nullptr;
      (void)ck;
      auto save_ckpt = [&](int jc) {
        if (jc >= a.ckpt_cap) {
          st = kPairScratch;
          return;
        }
        uint8_t* base = ck + (int64_t)jc * a.ckpt_bytes;
        int* lim = reinterpret_cast<int*>(base);
        RT* val = reinterpret_cast<RT*>(base + 12 * ns);
        for (int i = gt; i < ns; i += GT) {
          lim[i] = s_lo[i];
          lim[ns + i] = s_hi[i];
          lim[2 * ns + i] = s_alo[i];
        }
        for (int sl = 0; sl < ns; ++sl) {
          const int l = s_lo[sl], h = s_hi[sl];
          const int b = sl * W - s_alo[sl];
          for (int k = l + gt; k <= h; k += GT) val[b + k] = ring[b + k];
        }
        group_sync<GW>(gid);  // copied before the next step overwrites the ring
      };
      auto restore_ckpt = [&](int jc) {
        const uint8_t* base = ck + (int64_t)jc * a.ckpt_bytes;
        const int* lim = reinterpret_cast<const int*>(base);
        const RT* val = reinterpret_cast<const RT*>(base + 12 * ns);
        group_sync<GW>(gid);  // the previous segment is done with the ring and limits
        for (int i = gt; i < ns; i += GT) {
          s_lo[i] = lim[i];
          s_hi[i] = lim[ns + i];
          s_alo[i] = lim[2 * ns + i];
        }
        for (int sl = 0; sl < ns; ++sl) {
          const int l = lim[sl], h = lim[ns + sl];
          const int b = sl * W - lim[2 * ns + sl];
          for (int k = l + gt; k <= h; k += GT) ring[b + k] = val[b + k];
        }
        group_sync<GW>(gid);
      };

      if constexpr (lowmem) {
        if (st == kPairOk && s_end < 0) save_ckpt(0);
        while (s_end < 0 && st == kPairOk) {
          step(std::false_type{}, true);
          if (st == kPairOk && s % K == 0) save_ckpt(s / K);
        }
        if (st == kPairOk && s_end >= a.table_cap) st = kPairScratch;
      } else {
        while (s_end < 0 && st == kPairOk) step(std::true_type{}, true);
      }

      if constexpr (lowmem) {
       if (st == kPairOk) {
        // reserve the run bound in the arena, then walk segment by segment
        const int64_t bound = 2 * (int64_t)s_end / a.pen.min_pen() + 3;  // + a free gap at each end
        unsigned long long at = 0;
        if (gt == 0) {
          at = atomicAdd(a.arena_cursor, (unsigned long long)bound);
          bc[2] = ((int64_t)(at + bound) > a.arena_cap) ? kPairArena : kPairOk;
        }
        group_sync<GW>(gid);
        st = bc[2];
        Walk wk;
        if (gt == 0 && st == kPairOk) walk_begin(wk, s_end, k_fin, m, n, a.arena + at + bound, (int)bound);
        for (int jc = s_end > 0 ? (s_end - 1) / K : -1; jc >= 0 && st == kPairOk; --jc) {
          restore_ckpt(jc);
          s = jc * K;
          slm = s % rm;
          if constexpr (!kLin) sli = s % re;
          if constexpr (kDual) sli2 = s % a.pen.re2;
          hbase = 0;
          const int s_stop = min(s + K, s_end);
          while (s < s_stop && st == kPairOk) step(std::true_type{}, false);
          if (st != kPairOk) break;
          group_sync<GW>(gid);  // the segment's backtrace words and step table are written
          if (gt == 0) {
            int r;
            if constexpr (kDual)
              r = walk_run_dual(wk, hist, hbase, table, jc * K, a.pen);
            else
              r = walk_run(wk, hist, hbase, table, jc * K, a.pen.x, a.pen.go, a.pen.ge);
            bc[2] = r ? kPairInternal : kPairOk;
            bc[3] = walk_done(wk) ? 1 : 0;
          }
          group_sync<GW>(gid);
          st = bc[2];
          if (bc[3]) break;
        }
        if (gt == 0 && st == kPairOk) {
          const int r = walk_finish(wk);
          if (r < 0) {
            st = kPairInternal;
          } else {
            lm_len = r;
            lm_pos = (int64_t)(at + bound) - r;
          }
        }
       }
      }
    }

    if (st == kPairOk) {
      if (gt == 0) a.score[pair] = s_end * a.g;
      if (kCigar && lowmem) {
        if (gt == 0) {
          a.cig_pos[pair] = lm_pos;
          a.cig_len[pair] = lm_len;
        }
      } else if (kCigar) {
        // reserve the run bound 2*s/min_pen + 1 in the arena, then walk
        const int min_pen = a.pen.min_pen();
        const int64_t bound = 2 * (int64_t)s_end / min_pen + 3;  // + a free gap at each end
        if (gt == 0) {
          int32_t len = 0;
          int64_t pos = 0;
          const unsigned long long at = atomicAdd(a.arena_cursor, (unsigned long long)bound);
          if ((int64_t)(at + bound) > a.arena_cap) {
            st = kPairArena;
          } else {
            int r;
            if constexpr (kDual)
              r = backtrace_walk_dual(hist, hbase, table, s_end, k_fin, m, n, a.pen, a.arena + at + bound,
                                      (int)bound);
            else
              r = backtrace_walk(hist, hbase, table, s_end, k_fin, m, n, a.pen.x, a.pen.go, a.pen.ge,
                                 a.arena + at + bound, (int)bound);
            if (r < 0) {
              st = kPairInternal;
            } else {
              len = r;
              pos = (int64_t)(at + bound) - r;
            }
          }
          a.cig_pos[pair] = pos;
          a.cig_len[pair] = len;
        }
      }
    }
    if (a.work) {
      const unsigned we = __reduce_add_sync(FULL, n_ext);
      if (lane == 0 && we) atomicAdd(a.work + 2, (unsigned long long)we);
    }
    if (gt == 0) {
      a.status[pair] = st;
      if (st == kPairScratch || st == kPairArena) {
        const unsigned r = atomicAdd(a.retry_count, 1u);
        a.retry[r] = (int32_t)pair;
      }
      if (a.work) {
        atomicAdd(a.work, n_cells);
        atomicAdd(a.work + 1, n_steps);
      }
    }
    group_sync<GW>(gid);  // the group's shared memory is free for the next pair
  }
}

}  // namespace tsu
