/*
 * ref_kernel_model.c -- a CPU model of the reference's GPU kernel, defects
 * included.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference kernel wfa_dispatcher
 * (wfa_gpu.cu:191-722, with count_chars, wfa_gpu.cu:724-752) is built from
 * its own source by oracle/ref_build.sh and run by oracle/ref_harness.cu to
 * pin this project's scores to the reference itself.  That kernel has no
 * bounds checks on its wavefront slots, reads past the ends of its pairs and
 * has no step limit, so the harness runs it only on inputs this model has
 * certified first:
 *   - every wavefront-ring index stays inside the pair's own ring
 *     (num_wavefronts * wf_length shorts), with the reference's `short`
 *     slot base (wfa_gpu.cu:217,341) reproduced and checked;
 *   - every pattern/text byte read lies inside the caller's padded buffers;
 *   - the score loop ends within step_cap steps.
 * The model executes the kernel's semantics one lane after another, on the
 * same flat buffers (pair i at base + i * seq_len), including:
 *   - extension by 32-character windows with the unguarded first window and
 *     the jump of a whole window when the loop stops on a bound with no
 *     mismatch (wfa_gpu.cu:257-285), then lane 0's byte tail bounded by
 *     pattern_len only (wfa_gpu.cu:272-281);
 *   - the end test on M only (wfa_gpu.cu:288-300);
 *   - the null-step counter (wfa_gpu.cu:246-251,417-423);
 *   - source selection, envelope and the I/D allocation rule
 *     (wfa_gpu.cu:340-468), reading stale ring values when a source's
 *     null flag is set but its score is not negative (wfa_gpu.cu:614-619);
 *   - lane 0's "init ends" that null-pad only every 32nd element, with the
 *     D-source lower bound taken from the I limits (wfa_gpu.cu:470-606);
 *   - M = max(D, M[s-x] + 1, I) with the unguarded M[s-x] read and the
 *     pattern-bound test written as offset - idx + lo (wfa_gpu.cu:610-631);
 *   - the end trimming of M, I and D, which also runs (on stale limits)
 *     for a component that was not allocated this step (wfa_gpu.cu:636-719).
 * maxk[i] (nullable) receives the largest |diagonal| addressed: with
 * wf_length > 2 * (seq_len + 3) no access can leave its slot, and a run with
 * wf_length >= 2 * max(maxk) + 2 addresses the same cells inside each slot.
 * The wavefronts are int16, the limits int16, the score int16, as in the
 * reference.  Limits words the kernel never initialises start at 0 (the
 * harness clears them before the launch).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "wfa_oracle.h"

#define RK_NULL ((int16_t)(INT16_MIN / 2)) /* common.h:6 */
#define RK_LANES 32                        /* wfa_gpu.cu:34 */

typedef struct {
  const char* pat;   /* this pair's pattern (may be read before/after) */
  const char* txt;
  int64_t pat_lo, pat_hi; /* readable byte range relative to pat: [lo, hi) */
  int64_t txt_lo, txt_hi;
  int16_t* M;
  int16_t* I;
  int16_t* D;
  uint8_t* nm;
  uint8_t* ni;
  uint8_t* nd;
  int16_t* lm;
  int16_t* li;
  int16_t* ld;
  int64_t ring; /* num_wavefronts * wf_length */
  int wf;
  int maxk;     /* largest |diagonal| addressed (slot position - wf / 2) */
  int bad;      /* first violation (ORA_REFK_*) */
} rk_pair;

static int rk_ok_ring(rk_pair* p, int64_t idx) {
  if (idx < 0 || idx >= p->ring) {
    if (!p->bad) p->bad = ORA_REFK_RING;
    return 0;
  }
  int k = (int)(idx % p->wf) - p->wf / 2;
  if (k < 0) k = -k;
  if (k > p->maxk) p->maxk = k;
  return 1;
}

static int16_t rk_get(rk_pair* p, const int16_t* w, int64_t idx) { return rk_ok_ring(p, idx) ? w[idx] : RK_NULL; }

static void rk_put(rk_pair* p, int16_t* w, int64_t idx, int v) {
  if (rk_ok_ring(p, idx)) w[idx] = (int16_t)v;
}

static char rk_pc(rk_pair* p, int64_t i) {
  if (i < p->pat_lo || i >= p->pat_hi) {
    if (!p->bad) p->bad = ORA_REFK_SEQ;
    return 0;
  }
  return p->pat[i];
}

static char rk_tc(rk_pair* p, int64_t i) {
  if (i < p->txt_lo || i >= p->txt_hi) {
    if (!p->bad) p->bad = ORA_REFK_SEQ;
    return 1;
  }
  return p->txt[i];
}

/* count_chars (wfa_gpu.cu:724-752): mismatches among 32 characters. */
static int rk_count(rk_pair* p, int64_t v, int64_t h) {
  int d = 0;
  for (int t = 0; t < RK_LANES; ++t) d += rk_pc(p, v + t) != rk_tc(p, h + t);
  return d;
}

static int rk_max(int a, int b) { return a >= b ? a : b; } /* common.h:8 */
static int rk_min(int a, int b) { return a <= b ? a : b; } /* common.h:7 */

/* Lane 0's null padding of one source slot's upper / lower side
 * (wfa_gpu.cu:470-606): k steps by the block size, the write tests k + 0. */
static void rk_pad_hi(rk_pair* p, int16_t* w, int base, int from, int to_incl, int bound_incl) {
  for (int k = from; k <= to_incl; k += RK_LANES)
    if (k <= bound_incl) rk_put(p, w, (int64_t)base + k, RK_NULL);
}
static void rk_pad_lo(rk_pair* p, int16_t* w, int base, int from, int below) {
  for (int k = from; k < below; k += RK_LANES)
    if (k < below) rk_put(p, w, (int64_t)base + k, RK_NULL);
}

/* Trim one component's ends (wfa_gpu.cu:636-719). */
static void rk_trim(rk_pair* p, int16_t* w, int16_t* lim, uint8_t* nul, int mi, int li, int L) {
  int k;
  const int lo0 = lim[li];
  for (k = lim[li + 1]; k >= lo0; --k) {
    const int16_t off = rk_get(p, w, (int64_t)mi + k);
    const uint32_t h = (uint32_t)(int32_t)off, v = (uint32_t)(int32_t)(off - k);
    if (h <= (uint32_t)L && v <= (uint32_t)L) break;
  }
  lim[li + 1] = (int16_t)k;
  lim[li + 3] = (int16_t)k;
  const int hi = lim[li + 1];
  for (k = lim[li]; k <= hi; ++k) {
    const int16_t off = rk_get(p, w, (int64_t)mi + k);
    const uint32_t h = (uint32_t)(int32_t)off, v = (uint32_t)(int32_t)(off - k);
    if (h <= (uint32_t)L && v <= (uint32_t)L) break;
  }
  lim[li] = (int16_t)k;
  lim[li + 2] = (int16_t)k;
  *nul = lim[li] > lim[li + 1];
}

/* One pair: the kernel's loop over s.  Returns the score (>= 0) or a
 * negative ORA_REFK_* code; *steps receives the steps taken. */
static int rk_align(rk_pair* p, int L, int x, int o, int e, int nw, int wf, int step_cap, int* steps) {
  const int max_score = rk_max(o + e, x) + 1;
  for (int64_t i = 0; i < p->ring; ++i) p->M[i] = p->I[i] = p->D[i] = RK_NULL;
  for (int i = 0; i < nw; ++i) p->nm[i] = p->ni[i] = p->nd[i] = 1;
  int s = 0;
  int num_null_steps = 0;
  const int align_k = 0, align_off = L; /* equal lengths: text_len - pattern_len = 0 */
  int32_t mi_full = (s % nw) * wf + wf / 2;
  int16_t mi = (int16_t)mi_full; /* `short matr_idx` (wfa_gpu.cu:217) */
  int li = (s % nw) * 4;
  if (mi != mi_full) return ORA_REFK_RING;
  rk_put(p, p->M, mi, 0);
  p->nm[0] = 0;
  p->lm[0] = 0;
  p->lm[1] = 0;
  *steps = 0;
  for (;;) {
    int finish;
    if (p->nm[s % nw]) {
      finish = num_null_steps > max_score;
    } else {
      for (int k = p->lm[li]; k <= p->lm[li + 1]; ++k) { /* extend, wfa_gpu.cu:257-285 */
        int off = rk_get(p, p->M, (int64_t)mi + k);
        if (off < 0) continue;
        int diffs = rk_count(p, (int64_t)off - k, off);
        while (diffs == 0 && off - k + RK_LANES <= L && off + RK_LANES <= L) {
          off = (int16_t)(off + RK_LANES);
          diffs = rk_count(p, (int64_t)off - k, off);
        }
        int eq = 0;
        if (!diffs) off = (int16_t)(off + RK_LANES);
        if (off - k < L) {
          for (int i = off; i < L; ++i) {
            if (rk_pc(p, (int64_t)i - k) == rk_tc(p, i))
              ++eq;
            else
              break;
          }
        }
        off = (int16_t)(off + eq);
        rk_put(p, p->M, (int64_t)mi + k, off);
        if (p->bad) return p->bad;
      }
      int end = 0; /* wfa_gpu.cu:288-300 */
      if (!(p->lm[li] > align_k || align_k > p->lm[li + 1])) end = rk_get(p, p->M, (int64_t)mi + align_k) >= align_off;
      finish = end;
    }
    if (p->bad) return p->bad;
    if (finish) return (int16_t)s;
    ++s;
    if (s > step_cap) return ORA_REFK_STEPS;
    ++*steps;
    mi_full = (s % nw) * wf + wf / 2;
    mi = (int16_t)mi_full;
    if (mi != mi_full) return ORA_REFK_RING;
    li = (s % nw) * 4;
    p->nm[s % nw] = p->ni[s % nw] = p->nd[s % nw] = 0;
    const int so = s - o - e, sx = s - x, se = s - e;
    /* C's % keeps the sign of a negative score; those bases are used only
     * behind a score >= 0 test, except M[s - x] in the compute loop */
    const int gap_open = (so % nw) * wf + wf / 2, mism = (sx % nw) * wf + wf / 2, gap_ext = (se % nw) * wf + wf / 2;
    const int l_open = (so % nw) * 4, l_mism = (sx % nw) * 4, l_ext = (se % nw) * 4;
    int n_mism, n_open, n_iext, n_dext;
    int lo_mism, hi_mism, lo_open, hi_open, lo_iext, hi_iext, lo_dext, hi_dext;
    if (sx < 0 || p->nm[sx % nw]) {
      n_mism = 1, lo_mism = 1, hi_mism = -1;
    } else {
      n_mism = 0, lo_mism = p->lm[l_mism], hi_mism = p->lm[l_mism + 1];
    }
    if (so < 0 || p->nm[so % nw]) {
      n_open = 1, lo_open = 1, hi_open = -1;
    } else {
      n_open = 0, lo_open = p->lm[l_open], hi_open = p->lm[l_open + 1];
    }
    if (se < 0 || p->ni[se % nw]) {
      n_iext = 1, lo_iext = 1, hi_iext = -1;
    } else {
      n_iext = 0, lo_iext = p->li[l_ext], hi_iext = p->li[l_ext + 1];
    }
    if (se < 0 || p->nd[se % nw]) {
      n_dext = 1, lo_dext = 1, hi_dext = -1;
    } else {
      n_dext = 0, lo_dext = p->ld[l_ext], hi_dext = p->ld[l_ext + 1];
    }
    if (n_mism && n_open && n_iext && n_dext) {
      ++num_null_steps;
      p->nm[s % nw] = p->ni[s % nw] = p->nd[s % nw] = 1;
      continue;
    }
    num_null_steps = 0;
    int lo = lo_mism, hi = hi_mism; /* envelope, wfa_gpu.cu:429-439 */
    if (lo > lo_open - 1 && !n_open) lo = lo_open - 1;
    if (hi < hi_open + 1 && !n_open) hi = hi_open + 1;
    if (lo > lo_iext + 1 && !n_iext) lo = lo_iext + 1;
    if (hi < hi_iext + 1 && !n_iext) hi = hi_iext + 1;
    if (lo > lo_dext - 1 && !n_dext) lo = lo_dext - 1;
    if (hi < hi_dext - 1 && !n_dext) hi = hi_dext - 1;
    p->lm[li] = (int16_t)lo;
    p->lm[li + 1] = (int16_t)hi;
    if (!n_open || !n_iext) {
      p->li[li] = (int16_t)lo;
      p->li[li + 1] = (int16_t)hi;
    } else {
      p->ni[s % nw] = 1;
    }
    if (!n_open || !n_dext) {
      p->ld[li] = (int16_t)lo;
      p->ld[li + 1] = (int16_t)hi;
    } else {
      p->nd[s % nw] = 1;
    }
    /* lane 0's init ends (wfa_gpu.cu:470-606) */
    if (!n_mism) {
      if (!(p->lm[l_mism + 3] >= hi)) {
        rk_pad_hi(p, p->M, mism, rk_max(p->lm[l_mism + 3], p->lm[l_mism + 1]) + 1, hi, hi);
        p->lm[l_mism + 3] = (int16_t)hi;
      }
      if (!(p->lm[l_mism + 2] <= lo)) {
        rk_pad_lo(p, p->M, mism, lo, rk_min(p->lm[l_mism + 2], p->lm[l_mism]));
        p->lm[l_mism + 2] = (int16_t)lo;
      }
    }
    if (!n_open) {
      if (!(p->lm[l_open + 3] >= hi + 1)) {
        rk_pad_hi(p, p->M, gap_open, rk_max(p->lm[l_open + 3], p->lm[l_open + 1]) + 1, hi + 1, hi);
        p->lm[l_open + 3] = (int16_t)(hi + 1);
      }
      if (!(p->lm[l_open + 2] <= lo - 1)) {
        rk_pad_lo(p, p->M, gap_open, lo - 1, rk_min(p->lm[l_open + 2], p->lm[l_open]));
        p->lm[l_open + 2] = (int16_t)(lo - 1);
      }
    }
    if (!n_iext) {
      if (!(p->li[l_ext + 3] >= hi)) {
        rk_pad_hi(p, p->I, gap_ext, rk_max(p->li[l_ext + 3], p->li[l_ext + 1]) + 1, hi, hi);
        p->li[l_ext + 3] = (int16_t)hi;
      }
      if (!(p->li[l_ext + 2] <= lo - 1)) {
        rk_pad_lo(p, p->I, gap_ext, lo - 1, rk_min(p->li[l_ext + 2], p->li[l_ext]));
        p->li[l_ext + 2] = (int16_t)(lo - 1);
      }
    }
    if (!n_dext) {
      if (!(p->ld[l_ext + 3] >= hi + 1)) {
        rk_pad_hi(p, p->D, gap_ext, rk_max(p->ld[l_ext + 3], p->ld[l_ext + 1]) + 1, hi + 1, hi + 1);
        p->ld[l_ext + 3] = (int16_t)(hi + 1);
      }
      if (!(p->ld[l_ext + 2] <= lo)) {
        rk_pad_lo(p, p->D, gap_ext, lo, rk_min(p->ld[l_ext + 2], p->li[l_ext]));
        p->ld[l_ext + 2] = (int16_t)lo;
      }
    }
    if (p->bad) return p->bad;
    /* compute (wfa_gpu.cu:610-631): sources and output slot differ, so lane
     * order does not matter */
    for (int idx = 0; idx <= hi - lo; ++idx) {
      const int k = idx + lo;
      const int ins_o = so < 0 ? RK_NULL : rk_get(p, p->M, (int64_t)gap_open + k - 1);
      const int ins_e = se < 0 ? RK_NULL : rk_get(p, p->I, (int64_t)gap_ext + k - 1);
      rk_put(p, p->I, (int64_t)mi + k, rk_max(ins_o, ins_e) + 1);
      const int del_o = so < 0 ? RK_NULL : rk_get(p, p->M, (int64_t)gap_open + k + 1);
      const int del_e = se < 0 ? RK_NULL : rk_get(p, p->D, (int64_t)gap_ext + k + 1);
      rk_put(p, p->D, (int64_t)mi + k, rk_max(del_o, del_e));
      const int mis = rk_get(p, p->M, (int64_t)mism + k) + 1; /* no s - x >= 0 test */
      const int dv = rk_get(p, p->D, (int64_t)mi + k), iv = rk_get(p, p->I, (int64_t)mi + k);
      rk_put(p, p->M, (int64_t)mi + k, rk_max(dv, rk_max(mis, iv)));
      if (rk_get(p, p->M, (int64_t)mi + k) > L) rk_put(p, p->M, (int64_t)mi + k, RK_NULL);
      if (rk_get(p, p->M, (int64_t)mi + k) - idx + lo > L) rk_put(p, p->M, (int64_t)mi + k, RK_NULL);
    }
    if (p->bad) return p->bad;
    rk_trim(p, p->M, p->lm, &p->nm[s % nw], mi, li, L);
    rk_trim(p, p->I, p->li, &p->ni[s % nw], mi, li, L);
    rk_trim(p, p->D, p->ld, &p->nd[s % nw], mi, li, L);
    if (p->bad) return p->bad;
  }
}

int ora_refk_batch(const char* pat0, const char* txt0, int64_t front, int64_t back, int64_t num, int seq_len, int x,
                   int o, int e, int wf_length, int step_cap, int16_t* scores, int32_t* codes, int32_t* steps,
                   int32_t* maxk) {
  if (!pat0 || !txt0 || num < 0 || seq_len < 0 || x < 0 || o < 0 || e <= 0 || wf_length <= 0 || !scores || !codes)
    return ORA_EINVAL;
  const int nw = rk_max(o + e, x) + 1; /* wfa_gpu.cu:83-84 */
  const int64_t ring = (int64_t)nw * wf_length;
  int rc = 0;
#pragma omp parallel
  {
    int16_t* buf = (int16_t*)malloc(sizeof(int16_t) * (size_t)(3 * ring + 12 * nw));
    uint8_t* flags = (uint8_t*)malloc((size_t)(3 * nw));
    if (!buf || !flags) {
#pragma omp atomic write
      rc = ORA_ENOMEM;
    } else {
#pragma omp for schedule(dynamic, 16)
      for (int64_t i = 0; i < num; ++i) {
        rk_pair p;
        memset(&p, 0, sizeof p);
        p.pat = pat0 + i * (int64_t)seq_len;
        p.txt = txt0 + i * (int64_t)seq_len;
        p.pat_lo = p.txt_lo = -front - i * (int64_t)seq_len;
        p.pat_hi = p.txt_hi = (num - i) * (int64_t)seq_len + back;
        p.M = buf;
        p.I = buf + ring;
        p.D = buf + 2 * ring;
        p.lm = buf + 3 * ring;
        p.li = p.lm + 4 * nw;
        p.ld = p.li + 4 * nw;
        memset(p.lm, 0, sizeof(int16_t) * 12 * (size_t)nw);
        p.nm = flags;
        p.ni = flags + nw;
        p.nd = flags + 2 * nw;
        p.ring = ring;
        p.wf = wf_length;
        int st = 0;
        const int r = rk_align(&p, seq_len, x, o, e, nw, wf_length, step_cap, &st);
        if (r < 0) {
          scores[i] = -1;
          codes[i] = r;
        } else {
          scores[i] = (int16_t)r;
          codes[i] = 0;
        }
        if (steps) steps[i] = st;
        if (maxk) maxk[i] = p.maxk;
      }
    }
    free(buf);
    free(flags);
  }
  return rc;
}
