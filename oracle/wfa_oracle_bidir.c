/*
 * wfa_oracle_bidir.c -- CPU oracle of a bidirectional (BiWFA-style)
 * gap-affine alignment.  TEST INFRASTRUCTURE ONLY: nothing in the product
 * links it.
 *
 * A C restatement, step for step, of the pure-Python model in
 * oracle/bidir_rule.py (bialign), fast enough for pairs of kilobases; the
 * tests hold the two byte-identical.  What it computes:
 *   - forward wavefronts of a segment (offset = text position h on diagonal
 *     k = h - v, the recurrences of the reference kernel,
 *     wfa_gpu.cu:616-626) that may start inside a gap continued from the
 *     left (offset 0 in I or D at score 0) or be forced to open a gap first
 *     (a seed at score o + e);
 *   - the first breakpoint: for growing totals T, forward and reverse
 *     wavefronts that overlap -- M extension runs intersecting at sf + sr =
 *     T, or I/D cells meeting exactly at sf + sr = T + o -- searched from
 *     the middle score outwards, diagonals in ascending order;
 *   - the recursion on breakpoints down to segments of small score, each
 *     aligned by the plain WFA with its components and the backtrace of
 *     wfa_oracle.c (wf_backtrace; piggyback order M > D_ext > D_open >
 *     I_ext > I_open after the reference's bt_type_t, common.h:67-77).  A
 *     segment that must end in a gap is aligned on the reversed sequences.
 * Parity: every operation string is optimal (tests compare its cost with
 * the Gotoh DP); byte identity is with bidir_rule.bialign, whose pieces are
 * pinned against component-constrained DPs.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "wfa_oracle.h"

#define BNULL (-(1 << 30))
#define PNULL (INT64_MIN / 4)

enum { CM = 0, CMP = 1, CI = 2, CD = 3 };

typedef struct {
  int lo, hi;           /* computed diagonals (lo > hi: none)          */
  int plo[4], phi[4];   /* present cells per component                */
  int32_t* a;           /* 4 x (hi - lo + 1) offsets, BNULL = absent   */
} bwf_t;

typedef struct {
  const char* p;
  const char* t;
  int m, n, x, o, e;
  char start, forced;
  bwf_t* w;
  int count, cap;
} bpass_t;

static int32_t bw_get(const bwf_t* w, int c, int k) {
  if (k < w->lo || k > w->hi) return BNULL;
  return w->a[(size_t)c * (size_t)(w->hi - w->lo + 1) + (size_t)(k - w->lo)];
}

static int32_t bget(const bpass_t* bp, int s, int c, int k) {
  if (s < 0 || s >= bp->count) return BNULL;
  return bw_get(&bp->w[s], c, k);
}

static int inb(const bpass_t* bp, int32_t off, int k) {
  return off >= 0 && off <= bp->n && off - k >= 0 && off - k <= bp->m;
}

static int32_t ext(const bpass_t* bp, int k, int32_t off) {
  int v = off - k;
  while (v < bp->m && off < bp->n && bp->p[v] == bp->t[off]) {
    ++v;
    ++off;
  }
  return off;
}

static int32_t max32(int32_t a, int32_t b) { return a > b ? a : b; }

static void bp_free(bpass_t* bp) {
  for (int s = 0; s < bp->count; ++s) free(bp->w[s].a);
  free(bp->w);
  bp->w = NULL;
  bp->count = bp->cap = 0;
}

static int bw_alloc(bwf_t* w, int lo, int hi) {
  w->lo = lo;
  w->hi = hi;
  for (int c = 0; c < 4; ++c) {
    w->plo[c] = 1;
    w->phi[c] = 0;
  }
  const size_t width = hi >= lo ? (size_t)(hi - lo + 1) : 0;
  w->a = (int32_t*)malloc(4 * (width ? width : 1) * sizeof(int32_t));
  if (!w->a) return ORA_ENOMEM;
  for (size_t i = 0; i < 4 * width; ++i) w->a[i] = BNULL;
  return 0;
}

static void bw_set(bwf_t* w, int c, int k, int32_t v) {
  w->a[(size_t)c * (size_t)(w->hi - w->lo + 1) + (size_t)(k - w->lo)] = v;
  if (w->plo[c] > w->phi[c]) {
    w->plo[c] = w->phi[c] = k;
  } else {
    if (k < w->plo[c]) w->plo[c] = k;
    if (k > w->phi[c]) w->phi[c] = k;
  }
}

/* Compute wavefronts up to score s (inclusive). */
static int bp_upto(bpass_t* bp, int s_need) {
  while (bp->count <= s_need) {
    if (bp->count == bp->cap) {
      const int nc = bp->cap ? 2 * bp->cap : 64;
      bwf_t* nw = (bwf_t*)realloc(bp->w, (size_t)nc * sizeof(bwf_t));
      if (!nw) return ORA_ENOMEM;
      bp->w = nw;
      bp->cap = nc;
    }
    const int s = bp->count;
    bwf_t* w = &bp->w[s];
    const int oe = bp->o + bp->e;
    const int seed_i = bp->forced == 'I' && s == oe && inb(bp, 1, 1);
    const int seed_d = bp->forced == 'D' && s == oe && inb(bp, 0, -1);
    if (s == 0) {
      if (bp->forced == 'M') {
        if (bw_alloc(w, 0, 0)) return ORA_ENOMEM;
        bw_set(w, CMP, 0, 0);
        bw_set(w, CM, 0, ext(bp, 0, 0));
        if (bp->start == 'I') bw_set(w, CI, 0, 0);
        if (bp->start == 'D') bw_set(w, CD, 0, 0);
      } else if (bw_alloc(w, 1, 0)) {
        return ORA_ENOMEM;
      }
      bp->count = 1;
      continue;
    }
    int lo = 1 << 30, hi = -(1 << 30);
    const struct { int s, c; } srcs[4] = {{s - bp->x, CM}, {s - oe, CM}, {s - bp->e, CI}, {s - bp->e, CD}};
    for (int i = 0; i < 4; ++i) {
      if (srcs[i].s < 0) continue;
      const bwf_t* sw = &bp->w[srcs[i].s];
      const int c = srcs[i].c;
      if (sw->plo[c] > sw->phi[c]) continue;
      if (sw->plo[c] - 1 < lo) lo = sw->plo[c] - 1;
      if (sw->phi[c] + 1 > hi) hi = sw->phi[c] + 1;
    }
    if (seed_i) {
      if (1 < lo) lo = 1;
      if (1 > hi) hi = 1;
    }
    if (seed_d) {
      if (-1 < lo) lo = -1;
      if (-1 > hi) hi = -1;
    }
    if (lo > hi) {
      lo = 1;
      hi = 0;
    }
    if (bw_alloc(w, lo, hi)) return ORA_ENOMEM;
    bp->count = s + 1; /* this wavefront's own reads see only earlier scores */
    for (int k = lo; k <= hi; ++k) {
      int32_t ins = max32(bget(bp, s - oe, CM, k - 1), bget(bp, s - bp->e, CI, k - 1)) + 1;
      if (seed_i && k == 1) ins = max32(ins, 1);
      int32_t del = max32(bget(bp, s - oe, CM, k + 1), bget(bp, s - bp->e, CD, k + 1));
      if (seed_d && k == -1) del = max32(del, 0);
      const int32_t mis = bget(bp, s - bp->x, CM, k) + 1;
      if (inb(bp, ins, k)) bw_set(w, CI, k, ins);
      if (inb(bp, del, k)) bw_set(w, CD, k, del);
      const int32_t pv = max32(mis, max32(ins, del));
      if (inb(bp, pv, k)) {
        bw_set(w, CMP, k, pv);
        bw_set(w, CM, k, ext(bp, k, pv));
      }
    }
  }
  return 0;
}

static void rev_copy(const char* s, int len, char* out) {
  for (int i = 0; i < len; ++i) out[i] = s[len - 1 - i];
}

/* ---- plain WFA of a segment with components, and its backtrace ---------- */

static int64_t bsrc(const bpass_t* bp, int s, int c, int k, int delta, int code) {
  const int32_t v = bget(bp, s, c, k);
  if (v == BNULL) return PNULL;
  return (int64_t)(v + delta) * 16 + code;
}

static int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }

/* Operations of (p, t) forward from start/forced, ended in M or (free_end
 * I/D) in that gap at a discount of o; written in order to ops[0..len). */
static int wfa_forward(const char* p, int m, const char* t, int n, int x, int o, int e, char start, char forced,
                       char free_end, char* ops, int* len, int* cost) {
  bpass_t bp = {p, t, m, n, x, o, e, start, forced, NULL, 0, 0};
  const int k_end = n - m;
  const int mx = x > o + e ? x : o + e;
  const int smax = (m + n) * mx + 2 * (o + e);
  int have = 0, best_cost = 0, s_end = 0;
  char state = 'M';
  int rc = 0;
  for (int s = 0; s <= smax; ++s) {
    if (have && s - (free_end != 'M' ? o : 0) > best_cost) break;
    if ((rc = bp_upto(&bp, s))) goto out;
    if (bget(&bp, s, CM, k_end) >= n && (!have || s < best_cost)) {
      have = 1;
      best_cost = s;
      s_end = s;
      state = 'M';
    }
    if (free_end == 'I' || free_end == 'D') {
      const int32_t g = bget(&bp, s, free_end == 'I' ? CI : CD, k_end);
      if (g == n && (!have || s - o < best_cost)) {
        have = 1;
        best_cost = s - o;
        s_end = s;
        state = free_end;
      }
    }
  }
  if (!have) {
    rc = ORA_EINVAL;
    goto out;
  }
  if (cost) *cost = best_cost;
  {
    /* operations backwards into ops[cap-1 ...] */
    const int cap = m + n + 1;
    char* buf = (char*)malloc((size_t)cap);
    if (!buf) {
      rc = ORA_ENOMEM;
      goto out;
    }
    int pos = cap - 1;
#define BEMIT(ch)           \
  do {                      \
    if (pos < 0) {          \
      free(buf);            \
      rc = ORA_ECIGCAP;     \
      goto out;             \
    }                       \
    buf[pos--] = (ch);      \
  } while (0)
    int s = s_end, k = k_end;
    int32_t off = bget(&bp, s_end, state == 'M' ? CM : (state == 'I' ? CI : CD), k_end);
    int v = off - k, h = off;
    while (v > 0 && h > 0 && s > 0) {
      int64_t io = bsrc(&bp, s - o - e, CM, k - 1, 1, 1);
      const int64_t ix = bsrc(&bp, s - e, CI, k - 1, 1, 2);
      int64_t dop = bsrc(&bp, s - o - e, CM, k + 1, 0, 5);
      const int64_t dx = bsrc(&bp, s - e, CD, k + 1, 0, 6);
      /* a forced first gap opens from the empty origin */
      if (forced == 'I' && s == o + e && k == 1) io = max64(io, 1 * 16 + 1);
      if (forced == 'D' && s == o + e && k == -1) dop = max64(dop, 0 * 16 + 5);
      int64_t best;
      if (state == 'M')
        best = max64(bsrc(&bp, s - x, CM, k, 1, 9), max64(max64(io, ix), max64(dop, dx)));
      else if (state == 'I')
        best = max64(io, ix);
      else
        best = max64(dop, dx);
      if (best < 0) {
        free(buf);
        rc = ORA_EINVAL;
        goto out;
      }
      if (state == 'M') {
        const int32_t moff = (int32_t)(best / 16);
        for (int32_t i = moff; i < off; ++i) BEMIT('M');
        off = moff;
        v = off - k;
        h = off;
        if (v <= 0 || h <= 0) break;
      }
      switch ((int)(best % 16)) {
        case 9: s -= x; state = 'M'; BEMIT('X'); off--; break;
        case 1: s -= o + e; state = 'M'; BEMIT('I'); k--; off--; break;
        case 2: s -= e; state = 'I'; BEMIT('I'); k--; off--; break;
        case 5: s -= o + e; state = 'M'; BEMIT('D'); k++; break;
        default: s -= e; state = 'D'; BEMIT('D'); k++; break;
      }
      v = off - k;
      h = off;
    }
    if (v > 0 && h > 0) {
      const int nm = v < h ? v : h;
      for (int i = 0; i < nm; ++i) BEMIT('M');
      v -= nm;
      h -= nm;
    }
    while (v > 0) { BEMIT('D'); --v; }
    while (h > 0) { BEMIT('I'); --h; }
#undef BEMIT
    *len = cap - 1 - pos;
    memcpy(ops, buf + pos + 1, (size_t)*len);
    free(buf);
  }
out:
  bp_free(&bp);
  return rc;
}

static int wfa_segment(const char* p, int m, const char* t, int n, int x, int o, int e, char begin, char end,
                       char* ops, int* len, int* cost) {
  if (m == 0 && n == 0) {
    *len = 0;
    if (cost) *cost = 0;
    return 0;
  }
  if (end == 'M') return wfa_forward(p, m, t, n, x, o, e, begin, 'M', 'M', ops, len, cost);
  char* rp = (char*)malloc((size_t)m + 1);
  char* rt = (char*)malloc((size_t)n + 1);
  if (!rp || !rt) {
    free(rp);
    free(rt);
    return ORA_ENOMEM;
  }
  rev_copy(p, m, rp);
  rev_copy(t, n, rt);
  int rc = wfa_forward(rp, m, rt, n, x, o, e, 'M', end, begin, ops, len, cost);
  free(rp);
  free(rt);
  if (rc) return rc;
  for (int i = 0, j = *len - 1; i < j; ++i, --j) {
    const char c = ops[i];
    ops[i] = ops[j];
    ops[j] = c;
  }
  return 0;
}

/* ---- breakpoint search ---------------------------------------------------- */

/* sf values 0..hi ordered by |2 sf - mid2|, then sf (middle first). */
static void mid_order(int* out, int hi, int mid2) {
  int cnt = 0;
  const int dmax = mid2 > 2 * hi - mid2 ? mid2 : 2 * hi - mid2;
  for (int d = 0; d <= dmax && cnt <= hi; ++d) {
    if (((mid2 - d) & 1) == 0) {
      const int a = (mid2 - d) / 2;
      if (a >= 0 && a <= hi) out[cnt++] = a;
    }
    if (d > 0 && ((mid2 + d) & 1) == 0) {
      const int a = (mid2 + d) / 2;
      if (a >= 0 && a <= hi) out[cnt++] = a;
    }
  }
}

/* First breakpoint of a segment: *T, component ('M','I','D'), diagonal k
 * and cut offset h.  Returns 1 if found, 0 if not, < 0 on error. */
static int first_breakpoint(const char* p, int m, const char* t, int n, int x, int o, int e, char begin, char end,
                            int* T_out, char* comp, int* k_out, int* h_out) {
  const int mx = x > o + e ? x : o + e;
  const int smax = (m > n ? m : n) * mx + o + e + 2;
  char* rp = (char*)malloc((size_t)m + 1);
  char* rt = (char*)malloc((size_t)n + 1);
  int* order = (int*)malloc(sizeof(int) * (size_t)(smax + 1));
  bpass_t F = {p, t, m, n, x, o, e, begin, 'M', NULL, 0, 0};
  bpass_t R = {NULL, NULL, m, n, x, o, e, 'M', end, NULL, 0, 0};
  int found = 0, rc = 0;
  if (!rp || !rt || !order) {
    rc = ORA_ENOMEM;
    goto out;
  }
  rev_copy(p, m, rp);
  rev_copy(t, n, rt);
  R.p = rp;
  R.t = rt;
  for (int T = 0; T <= 2 * smax && !found; ++T) {
    const int hi1 = T < smax ? T : smax;
    if ((rc = bp_upto(&F, hi1)) || (rc = bp_upto(&R, hi1))) goto out;
    mid_order(order, hi1, T);
    for (int i = 0; i <= hi1 && !found; ++i) {
      const int sf = order[i], sr = T - sf;
      if (sr > smax) continue;
      const bwf_t* fw = &F.w[sf];
      for (int k = fw->plo[CM]; k <= fw->phi[CM] && fw->plo[CM] <= fw->phi[CM]; ++k) {
        const int32_t hf = bw_get(fw, CM, k);
        if (hf == BNULL) continue;
        const int kr = (n - m) - k;
        const int32_t rm = bget(&R, sr, CM, kr);
        if (rm == BNULL) continue;
        const int32_t fmp = bw_get(fw, CMP, k), rmp = bget(&R, sr, CMP, kr);
        const int32_t lo = fmp > n - rm ? fmp : n - rm;
        const int32_t hi = hf < n - rmp ? hf : n - rmp;
        if (lo <= hi) {
          *T_out = T;
          *comp = 'M';
          *k_out = k;
          *h_out = lo;
          found = 1;
          break;
        }
      }
    }
    if (found) break;
    const int hi2 = T + o < smax ? T + o : smax;
    if ((rc = bp_upto(&F, hi2)) || (rc = bp_upto(&R, hi2))) goto out;
    mid_order(order, hi2, T + o);
    for (int i = 0; i <= hi2 && !found; ++i) {
      const int sf = order[i], sr = T + o - sf;
      if (sr > smax || sr < 0) continue;
      const bwf_t* fw = &F.w[sf];
      for (int ci = 0; ci < 2 && !found; ++ci) {
        const int c = ci == 0 ? CI : CD;
        for (int k = fw->plo[c]; k <= fw->phi[c] && fw->plo[c] <= fw->phi[c]; ++k) {
          const int32_t hf = bw_get(fw, c, k);
          if (hf == BNULL) continue;
          const int32_t rg = bget(&R, sr, c, (n - m) - k);
          if (rg != BNULL && hf + rg == n) {
            *T_out = T;
            *comp = c == CI ? 'I' : 'D';
            *k_out = k;
            *h_out = hf;
            found = 1;
            break;
          }
        }
      }
    }
  }
out:
  bp_free(&F);
  bp_free(&R);
  free(rp);
  free(rt);
  free(order);
  return rc ? rc : found;
}

/* The two-ring search: forward and reverse advance in turns (the lower
 * score first, forward on ties); each new wavefront is checked against the
 * other side's last max(x, o+e) + 1 scores for offsets crossing on a
 * diagonal (forward + reverse >= n; gaps count one opening), components M,
 * I, D in turn, diagonals ascending, the strictly lowest total kept.  An M
 * crossing is cut at max(forward pre-extension offset, n - reverse
 * offset), a gap crossing at the forward gap cell (bidir_rule.py
 * _crossing_search). */
typedef struct {
  int have, T, k, h;
  char comp;
} bcut_t;

static void cross_check(const bpass_t* F, const bpass_t* R, int sf, int sr, int n, int m, int o, bcut_t* best) {
  const bwf_t* fw = &F->w[sf];
  static const int comps[3] = {CM, CI, CD};
  for (int ci = 0; ci < 3; ++ci) {
    const int c = comps[ci];
    if (fw->plo[c] > fw->phi[c]) continue;
    for (int k = fw->plo[c]; k <= fw->phi[c]; ++k) {
      const int32_t hf = bw_get(fw, c, k);
      if (hf == BNULL) continue;
      const int32_t hr = bget(R, sr, c, (n - m) - k);
      if (hr == BNULL || hf + hr < n) continue;
      const int total = sf + sr - (c == CM ? 0 : o);
      if (best->have && total >= best->T) continue;
      best->have = 1;
      best->T = total;
      best->k = k;
      best->comp = c == CM ? 'M' : (c == CI ? 'I' : 'D');
      if (c == CM) {
        const int32_t pre = bw_get(fw, CMP, k);
        best->h = pre > n - hr ? pre : n - hr;
      } else {
        best->h = hf;
      }
    }
  }
}

static int crossing_breakpoint(const char* p, int m, const char* t, int n, int x, int o, int e, char begin,
                               char end, int* T_out, char* comp, int* k_out, int* h_out) {
  const int mx = x > o + e ? x : o + e;
  const int smax = (m + n) * mx + 2 * (o + e) + 2;
  char* rp = (char*)malloc((size_t)m + 1);
  char* rt = (char*)malloc((size_t)n + 1);
  bpass_t F = {p, t, m, n, x, o, e, begin, 'M', NULL, 0, 0};
  bpass_t R = {NULL, NULL, m, n, x, o, e, 'M', end, NULL, 0, 0};
  bcut_t best = {0, 0, 0, 0, 'M'};
  int rc = 0;
  if (!rp || !rt) {
    rc = ORA_ENOMEM;
    goto out;
  }
  rev_copy(p, m, rp);
  rev_copy(t, n, rt);
  R.p = rp;
  R.t = rt;
  if ((rc = bp_upto(&F, 0)) || (rc = bp_upto(&R, 0))) goto out;
  cross_check(&F, &R, 0, 0, n, m, o, &best);
  int sf = 0, sr = 0;
  while (sf <= smax) {
    if (best.have && sf + sr - 2 * mx - o > best.T) break;
    if (sf <= sr) {
      ++sf;
      if ((rc = bp_upto(&F, sf))) goto out;
      for (int s2 = sr - mx > 0 ? sr - mx : 0; s2 <= sr; ++s2) cross_check(&F, &R, sf, s2, n, m, o, &best);
    } else {
      ++sr;
      if ((rc = bp_upto(&R, sr))) goto out;
      for (int s1 = sf - mx > 0 ? sf - mx : 0; s1 <= sf; ++s1) cross_check(&F, &R, s1, sr, n, m, o, &best);
    }
  }
  if (best.have) {
    *T_out = best.T;
    *comp = best.comp;
    *k_out = best.k;
    *h_out = best.h;
  }
out:
  bp_free(&F);
  bp_free(&R);
  free(rp);
  free(rt);
  return rc ? rc : best.have;
}

static int bialign_rec(const char* p, int m, const char* t, int n, int x, int o, int e, char begin, char end,
                       int base, int ring, char* ops, int* len) {
  if (m == 0 && n == 0) {
    *len = 0;
    return 0;
  }
  int T = 0, k = 0, h = 0;
  char comp = 'M';
  const int f = ring ? crossing_breakpoint(p, m, t, n, x, o, e, begin, end, &T, &comp, &k, &h)
                    : first_breakpoint(p, m, t, n, x, o, e, begin, end, &T, &comp, &k, &h);
  if (f < 0) return f;
  if (f == 0) return ORA_EINVAL;
  const int v = h - k;
  const int whole = m + n, left = v + h, right = whole - left;
  if (T <= base || left == 0 || left == whole || right == 0 || right == whole)
    return wfa_segment(p, m, t, n, x, o, e, begin, end, ops, len, NULL);
  int l1 = 0, l2 = 0;
  int rc = bialign_rec(p, v, t, h, x, o, e, begin, comp, base, ring, ops, &l1);
  if (rc) return rc;
  rc = bialign_rec(p + v, m - v, t + h, n - h, x, o, e, comp, end, base, ring, ops + l1, &l2);
  if (rc) return rc;
  *len = l1 + l2;
  return 0;
}

int ora_bialign(const char* pattern, int m, const char* text, int n, int x, int o, int e, int base_score,
                char* ops, int ops_cap, int* ops_len) {
  if (!pattern || !text || !ops || !ops_len || m < 0 || n < 0 || x <= 0 || o < 0 || e <= 0) return ORA_EINVAL;
  if (ops_cap < m + n) return ORA_ECIGCAP;
  const int mx = x > o + e ? x : o + e;
  return bialign_rec(pattern, m, text, n, x, o, e, 'M', 'M', base_score > 0 ? base_score : 2 * mx, 0, ops,
                     ops_len);
}

int ora_bialign_ring(const char* pattern, int m, const char* text, int n, int x, int o, int e, int base_score,
                     char* ops, int ops_cap, int* ops_len) {
  if (!pattern || !text || !ops || !ops_len || m < 0 || n < 0 || x <= 0 || o < 0 || e <= 0) return ORA_EINVAL;
  if (ops_cap < m + n) return ORA_ECIGCAP;
  const int mx = x > o + e ? x : o + e;
  return bialign_rec(pattern, m, text, n, x, o, e, 'M', 'M', base_score > 0 ? base_score : 2 * mx, 1, ops,
                     ops_len);
}

int ora_crossing_split(const char* pattern, int m, const char* text, int n, int x, int o, int e, char begin,
                       char end, int* T, char* comp, int* k, int* h) {
  if (!pattern || !text || !T || !comp || !k || !h || m < 0 || n < 0 || x <= 0 || o < 0 || e <= 0) return ORA_EINVAL;
  if (!strchr("MID", begin) || !strchr("MID", end) || !begin || !end) return ORA_EINVAL;
  return crossing_breakpoint(pattern, m, text, n, x, o, e, begin, end, T, comp, k, h);
}

int ora_crossing_split_batch(int64_t num, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                             const int64_t* toff, const int32_t* tlen, const char* begin, const char* end, int x,
                             int o, int e, int32_t* T, char* comp, int32_t* k, int32_t* h) {
  if (num < 0 || !pat || !poff || !plen || !txt || !toff || !tlen || !begin || !end || !T || !comp || !k || !h)
    return ORA_EINVAL;
  int rc = 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < num; ++i) {
    int t_ = 0, k_ = 0, h_ = 0;
    char c_ = 'M';
    const int r = ora_crossing_split(pat + poff[i], plen[i], txt + toff[i], tlen[i], x, o, e, begin[i], end[i], &t_,
                                     &c_, &k_, &h_);
    if (r < 0) {
#pragma omp atomic write
      rc = r;
    }
    T[i] = r == 1 ? t_ : -1;
    comp[i] = c_;
    k[i] = k_;
    h[i] = h_;
  }
  return rc;
}

int ora_align_segment(const char* pattern, int m, const char* text, int n, int x, int o, int e, char begin,
                      char end, char* ops, int ops_cap, int* ops_len) {
  if (!pattern || !text || !ops || !ops_len || m < 0 || n < 0 || x <= 0 || o < 0 || e <= 0) return ORA_EINVAL;
  if (!strchr("MID", begin) || !strchr("MID", end) || !begin || !end) return ORA_EINVAL;
  if (ops_cap < m + n) return ORA_ECIGCAP;
  int cost = 0;
  const int rc = wfa_segment(pattern, m, text, n, x, o, e, begin, end, ops, ops_len, &cost);
  return rc ? rc : cost;
}
