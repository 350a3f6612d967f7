/*
 * wfa_oracle_linear.c -- CPU oracle for gap-linear end-to-end WaveFront
 * Alignment (edit and indel distance are its special cases).  TEST
 * INFRASTRUCTURE ONLY (see wfa_oracle.h): the parity checker of the engine's
 * gap-linear mode, never used by the product.
 *
 * The model: match 0, mismatch x, each gap base e (a gap of length L costs
 * e*L).  The reference aligns with WFA2-lib's gap_affine metric
 * (wfa_gpu.cu:157-160); WFA2-lib's other distance metrics (indel, edit,
 * gap_linear) have one wavefront component.  Restated from the published WFA
 * algorithm (Marco-Sola et al. 2021):
 *   M[s][k] = max(M[s-x][k] + 1, M[s-e][k-1] + 1, M[s-e][k+1])
 * nullified out of bounds, extended along the diagonal; limits, trimming and
 * null steps as in the gap-affine oracle; the backtrace resolves ties
 * mismatch > deletion > insertion (the reference's piggyback order,
 * common.h:67-77, without the gap-extension codes).  Edit distance is x = e
 * = 1; indel distance is x = 3, e = 1 (a mismatch never beats a deletion
 * plus an insertion).  Scores are pinned by ora_linear_dp_score.
 */
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "wfa_oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define LNULL ((int32_t)(INT32_MIN / 2))

typedef struct {
  int present, lo, hi, alo, ahi;
  int64_t base;
} wfl_t;

typedef struct {
  wfl_t* w;
  int cap_s;
  int32_t* arena;
  int64_t arena_cap, arena_used;
  char* opbuf;
  int opbuf_cap;
} wsl_t;

static int wsl_reserve(wsl_t* ws, int need) {
  if (need <= ws->cap_s) return 0;
  int nc = ws->cap_s ? ws->cap_s : 64;
  while (nc < need) nc *= 2;
  wfl_t* nw = (wfl_t*)realloc(ws->w, sizeof(wfl_t) * (size_t)nc);
  if (!nw) return ORA_ENOMEM;
  memset(nw + ws->cap_s, 0, sizeof(wfl_t) * (size_t)(nc - ws->cap_s));
  ws->w = nw;
  ws->cap_s = nc;
  return 0;
}

static int64_t wsl_alloc(wsl_t* ws, int64_t n) {
  if (ws->arena_used + n > ws->arena_cap) {
    int64_t nc = ws->arena_cap ? ws->arena_cap : 4096;
    while (nc < ws->arena_used + n) nc *= 2;
    int32_t* na = (int32_t*)realloc(ws->arena, sizeof(int32_t) * (size_t)nc);
    if (!na) return -1;
    ws->arena = na;
    ws->arena_cap = nc;
  }
  const int64_t b = ws->arena_used;
  ws->arena_used += n;
  return b;
}

static inline int wl_null(const wfl_t* w) { return !w || !w->present || w->lo > w->hi; }
static inline int32_t wl_get(const wsl_t* ws, const wfl_t* w, int k) {
  if (wl_null(w) || k < w->lo || k > w->hi) return LNULL;
  return ws->arena[w->base + (k - w->alo)];
}
static inline int inbl(int32_t off, int k, int m, int n) {
  return (uint32_t)off <= (uint32_t)n && (uint32_t)(off - k) <= (uint32_t)m;
}
static const wfl_t* srcl(const wsl_t* ws, int s) { return s >= 0 ? &ws->w[s] : NULL; }

static int wl_compute(wsl_t* ws, int s, int x, int e, int m, int n, ora_stats_t* st) {
  const wfl_t* mm = srcl(ws, s - x);
  const wfl_t* me = srcl(ws, s - e);
  wfl_t* out = &ws->w[s];
  memset(out, 0, sizeof(*out));
  out->lo = 1;
  out->hi = 0;
  if (wl_null(mm) && wl_null(me)) return 0;
  int lo = INT_MAX, hi = INT_MIN;
  if (!wl_null(mm)) {
    lo = mm->lo;
    hi = mm->hi;
  }
  if (!wl_null(me)) {
    if (lo > me->lo - 1) lo = me->lo - 1;
    if (hi < me->hi + 1) hi = me->hi + 1;
  }
  const int64_t b = wsl_alloc(ws, hi - lo + 1);
  if (b < 0) return ORA_ENOMEM;
  out->present = 1;
  out->alo = lo;
  out->ahi = hi;
  out->base = b;
  for (int k = lo; k <= hi; ++k) {
    const int32_t mis = wl_get(ws, mm, k) + 1;
    const int32_t ins = wl_get(ws, me, k - 1) + 1;
    const int32_t del = wl_get(ws, me, k + 1);
    int32_t v = mis > ins ? mis : ins;
    if (del > v) v = del;
    ws->arena[b + (k - lo)] = inbl(v, k, m, n) ? v : LNULL;
  }
  int k;
  for (k = hi; k >= lo; --k)
    if (ws->arena[b + (k - lo)] != LNULL) break;
  out->hi = k;
  for (k = lo; k <= out->hi; ++k)
    if (ws->arena[b + (k - lo)] != LNULL) break;
  out->lo = k;
  if (st) {
    st->steps++;
    st->cells += hi - lo + 1;
  }
  return 0;
}

static void wl_extend(wsl_t* ws, int s, const unsigned char* p, int m, const unsigned char* t, int n) {
  wfl_t* M = &ws->w[s];
  if (wl_null(M)) return;
  for (int k = M->lo; k <= M->hi; ++k) {
    int32_t* po = &ws->arena[M->base + (k - M->alo)];
    if (*po == LNULL) continue;
    const int v = *po - k, h = *po;
    const int rem = (m - v) < (n - h) ? (m - v) : (n - h);
    int l = 0;
    while (l < rem && p[v + l] == t[h + l]) ++l;
    *po += l;
  }
}

/* piggyback: offset * 16 + code, mismatch 9 > deletion 5 > insertion 1 */
static inline int64_t pbl(const wsl_t* ws, const wfl_t* w, int k, int delta, int code) {
  const int32_t o = wl_get(ws, w, k);
  if (o == LNULL) return (int64_t)INT64_MIN / 4;
  return (int64_t)(o + delta) * 16 + code;
}

static int wl_backtrace(wsl_t* ws, int s_end, int k_end, int x, int e, int m, int n, int* start) {
  const int cap = m + n + 1;
  if (ws->opbuf_cap < cap) {
    char* nb = (char*)realloc(ws->opbuf, (size_t)cap);
    if (!nb) return ORA_ENOMEM;
    ws->opbuf = nb;
    ws->opbuf_cap = cap;
  }
  char* ops = ws->opbuf;
  int pos = cap - 1;
#define EMITL(c)                     \
  do {                               \
    if (pos < 0) return ORA_ECIGCAP; \
    ops[pos--] = (c);                \
  } while (0)
  int s = s_end, k = k_end;
  int32_t off = wl_get(ws, &ws->w[s_end], k_end);
  int v = off - k, h = off;
  for (int i = v; i < m; ++i) EMITL('D');  /* free trailing gap */
  for (int i = h; i < n; ++i) EMITL('I');
  while (v > 0 && h > 0 && s > 0) {
    const int64_t mis = pbl(ws, srcl(ws, s - x), k, 1, 9);
    const int64_t del = pbl(ws, srcl(ws, s - e), k + 1, 0, 5);
    const int64_t ins = pbl(ws, srcl(ws, s - e), k - 1, 1, 1);
    int64_t best = mis > del ? mis : del;
    if (ins > best) best = ins;
    if (best < 0) return ORA_EINVAL;
    const int32_t moff = (int32_t)((best - (best & 15)) / 16);
    for (int32_t i = moff; i < off; ++i) EMITL('M');
    off = moff;
    v = off - k;
    h = off;
    if (v <= 0 || h <= 0) break;
    switch ((int)(best & 15)) {
      case 9: s -= x; EMITL('X'); off--; break;
      case 5: s -= e; EMITL('D'); k++; break;
      default: s -= e; EMITL('I'); k--; off--; break;
    }
    v = off - k;
    h = off;
  }
  if (v > 0 && h > 0) {
    const int nm = v < h ? v : h;
    for (int i = 0; i < nm; ++i) EMITL('M');
    v -= nm;
    h -= nm;
  }
  while (v > 0) {
    EMITL('D');
    --v;
  }
  while (h > 0) {
    EMITL('I');
    --h;
  }
#undef EMITL
  *start = pos + 1;
  return 0;
}

static int alignl_ws(wsl_t* ws, const char* pattern, int m, const char* text, int n, int x, int e,
                     const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st) {
  if (m < 0 || n < 0 || x <= 0 || e <= 0) return ORA_EINVAL;
  const unsigned char* p = (const unsigned char*)pattern;
  const unsigned char* t = (const unsigned char*)text;
  ws->arena_used = 0;
  if (wsl_reserve(ws, 1)) return ORA_ENOMEM;
  /* score 0: diagonal 0, or every free start (as in the gap-affine oracle) */
  const int lo0 = -(ef->pattern_begin_free < m ? ef->pattern_begin_free : m);
  const int hi0 = ef->text_begin_free < n ? ef->text_begin_free : n;
  wfl_t* M0 = &ws->w[0];
  memset(M0, 0, sizeof(*M0));
  const int64_t b0 = wsl_alloc(ws, hi0 - lo0 + 1);
  if (b0 < 0) return ORA_ENOMEM;
  M0->present = 1;
  M0->lo = M0->alo = lo0;
  M0->hi = M0->ahi = hi0;
  M0->base = b0;
  for (int k = lo0; k <= hi0; ++k) ws->arena[b0 + (k - lo0)] = k > 0 ? k : 0;
  if (st) {
    st->steps++;
    st->cells += hi0 - lo0 + 1;
  }
  int s = 0, k_end = INT_MIN;
  for (;;) {
    wl_extend(ws, s, p, m, t, n);
    const wfl_t* M = &ws->w[s];
    k_end = INT_MIN;
    if (!wl_null(M))
      for (int k = M->lo; k <= M->hi; ++k) {  /* lowest ending diagonal */
        const int32_t off = wl_get(ws, M, k);
        if (off == LNULL) continue;
        const int v = off - k;
        if ((off >= n && v >= m - ef->pattern_end_free) || (v >= m && off >= n - ef->text_end_free)) {
          k_end = k;
          break;
        }
      }
    if (k_end != INT_MIN) break;
    ++s;
    if (wsl_reserve(ws, s + 1)) return ORA_ENOMEM;
    const int rc = wl_compute(ws, s, x, e, m, n, st);
    if (rc) return rc;
  }
  if (st) st->final_score = s;
  if (ops) {
    int start = 0;
    const int rc = wl_backtrace(ws, s, k_end, x, e, m, n, &start);
    if (rc) return rc;
    const int len = (m + n + 1) - start;
    if (len > ops_cap) return ORA_ECIGCAP;
    memcpy(ops, ws->opbuf + start, (size_t)len);
    if (ops_len) *ops_len = len;
  }
  return s;
}

static void wsl_free(wsl_t* ws) {
  free(ws->w);
  free(ws->arena);
  free(ws->opbuf);
}

static const ora_ends_t kLinEndToEnd = {0, 0, 0, 0};

int ora_align_linear(const char* pattern, int m, const char* text, int n, int x, int e, char* ops, int ops_cap,
                     int* ops_len, ora_stats_t* st) {
  return ora_align_linear_ends_free(pattern, m, text, n, x, e, &kLinEndToEnd, ops, ops_cap, ops_len, st);
}

int ora_align_linear_ends_free(const char* pattern, int m, const char* text, int n, int x, int e,
                               const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st) {
  wsl_t ws;
  memset(&ws, 0, sizeof(ws));
  const int r = alignl_ws(&ws, pattern, m, text, n, x, e, ef ? ef : &kLinEndToEnd, ops, ops_cap, ops_len, st);
  wsl_free(&ws);
  return r;
}

/* Needleman-Wunsch with linear gaps, O(n) memory. */
int ora_linear_dp_score(const char* pattern, int m, const char* text, int n, int x, int e) {
  int64_t* H = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  if (!H) return ORA_ENOMEM;
  for (int j = 0; j <= n; ++j) H[j] = (int64_t)e * j;
  for (int i = 1; i <= m; ++i) {
    int64_t diag = H[0];
    H[0] = (int64_t)e * i;
    for (int j = 1; j <= n; ++j) {
      const int64_t up = H[j];
      int64_t best = diag + (pattern[i - 1] == text[j - 1] ? 0 : x);
      if (up + e < best) best = up + e;
      if (H[j - 1] + e < best) best = H[j - 1] + e;
      diag = up;
      H[j] = best;
    }
  }
  const int64_t r = H[n];
  free(H);
  return (int)r;
}

int ora_align_batch_linear(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                           const int64_t* toff, const int32_t* tlen, int x, int e, int32_t* scores, char* ops,
                           const int64_t* ops_off, int32_t* ops_len, int nthreads) {
  return ora_align_batch_linear_ends_free(npairs, pat, poff, plen, txt, toff, tlen, x, e, &kLinEndToEnd, scores, ops,
                                          ops_off, ops_len, nthreads);
}

int ora_align_batch_linear_ends_free(int npairs, const char* pat, const int64_t* poff, const int32_t* plen,
                                     const char* txt, const int64_t* toff, const int32_t* tlen, int x, int e,
                                     const ora_ends_t* ef, int32_t* scores, char* ops, const int64_t* ops_off,
                                     int32_t* ops_len, int nthreads) {
  int err = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    wsl_t ws;
    memset(&ws, 0, sizeof(ws));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int i = 0; i < npairs; ++i) {
      int ol = 0;
      const int r = alignl_ws(&ws, pat + poff[i], plen[i], txt + toff[i], tlen[i], x, e, ef ? ef : &kLinEndToEnd,
                              ops ? ops + ops_off[i] : NULL, ops ? (int)(ops_off[i + 1] - ops_off[i]) : 0, &ol, NULL);
      if (r < 0) {
#ifdef _OPENMP
#pragma omp critical
#endif
        if (!err) err = r;
      } else {
        scores[i] = r;
        if (ops_len) ops_len[i] = ol;
      }
    }
    wsl_free(&ws);
  }
  return err;
}
