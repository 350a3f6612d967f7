/*
 * wfa_oracle2.c -- CPU oracle for dual gap-affine ("affine 2-pieces")
 * end-to-end WaveFront Alignment.  TEST INFRASTRUCTURE ONLY (see
 * wfa_oracle.h): used by tests/ as the parity checker of the engine's dual
 * gap-affine mode, never by the product.
 *
 * The model: match 0, mismatch x, a gap of length L costs
 * min(o1 + e1*L, o2 + e2*L).  The reference declares this mode but does not
 * implement it: its penalties carry gap_open2 / gap_ext2 (common.h:80-87),
 * its matrix types I2 / D2 (common.h:52-58) and its backtrace codes
 * bt_I2_open 3, bt_I2_ext 4, bt_D2_open 7, bt_D2_ext 8 beside the one-piece
 * ones (common.h:67-77).  Restated here from the published WFA algorithm
 * (WFA2-lib's gap-affine 2-pieces distance, Marco-Sola et al.):
 *   I1[s][k] = max(M[s-o1-e1][k-1], I1[s-e1][k-1]) + 1
 *   I2[s][k] = max(M[s-o2-e2][k-1], I2[s-e2][k-1]) + 1
 *   D1[s][k] = max(M[s-o1-e1][k+1], D1[s-e1][k+1])
 *   D2[s][k] = max(M[s-o2-e2][k+1], D2[s-e2][k+1])
 *   M[s][k]  = max(M[s-x][k] + 1, I1, I2, D1, D2), nullified out of bounds
 * with the same limits, trimming and null steps as the one-piece oracle, and
 * the wavefront backtrace resolving ties by the piggyback codes (mismatch 9 >
 * D2 ext 8 > D2 open 7 > D1 ext 6 > D1 open 5 > I2 ext 4 > I2 open 3 > I1 ext
 * 2 > I1 open 1).  Scores are pinned by an independent five-matrix DP
 * (ora_gotoh2_score); CIGAR identity with WFA2-lib is unpinned, as for the
 * one-piece mode.
 */
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "wfa_oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define ONULL2 ((int32_t)(INT32_MIN / 2))
#define PB_NULL2 ((int64_t)INT64_MIN / 4)

enum { B_I1O = 1, B_I1E = 2, B_I2O = 3, B_I2E = 4, B_D1O = 5, B_D1E = 6, B_D2O = 7, B_D2E = 8, B_M = 9 };
enum { C_M = 0, C_I1 = 1, C_D1 = 2, C_I2 = 3, C_D2 = 4, C_N = 5 };

typedef struct {
  int present;
  int lo, hi;    /* trimmed limits (lo > hi: null) */
  int alo, ahi;  /* compute range */
  int64_t base;  /* arena index of k = alo */
} wf2_t;

typedef struct {
  wf2_t* w[C_N];
  int cap_s;
  int32_t* arena;
  int64_t arena_cap, arena_used;
  char* opbuf;
  int opbuf_cap;
} ws2_t;

static int ws2_reserve(ws2_t* ws, int need) {
  if (need <= ws->cap_s) return 0;
  int nc = ws->cap_s ? ws->cap_s : 64;
  while (nc < need) nc *= 2;
  for (int c = 0; c < C_N; ++c) {
    wf2_t* nw = (wf2_t*)realloc(ws->w[c], sizeof(wf2_t) * (size_t)nc);
    if (!nw) return ORA_ENOMEM;
    memset(nw + ws->cap_s, 0, sizeof(wf2_t) * (size_t)(nc - ws->cap_s));
    ws->w[c] = nw;
  }
  ws->cap_s = nc;
  return 0;
}

static int64_t ws2_alloc(ws2_t* ws, int64_t n) {
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

static void ws2_free(ws2_t* ws) {
  for (int c = 0; c < C_N; ++c) free(ws->w[c]);
  free(ws->arena);
  free(ws->opbuf);
}

static inline int w2_null(const wf2_t* w) { return !w || !w->present || w->lo > w->hi; }
static inline int32_t w2_get(const ws2_t* ws, const wf2_t* w, int k) {
  if (w2_null(w) || k < w->lo || k > w->hi) return ONULL2;
  return ws->arena[w->base + (k - w->alo)];
}
static inline int32_t mx32(int32_t a, int32_t b) { return a > b ? a : b; }
static inline int inb(int32_t off, int k, int m, int n) {
  return (uint32_t)off <= (uint32_t)n && (uint32_t)(off - k) <= (uint32_t)m;
}

static void w2_trim(ws2_t* ws, wf2_t* w, int m, int n) {
  int k;
  for (k = w->ahi; k >= w->alo; --k)
    if (inb(ws->arena[w->base + (k - w->alo)], k, m, n)) break;
  w->hi = k;
  for (k = w->alo; k <= w->hi; ++k)
    if (inb(ws->arena[w->base + (k - w->alo)], k, m, n)) break;
  w->lo = k;
}

static const wf2_t* src(const ws2_t* ws, int c, int s) { return s >= 0 ? &ws->w[c][s] : NULL; }

static int w2_compute(ws2_t* ws, int s, int x, int o1, int e1, int o2, int e2, int m, int n, ora_stats_t* st) {
  const wf2_t* mm = src(ws, C_M, s - x);
  const wf2_t* mo1 = src(ws, C_M, s - o1 - e1);
  const wf2_t* mo2 = src(ws, C_M, s - o2 - e2);
  const wf2_t* i1e = src(ws, C_I1, s - e1);
  const wf2_t* d1e = src(ws, C_D1, s - e1);
  const wf2_t* i2e = src(ws, C_I2, s - e2);
  const wf2_t* d2e = src(ws, C_D2, s - e2);
  wf2_t* out[C_N];
  for (int c = 0; c < C_N; ++c) {
    out[c] = &ws->w[c][s];
    memset(out[c], 0, sizeof(wf2_t));
    out[c]->lo = 1;
    out[c]->hi = 0;
  }
  const int n_mm = w2_null(mm), n_mo1 = w2_null(mo1), n_mo2 = w2_null(mo2), n_i1 = w2_null(i1e),
            n_d1 = w2_null(d1e), n_i2 = w2_null(i2e), n_d2 = w2_null(d2e);
  if (n_mm && n_mo1 && n_mo2 && n_i1 && n_d1 && n_i2 && n_d2) return 0; /* null step */
  int lo = INT_MAX, hi = INT_MIN;
#define ENV(cond, l, h)       \
  if (!(cond)) {              \
    if (lo > (l)) lo = (l);   \
    if (hi < (h)) hi = (h);   \
  }
  ENV(n_mm, mm->lo, mm->hi)
  ENV(n_mo1, mo1->lo - 1, mo1->hi + 1)
  ENV(n_mo2, mo2->lo - 1, mo2->hi + 1)
  ENV(n_i1, i1e->lo + 1, i1e->hi + 1)
  ENV(n_i2, i2e->lo + 1, i2e->hi + 1)
  ENV(n_d1, d1e->lo - 1, d1e->hi - 1)
  ENV(n_d2, d2e->lo - 1, d2e->hi - 1)
#undef ENV
  const int width = hi - lo + 1;
  const int present[C_N] = {1, !n_mo1 || !n_i1, !n_mo1 || !n_d1, !n_mo2 || !n_i2, !n_mo2 || !n_d2};
  int64_t base[C_N];
  for (int c = 0; c < C_N; ++c) {
    base[c] = present[c] ? ws2_alloc(ws, width) : 0;
    if (base[c] < 0) return ORA_ENOMEM;
    if (present[c]) {
      out[c]->present = 1;
      out[c]->alo = lo;
      out[c]->ahi = hi;
      out[c]->base = base[c];
    }
  }
  for (int k = lo; k <= hi; ++k) {
    const int32_t i1 = mx32(w2_get(ws, mo1, k - 1), w2_get(ws, i1e, k - 1)) + 1;
    const int32_t i2 = mx32(w2_get(ws, mo2, k - 1), w2_get(ws, i2e, k - 1)) + 1;
    const int32_t d1 = mx32(w2_get(ws, mo1, k + 1), w2_get(ws, d1e, k + 1));
    const int32_t d2 = mx32(w2_get(ws, mo2, k + 1), w2_get(ws, d2e, k + 1));
    const int32_t mis = w2_get(ws, mm, k) + 1;
    int32_t mv = mx32(mx32(mis, mx32(i1, i2)), mx32(d1, d2));
    if (!inb(mv, k, m, n)) mv = ONULL2; /* only M is nullified */
    ws->arena[base[C_M] + (k - lo)] = mv;
    if (present[C_I1]) ws->arena[base[C_I1] + (k - lo)] = i1;
    if (present[C_D1]) ws->arena[base[C_D1] + (k - lo)] = d1;
    if (present[C_I2]) ws->arena[base[C_I2] + (k - lo)] = i2;
    if (present[C_D2]) ws->arena[base[C_D2] + (k - lo)] = d2;
  }
  for (int c = 0; c < C_N; ++c)
    if (present[c]) {
      out[c]->lo = lo;
      out[c]->hi = hi;
      w2_trim(ws, out[c], m, n);
    }
  if (st) {
    st->steps++;
    st->cells += width;
  }
  return 0;
}

static void w2_extend(ws2_t* ws, int s, const unsigned char* p, int m, const unsigned char* t, int n, ora_stats_t* st) {
  wf2_t* M = &ws->w[C_M][s];
  if (w2_null(M)) return;
  for (int k = M->lo; k <= M->hi; ++k) {
    int32_t* po = &ws->arena[M->base + (k - M->alo)];
    if (*po == ONULL2) continue;
    const int v = *po - k, h = *po;
    int rem = (m - v) < (n - h) ? (m - v) : (n - h), l = 0;
    while (l < rem && p[v + l] == t[h + l]) ++l;
    *po += l;
    if (st) {
      st->ext_chars += l;
      st->ext_calls++;
    }
  }
}

static inline int64_t pb2(int32_t off, int type) { return (int64_t)off * 16 + type; }
static inline int64_t mx64(int64_t a, int64_t b) { return a > b ? a : b; }
static inline int64_t bsrc(const ws2_t* ws, const wf2_t* w, int k, int delta, int type) {
  if (w2_null(w) || k < w->lo || k > w->hi) return PB_NULL2;
  return pb2(ws->arena[w->base + (k - w->alo)] + delta, type);
}

static int w2_backtrace(ws2_t* ws, int s_end, int k_end, int x, int o1, int e1, int o2, int e2, int m, int n,
                        int* start) {
  const int cap = m + n + 1;
  if (ws->opbuf_cap < cap) {
    char* nb = (char*)realloc(ws->opbuf, (size_t)cap);
    if (!nb) return ORA_ENOMEM;
    ws->opbuf = nb;
    ws->opbuf_cap = cap;
  }
  char* ops = ws->opbuf;
  int pos = cap - 1;
#define EMIT(c)                      \
  do {                               \
    if (pos < 0) return ORA_ECIGCAP; \
    ops[pos--] = (c);                \
  } while (0)
  int state = C_M, s = s_end, k = k_end;
  int32_t off = w2_get(ws, &ws->w[C_M][s_end], k_end);
  int v = off - k, h = off;
  for (int i = v; i < m; ++i) EMIT('D');  /* free trailing gap */
  for (int i = h; i < n; ++i) EMIT('I');
  while (v > 0 && h > 0 && s > 0) {
    const wf2_t* wmm = src(ws, C_M, s - x);
    const wf2_t* wo1 = src(ws, C_M, s - o1 - e1);
    const wf2_t* wo2 = src(ws, C_M, s - o2 - e2);
    const int64_t i1o = bsrc(ws, wo1, k - 1, 1, B_I1O), i1x = bsrc(ws, src(ws, C_I1, s - e1), k - 1, 1, B_I1E);
    const int64_t i2o = bsrc(ws, wo2, k - 1, 1, B_I2O), i2x = bsrc(ws, src(ws, C_I2, s - e2), k - 1, 1, B_I2E);
    const int64_t d1o = bsrc(ws, wo1, k + 1, 0, B_D1O), d1x = bsrc(ws, src(ws, C_D1, s - e1), k + 1, 0, B_D1E);
    const int64_t d2o = bsrc(ws, wo2, k + 1, 0, B_D2O), d2x = bsrc(ws, src(ws, C_D2, s - e2), k + 1, 0, B_D2E);
    int64_t best;
    switch (state) {
      case C_M: {
        const int64_t mis = bsrc(ws, wmm, k, 1, B_M);
        best = mx64(mx64(mis, mx64(mx64(i1o, i1x), mx64(i2o, i2x))), mx64(mx64(d1o, d1x), mx64(d2o, d2x)));
        break;
      }
      case C_I1: best = mx64(i1o, i1x); break;
      case C_I2: best = mx64(i2o, i2x); break;
      case C_D1: best = mx64(d1o, d1x); break;
      default: best = mx64(d2o, d2x); break;
    }
    if (best < 0) return ORA_EINVAL;
    if (state == C_M) {
      const int32_t moff = (int32_t)((best - (best & 15)) / 16);
      for (int32_t i = moff; i < off; ++i) EMIT('M');
      off = moff;
      v = off - k;
      h = off;
      if (v <= 0 || h <= 0) break;
    }
    switch ((int)(best & 15)) {
      case B_M: s -= x; state = C_M; EMIT('X'); off--; break;
      case B_I1O: s -= o1 + e1; state = C_M; EMIT('I'); k--; off--; break;
      case B_I1E: s -= e1; state = C_I1; EMIT('I'); k--; off--; break;
      case B_I2O: s -= o2 + e2; state = C_M; EMIT('I'); k--; off--; break;
      case B_I2E: s -= e2; state = C_I2; EMIT('I'); k--; off--; break;
      case B_D1O: s -= o1 + e1; state = C_M; EMIT('D'); k++; break;
      case B_D1E: s -= e1; state = C_D1; EMIT('D'); k++; break;
      case B_D2O: s -= o2 + e2; state = C_M; EMIT('D'); k++; break;
      case B_D2E: s -= e2; state = C_D2; EMIT('D'); k++; break;
      default: return ORA_EINVAL;
    }
    v = off - k;
    h = off;
  }
  if (v > 0 && h > 0) {
    const int nm = v < h ? v : h;
    for (int i = 0; i < nm; ++i) EMIT('M');
    v -= nm;
    h -= nm;
  }
  while (v > 0) {
    EMIT('D');
    --v;
  }
  while (h > 0) {
    EMIT('I');
    --h;
  }
#undef EMIT
  *start = pos + 1;
  return 0;
}

static int align2_ws(ws2_t* ws, const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2,
                     int e2, const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st) {
  if (m < 0 || n < 0 || x <= 0 || o1 < 0 || e1 <= 0 || o2 < 0 || e2 <= 0) return ORA_EINVAL;
  const unsigned char* p = (const unsigned char*)pattern;
  const unsigned char* t = (const unsigned char*)text;
  ws->arena_used = 0;
  if (ws2_reserve(ws, 1)) return ORA_ENOMEM;
  for (int c = 0; c < C_N; ++c) {
    memset(&ws->w[c][0], 0, sizeof(wf2_t));
    ws->w[c][0].lo = 1;
  }
  /* score 0: diagonal 0, or every free start (as in the gap-affine oracle) */
  const int lo0 = -(ef->pattern_begin_free < m ? ef->pattern_begin_free : m);
  const int hi0 = ef->text_begin_free < n ? ef->text_begin_free : n;
  wf2_t* M0 = &ws->w[C_M][0];
  const int64_t b0 = ws2_alloc(ws, hi0 - lo0 + 1);
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
    w2_extend(ws, s, p, m, t, n, st);
    const wf2_t* M = &ws->w[C_M][s];
    k_end = INT_MIN;
    if (!w2_null(M))
      for (int k = M->lo; k <= M->hi; ++k) {  /* lowest ending diagonal */
        const int32_t off = w2_get(ws, M, k);
        if (off == ONULL2) continue;
        const int v = off - k;
        if ((off >= n && v >= m - ef->pattern_end_free) || (v >= m && off >= n - ef->text_end_free)) {
          k_end = k;
          break;
        }
      }
    if (k_end != INT_MIN) break;
    ++s;
    if (ws2_reserve(ws, s + 1)) return ORA_ENOMEM;
    const int rc = w2_compute(ws, s, x, o1, e1, o2, e2, m, n, st);
    if (rc) return rc;
  }
  if (st) st->final_score = s;
  if (ops) {
    int start = 0;
    const int rc = w2_backtrace(ws, s, k_end, x, o1, e1, o2, e2, m, n, &start);
    if (rc) return rc;
    const int len = (m + n + 1) - start;
    if (len > ops_cap) return ORA_ECIGCAP;
    memcpy(ops, ws->opbuf + start, (size_t)len);
    if (ops_len) *ops_len = len;
  }
  return s;
}

static const ora_ends_t kEndToEnd2 = {0, 0, 0, 0};

int ora_align2(const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2, int e2, char* ops,
               int ops_cap, int* ops_len, ora_stats_t* st) {
  return ora_align2_ends_free(pattern, m, text, n, x, o1, e1, o2, e2, &kEndToEnd2, ops, ops_cap, ops_len, st);
}

int ora_align2_ends_free(const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2, int e2,
                         const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st) {
  ws2_t ws;
  memset(&ws, 0, sizeof(ws));
  const int r = align2_ws(&ws, pattern, m, text, n, x, o1, e1, o2, e2, ef ? ef : &kEndToEnd2, ops, ops_cap, ops_len,
                          st);
  ws2_free(&ws);
  return r;
}

/* Five-matrix DP: H best, E1/E2 ending in an insertion run of piece 1/2,
 * F1/F2 ending in a deletion run of piece 1/2.  O(n) memory.  With free
 * ends: a start (v, 0), v <= pattern_begin_free, or (0, h), h <= text_begin_free,
 * costs nothing, and the best of the last row (h >= n - text_end_free) and
 * column (v >= m - pattern_end_free) is the score. */
int ora_gotoh2_ends_free_score(const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2,
                               int e2, const ora_ends_t* ef) {
  const int64_t INF = (int64_t)1 << 40;
  int64_t* H = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t* F1 = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t* F2 = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  if (!H || !F1 || !F2) {
    free(H);
    free(F1);
    free(F2);
    return ORA_ENOMEM;
  }
#define MIN2(a, b) ((a) < (b) ? (a) : (b))
  int64_t E1 = INF, E2 = INF;
  H[0] = 0;
  F1[0] = F2[0] = INF;
  for (int j = 1; j <= n; ++j) {
    E1 = MIN2(E1 + e1, H[j - 1] + o1 + e1);
    E2 = MIN2(E2 + e2, H[j - 1] + o2 + e2);
    H[j] = j <= ef->text_begin_free ? 0 : MIN2(E1, E2);
    F1[j] = F2[j] = INF;
  }
  int64_t best = INF;
  if (m <= ef->pattern_end_free) best = H[n];
  if (m == 0)
    for (int j = n - ef->text_end_free > 0 ? n - ef->text_end_free : 0; j <= n; ++j) best = MIN2(best, H[j]);
  for (int i = 1; i <= m; ++i) {
    int64_t diag = H[0];
    F1[0] = MIN2(F1[0] + e1, H[0] + o1 + e1);
    F2[0] = MIN2(F2[0] + e2, H[0] + o2 + e2);
    H[0] = i <= ef->pattern_begin_free ? 0 : MIN2(F1[0], F2[0]);
    E1 = E2 = INF;
    for (int j = 1; j <= n; ++j) {
      const int64_t up = H[j];
      E1 = MIN2(E1 + e1, H[j - 1] + o1 + e1);
      E2 = MIN2(E2 + e2, H[j - 1] + o2 + e2);
      F1[j] = MIN2(F1[j] + e1, up + o1 + e1);
      F2[j] = MIN2(F2[j] + e2, up + o2 + e2);
      int64_t b = diag + (pattern[i - 1] == text[j - 1] ? 0 : x);
      b = MIN2(b, MIN2(MIN2(E1, E2), MIN2(F1[j], F2[j])));
      diag = up;
      H[j] = b;
    }
    if (i >= m - ef->pattern_end_free) best = MIN2(best, H[n]);
    if (i == m)
      for (int j = n - ef->text_end_free > 0 ? n - ef->text_end_free : 0; j <= n; ++j) best = MIN2(best, H[j]);
  }
#undef MIN2
  free(H);
  free(F1);
  free(F2);
  return (int)best;
}

int ora_gotoh2_score(const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2, int e2) {
  const int64_t INF = (int64_t)1 << 40;
  int64_t* H = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t* F1 = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t* F2 = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  if (!H || !F1 || !F2) {
    free(H);
    free(F1);
    free(F2);
    return ORA_ENOMEM;
  }
#define GAP(L) ((int64_t)o1 + (int64_t)e1 * (L) < (int64_t)o2 + (int64_t)e2 * (L) ? (int64_t)o1 + (int64_t)e1 * (L) \
                                                                                   : (int64_t)o2 + (int64_t)e2 * (L))
  H[0] = 0;
  F1[0] = F2[0] = INF;
  for (int j = 1; j <= n; ++j) {
    H[j] = GAP(j);
    F1[j] = F2[j] = INF;
  }
  for (int i = 1; i <= m; ++i) {
    int64_t diag = H[0];
    H[0] = GAP(i);
    F1[0] = (int64_t)o1 + (int64_t)e1 * i;
    F2[0] = (int64_t)o2 + (int64_t)e2 * i;
    int64_t E1 = INF, E2 = INF;
    for (int j = 1; j <= n; ++j) {
      const int64_t up = H[j];
      const int64_t a1 = E1 + e1, b1 = H[j - 1] + o1 + e1;
      E1 = a1 < b1 ? a1 : b1;
      const int64_t a2 = E2 + e2, b2 = H[j - 1] + o2 + e2;
      E2 = a2 < b2 ? a2 : b2;
      const int64_t c1 = F1[j] + e1, d1 = up + o1 + e1;
      F1[j] = c1 < d1 ? c1 : d1;
      const int64_t c2 = F2[j] + e2, d2 = up + o2 + e2;
      F2[j] = c2 < d2 ? c2 : d2;
      int64_t best = diag + (pattern[i - 1] == text[j - 1] ? 0 : x);
      if (E1 < best) best = E1;
      if (E2 < best) best = E2;
      if (F1[j] < best) best = F1[j];
      if (F2[j] < best) best = F2[j];
      diag = up;
      H[j] = best;
    }
  }
#undef GAP
  const int64_t r = H[n];
  free(H);
  free(F1);
  free(F2);
  return (int)r;
}

/* Cost of an operation string under the two-piece model: each maximal gap
 * run is charged its cheaper piece.  -1 if the string is not an alignment of
 * pattern to text. */
int64_t ora_cigar_cost2(const char* ops, int len, const char* pattern, int m, const char* text, int n, int x, int o1,
                        int e1, int o2, int e2) {
  int v = 0, h = 0;
  int64_t cost = 0;
  for (int i = 0; i < len;) {
    const char c = ops[i];
    if (c == 'M' || c == 'X') {
      if (v >= m || h >= n || (c == 'M') != (pattern[v] == text[h])) return -1;
      if (c == 'X') cost += x;
      ++v;
      ++h;
      ++i;
      continue;
    }
    if (c != 'I' && c != 'D') return -1;
    int j = i;
    while (j < len && ops[j] == c) ++j;
    const int64_t L = j - i;
    if (c == 'I') {
      if (h + L > n) return -1;
      h += (int)L;
    } else {
      if (v + L > m) return -1;
      v += (int)L;
    }
    const int64_t p1 = (int64_t)o1 + (int64_t)e1 * L, p2 = (int64_t)o2 + (int64_t)e2 * L;
    cost += p1 < p2 ? p1 : p2;
    i = j;
  }
  if (v != m || h != n) return -1;
  return cost;
}

int ora_align_batch2(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                     const int64_t* toff, const int32_t* tlen, int x, int o1, int e1, int o2, int e2, int32_t* scores,
                     char* ops, const int64_t* ops_off, int32_t* ops_len, int nthreads) {
  return ora_align_batch2_ends_free(npairs, pat, poff, plen, txt, toff, tlen, x, o1, e1, o2, e2, &kEndToEnd2, scores,
                                    ops, ops_off, ops_len, nthreads);
}

int ora_align_batch2_ends_free(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                               const int64_t* toff, const int32_t* tlen, int x, int o1, int e1, int o2, int e2,
                               const ora_ends_t* ef, int32_t* scores, char* ops, const int64_t* ops_off,
                               int32_t* ops_len, int nthreads) {
  int err = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    ws2_t ws;
    memset(&ws, 0, sizeof(ws));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int i = 0; i < npairs; ++i) {
      int ol = 0;
      const int r = align2_ws(&ws, pat + poff[i], plen[i], txt + toff[i], tlen[i], x, o1, e1, o2, e2,
                              ef ? ef : &kEndToEnd2, ops ? ops + ops_off[i] : NULL, ops ? (int)(ops_off[i + 1] - ops_off[i]) : 0, &ol, NULL);
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
    ws2_free(&ws);
  }
  return err;
}
