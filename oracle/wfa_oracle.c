/*
 * wfa_oracle.c -- CPU oracle for gap-affine end-to-end WaveFront Alignment.
 *
 * TEST INFRASTRUCTURE ONLY (see wfa_oracle.h for what it restates and its
 * parity status).  The product never links or calls this file.
 *
 * Conventions (same as the reference kernel, wfa_gpu.cu:214-215,643-645):
 *   pattern is vertical (index v), text is horizontal (index h),
 *   diagonal k = h - v, a wavefront offset is the text position h,
 *   the alignment ends on diagonal n - m at offset n.
 *   Penalties: match 0, mismatch x, gap of length L costs o + e*L.
 *
 * Memory mode: every wavefront of every score is kept ("high memory") so the
 * backtrace can read the offsets of the source wavefronts directly, the way
 * the WFA2-lib default configuration the reference checks against does
 * (wfa_gpu.cu:156-164).
 */
#include "wfa_oracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Null offset: INT32_MIN/2 so that +1 / +k never wraps (the reference uses
 * INT16_MIN/2 for its int16 offsets, common.h:6). */
#define ONULL ((int32_t)(INT32_MIN / 2))
/* Null piggyback value for a source outside its wavefront's [lo, hi]. */
#define PB_NULL ((int64_t)INT64_MIN / 4)

/* Piggyback codes: the numeric values the reference keeps in its bt_type_t
 * enum (common.h:67-77).  The larger code wins a tie on equal offsets. */
enum { BT_I_OPEN = 1, BT_I_EXT = 2, BT_D_OPEN = 5, BT_D_EXT = 6, BT_M = 9 };

typedef struct {
  int present;  /* allocated at this score (else: absent/null)              */
  int lo, hi;   /* trimmed limits; lo > hi means null                        */
  int alo;      /* compute range start (index of arena[base])                */
  int ahi;      /* compute range end                                         */
  int64_t base; /* arena index of k = alo                                    */
} wf_t;

typedef struct {
  wf_t *M, *I, *D;
  int cap_s;
  int32_t* arena;
  int64_t arena_cap, arena_used;
  char* opbuf;
  int opbuf_cap;
} ws_t;

static int ws_reserve_scores(ws_t* ws, int need) {
  if (need <= ws->cap_s) return 0;
  int cap = ws->cap_s ? ws->cap_s : 256;
  while (cap < need) cap *= 2;
  wf_t* nm = (wf_t*)realloc(ws->M, sizeof(wf_t) * (size_t)cap);
  if (!nm) return ORA_ENOMEM;
  ws->M = nm;
  wf_t* ni = (wf_t*)realloc(ws->I, sizeof(wf_t) * (size_t)cap);
  if (!ni) return ORA_ENOMEM;
  ws->I = ni;
  wf_t* nd = (wf_t*)realloc(ws->D, sizeof(wf_t) * (size_t)cap);
  if (!nd) return ORA_ENOMEM;
  ws->D = nd;
  ws->cap_s = cap;
  return 0;
}

static int64_t ws_alloc(ws_t* ws, int64_t n) {
  if (ws->arena_used + n > ws->arena_cap) {
    int64_t cap = ws->arena_cap ? ws->arena_cap : (1 << 16);
    while (cap < ws->arena_used + n) cap *= 2;
    int32_t* na = (int32_t*)realloc(ws->arena, sizeof(int32_t) * (size_t)cap);
    if (!na) return -1;
    ws->arena = na;
    ws->arena_cap = cap;
  }
  int64_t at = ws->arena_used;
  ws->arena_used += n;
  return at;
}

static void ws_free(ws_t* ws) {
  free(ws->M);
  free(ws->I);
  free(ws->D);
  free(ws->arena);
  free(ws->opbuf);
  memset(ws, 0, sizeof(*ws));
}

static inline int wf_null(const wf_t* w) { return !w || !w->present || w->lo > w->hi; }

/* Offset of component w at diagonal k; NULL outside the trimmed limits
 * (WFA2 pads sources with nulls outside [lo, hi] before reading them; the
 * reference does the same in its "init ends" block, wfa_gpu.cu:470-606). */
static inline int32_t wf_get(const ws_t* ws, const wf_t* w, int k) {
  if (wf_null(w) || k < w->lo || k > w->hi) return ONULL;
  return ws->arena[w->base + (k - w->alo)];
}

static inline int32_t* wf_ptr(ws_t* ws, wf_t* w, int k) { return &ws->arena[w->base + (k - w->alo)]; }

static inline int32_t max32(int32_t a, int32_t b) { return a > b ? a : b; }

/* Longest common prefix of p[0..rem) and t[0..rem), 8 bytes at a time. */
static inline int lcp_bytes(const unsigned char* p, const unsigned char* t, int rem) {
  int i = 0;
  while (i + 8 <= rem) {
    uint64_t a, b;
    memcpy(&a, p + i, 8);
    memcpy(&b, t + i, 8);
    uint64_t d = a ^ b;
    if (d) return i + (__builtin_ctzll(d) >> 3);
    i += 8;
  }
  while (i < rem && p[i] == t[i]) ++i;
  return i;
}

/* In-bounds test of the reference (wfa_gpu.cu:643-645): unsigned compares so
 * that negative h or v count as out of bounds. */
static inline int in_bounds(int32_t off, int k, int m, int n) {
  uint32_t h = (uint32_t)off;
  uint32_t v = (uint32_t)(off - k);
  return h <= (uint32_t)n && v <= (uint32_t)m;
}

/* Trim both ends of a computed component to its outermost in-bounds cells
 * (reference wfa_gpu.cu:636-719).  Interior out-of-bounds I/D offsets stay. */
static void wf_trim(ws_t* ws, wf_t* w, int m, int n) {
  int k;
  for (k = w->ahi; k >= w->alo; --k)
    if (in_bounds(*wf_ptr(ws, w, k), k, m, n)) break;
  w->hi = k;
  for (k = w->alo; k <= w->hi; ++k)
    if (in_bounds(*wf_ptr(ws, w, k), k, m, n)) break;
  w->lo = k;
}

/* Compute the M/I/D wavefronts of score s (reference wfa_gpu.cu:346-631). */
static int wf_compute(ws_t* ws, int s, int x, int o, int e, int m, int n, ora_stats_t* st) {
  const wf_t* mm = (s - x >= 0) ? &ws->M[s - x] : NULL;
  const wf_t* mo = (s - o - e >= 0) ? &ws->M[s - o - e] : NULL;
  const wf_t* ie = (s - e >= 0) ? &ws->I[s - e] : NULL;
  const wf_t* de = (s - e >= 0) ? &ws->D[s - e] : NULL;
  wf_t* M = &ws->M[s];
  wf_t* I = &ws->I[s];
  wf_t* D = &ws->D[s];
  memset(M, 0, sizeof(*M));
  memset(I, 0, sizeof(*I));
  memset(D, 0, sizeof(*D));
  M->lo = I->lo = D->lo = 1;
  M->hi = I->hi = D->hi = 0;
  const int nmm = wf_null(mm), nmo = wf_null(mo), nie = wf_null(ie), nde = wf_null(de);
  if (nmm && nmo && nie && nde) return 0; /* null step (wfa_gpu.cu:417-422) */
  /* Output limits: envelope of the sources' limits (wfa_gpu.cu:429-439). */
  int lo = INT_MAX, hi = INT_MIN;
  if (!nmm) { lo = mm->lo; hi = mm->hi; }
  if (!nmo) { if (lo > mo->lo - 1) lo = mo->lo - 1; if (hi < mo->hi + 1) hi = mo->hi + 1; }
  if (!nie) { if (lo > ie->lo + 1) lo = ie->lo + 1; if (hi < ie->hi + 1) hi = ie->hi + 1; }
  if (!nde) { if (lo > de->lo - 1) lo = de->lo - 1; if (hi < de->hi - 1) hi = de->hi - 1; }
  const int width = hi - lo + 1;
  const int i_present = !nmo || !nie; /* wfa_gpu.cu:455-461 */
  const int d_present = !nmo || !nde; /* wfa_gpu.cu:462-468 */
  int64_t bm = ws_alloc(ws, width);
  int64_t bi = i_present ? ws_alloc(ws, width) : 0;
  int64_t bd = d_present ? ws_alloc(ws, width) : 0;
  if (bm < 0 || bi < 0 || bd < 0) return ORA_ENOMEM;
  M->present = 1; M->alo = lo; M->ahi = hi; M->base = bm;
  if (i_present) { I->present = 1; I->alo = lo; I->ahi = hi; I->base = bi; }
  if (d_present) { D->present = 1; D->alo = lo; D->ahi = hi; D->base = bd; }
  /* Sources are read through wf_get (null outside their limits), and the
   * arena pointer may move during ws_alloc above, so fetch after allocating. */
  for (int k = lo; k <= hi; ++k) {
    const int32_t ins_o = wf_get(ws, mo, k - 1);
    const int32_t ins_e = wf_get(ws, ie, k - 1);
    const int32_t ins = max32(ins_o, ins_e) + 1;
    const int32_t del_o = wf_get(ws, mo, k + 1);
    const int32_t del_e = wf_get(ws, de, k + 1);
    const int32_t del = max32(del_o, del_e);
    const int32_t mis = wf_get(ws, mm, k) + 1;
    int32_t mx = max32(del, max32(mis, ins));
    if (!in_bounds(mx, k, m, n)) mx = ONULL; /* only M is nullified */
    ws->arena[bm + (k - lo)] = mx;
    if (i_present) ws->arena[bi + (k - lo)] = ins;
    if (d_present) ws->arena[bd + (k - lo)] = del;
  }
  M->lo = lo; M->hi = hi;
  wf_trim(ws, M, m, n);
  if (i_present) { I->lo = lo; I->hi = hi; wf_trim(ws, I, m, n); }
  if (d_present) { D->lo = lo; D->hi = hi; wf_trim(ws, D, m, n); }
  if (st) { st->steps++; st->cells += width; }
  return 0;
}

/* Extend M[s] along its diagonals (reference wfa_gpu.cu:257-287, computed
 * with explicit bounds instead of reading past the sequences). */
static void wf_extend(ws_t* ws, int s, const unsigned char* p, int m, const unsigned char* t, int n,
                      ora_stats_t* st) {
  wf_t* M = &ws->M[s];
  if (wf_null(M)) return;
  for (int k = M->lo; k <= M->hi; ++k) {
    int32_t* po = wf_ptr(ws, M, k);
    const int32_t off = *po;
    if (off == ONULL) continue;
    const int v = off - k, h = off;
    const int rem = (m - v) < (n - h) ? (m - v) : (n - h);
    const int l = lcp_bytes(p + v, t + h, rem);
    *po = off + l;
    if (st) { st->ext_chars += l; st->ext_calls++; }
  }
}

static inline int64_t pb(int32_t off, int type) { return (int64_t)off * 16 + type; }
static inline int32_t pb_off(int64_t v) { return (int32_t)((v - (v & 15)) / 16); }
static inline int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }

/* Backtrace source probes: the piggyback value of one candidate predecessor,
 * or PB_NULL when its wavefront is absent or k is outside its limits. */
static inline int64_t bt_src(const ws_t* ws, const wf_t* w, int k, int delta, int type) {
  if (wf_null(w) || k < w->lo || k > w->hi) return PB_NULL;
  return pb(ws->arena[w->base + (k - w->alo)] + delta, type);
}

enum { ST_M = 0, ST_I = 1, ST_D = 2 };

/* Wavefront backtrace from M[s_end][k_end] (n - m for end-to-end; with free
 * ends the end diagonal found by align_ws, whose trailing pattern or text
 * gap is emitted first).  Writes operations backwards into ws->opbuf and
 * returns the start index, or < 0. */
static int wf_backtrace(ws_t* ws, int s_end, int k_end, int x, int o, int e, int m, int n, int* start) {
  const int cap = m + n + 1;
  if (ws->opbuf_cap < cap) {
    char* nb = (char*)realloc(ws->opbuf, (size_t)cap);
    if (!nb) return ORA_ENOMEM;
    ws->opbuf = nb;
    ws->opbuf_cap = cap;
  }
  char* ops = ws->opbuf;
  int pos = cap - 1;
#define EMIT(c)                        \
  do {                                 \
    if (pos < 0) return ORA_ECIGCAP;   \
    ops[pos--] = (c);                  \
  } while (0)
  int state = ST_M, s = s_end, k = k_end;
  int32_t off = wf_get(ws, &ws->M[s_end], k_end);
  int v = off - k, h = off;
  /* free end gap: the rest of the pattern (text consumed) or of the text */
  for (int i = v; i < m; ++i) EMIT('D');
  for (int i = h; i < n; ++i) EMIT('I');
  while (v > 0 && h > 0 && s > 0) {
    const int smis = s - x, sgo = s - o - e, sge = s - e;
    const wf_t* wm_mis = smis >= 0 ? &ws->M[smis] : NULL;
    const wf_t* wm_go = sgo >= 0 ? &ws->M[sgo] : NULL;
    const wf_t* wi_ge = sge >= 0 ? &ws->I[sge] : NULL;
    const wf_t* wd_ge = sge >= 0 ? &ws->D[sge] : NULL;
    int64_t best;
    const int64_t io = bt_src(ws, wm_go, k - 1, 1, BT_I_OPEN);
    const int64_t ix = bt_src(ws, wi_ge, k - 1, 1, BT_I_EXT);
    const int64_t dop = bt_src(ws, wm_go, k + 1, 0, BT_D_OPEN);
    const int64_t dx = bt_src(ws, wd_ge, k + 1, 0, BT_D_EXT);
    if (state == ST_M) {
      const int64_t mis = bt_src(ws, wm_mis, k, 1, BT_M);
      best = max64(mis, max64(max64(io, ix), max64(dop, dx)));
    } else if (state == ST_I) {
      best = max64(io, ix);
    } else {
      best = max64(dop, dx);
    }
    if (best < 0) return ORA_EINVAL; /* no valid predecessor: internal error */
    if (state == ST_M) {
      const int32_t moff = pb_off(best);
      for (int32_t i = moff; i < off; ++i) EMIT('M');
      off = moff;
      v = off - k;
      h = off;
      if (v <= 0 || h <= 0) break;
    }
    switch ((int)(best & 15)) {
      case BT_M: s = smis; state = ST_M; EMIT('X'); off--; break;
      case BT_I_OPEN: s = sgo; state = ST_M; EMIT('I'); k--; off--; break;
      case BT_I_EXT: s = sge; state = ST_I; EMIT('I'); k--; off--; break;
      case BT_D_OPEN: s = sgo; state = ST_M; EMIT('D'); k++; break;
      case BT_D_EXT: s = sge; state = ST_D; EMIT('D'); k++; break;
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
  while (v > 0) { EMIT('D'); --v; }
  while (h > 0) { EMIT('I'); --h; }
#undef EMIT
  *start = pos + 1;
  return 0;
}

/* The end diagonal of M[s] (the lowest k that ends an alignment), or
 * INT_MIN.  End-to-end: k = n - m at offset n.  With free ends: the text is
 * consumed with at most pef pattern characters left, or the pattern with at
 * most tef text characters left (WFA2-lib's ends-free termination). */
static int wf_end_diagonal(const ws_t* ws, const wf_t* M, int m, int n, const ora_ends_t* ef) {
  if (wf_null(M)) return INT_MIN;
  for (int k = M->lo; k <= M->hi; ++k) {
    const int32_t off = wf_get(ws, M, k);
    if (off == ONULL) continue;
    const int v = off - k;
    if ((off >= n && v >= m - ef->pattern_end_free) || (v >= m && off >= n - ef->text_end_free)) return k;
  }
  return INT_MIN;
}

static int align_ws(ws_t* ws, const char* pattern, int m, const char* text, int n, int x, int o, int e,
                    const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st) {
  if (m < 0 || n < 0 || x <= 0 || o < 0 || e <= 0) return ORA_EINVAL;
  if (ef->pattern_begin_free < 0 || ef->pattern_end_free < 0 || ef->text_begin_free < 0 || ef->text_end_free < 0)
    return ORA_EINVAL;
  const unsigned char* p = (const unsigned char*)pattern;
  const unsigned char* t = (const unsigned char*)text;
  ws->arena_used = 0;
  if (ws_reserve_scores(ws, 1)) return ORA_ENOMEM;
  /* Score 0: M[0] = {k=0: offset 0} (wfa_gpu.cu:239-242); with free
   * beginnings every start (v, 0), v <= pattern_begin_free, and (0, h),
   * h <= text_begin_free: diagonals -pbf..tbf at offset max(k, 0). */
  const int lo0 = -(ef->pattern_begin_free < m ? ef->pattern_begin_free : m);
  const int hi0 = ef->text_begin_free < n ? ef->text_begin_free : n;
  wf_t* M0 = &ws->M[0];
  memset(M0, 0, sizeof(*M0));
  memset(&ws->I[0], 0, sizeof(wf_t));
  memset(&ws->D[0], 0, sizeof(wf_t));
  ws->I[0].lo = ws->D[0].lo = 1;
  int64_t b0 = ws_alloc(ws, hi0 - lo0 + 1);
  if (b0 < 0) return ORA_ENOMEM;
  M0->present = 1; M0->lo = M0->alo = lo0; M0->hi = M0->ahi = hi0; M0->base = b0;
  for (int k = lo0; k <= hi0; ++k) ws->arena[b0 + (k - lo0)] = k > 0 ? k : 0;
  if (st) { st->steps++; st->cells += hi0 - lo0 + 1; }
  int s = 0, k_end;
  for (;;) {
    wf_extend(ws, s, p, m, t, n, st);
    k_end = wf_end_diagonal(ws, &ws->M[s], m, n, ef);
    if (k_end != INT_MIN) break;
    ++s;
    if (ws_reserve_scores(ws, s + 1)) return ORA_ENOMEM;
    int rc = wf_compute(ws, s, x, o, e, m, n, st);
    if (rc) return rc;
  }
  if (st) st->final_score = s;
  if (ops) {
    int start = 0;
    int rc = wf_backtrace(ws, s, k_end, x, o, e, m, n, &start);
    if (rc) return rc;
    const int len = (m + n + 1) - start;
    if (len > ops_cap) return ORA_ECIGCAP;
    memcpy(ops, ws->opbuf + start, (size_t)len);
    if (ops_len) *ops_len = len;
  }
  return s;
}

static const ora_ends_t kEndToEnd = {0, 0, 0, 0};

int ora_align(const char* pattern, int m, const char* text, int n, int x, int o, int e, char* ops, int ops_cap,
              int* ops_len, ora_stats_t* st) {
  ws_t ws;
  memset(&ws, 0, sizeof(ws));
  int r = align_ws(&ws, pattern, m, text, n, x, o, e, &kEndToEnd, ops, ops_cap, ops_len, st);
  ws_free(&ws);
  return r;
}

int ora_align_ends_free(const char* pattern, int m, const char* text, int n, int x, int o, int e,
                        const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st) {
  ws_t ws;
  memset(&ws, 0, sizeof(ws));
  int r = align_ws(&ws, pattern, m, text, n, x, o, e, ef ? ef : &kEndToEnd, ops, ops_cap, ops_len, st);
  ws_free(&ws);
  return r;
}

int ora_gotoh_score(const char* pattern, int m, const char* text, int n, int x, int o, int e) {
  /* H: best score ending anywhere; E: ending with an insertion (text char);
   * F: ending with a deletion (pattern char).  Rows indexed by v (pattern). */
  const int64_t INF = (int64_t)1 << 40;
  int64_t* H = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t* F = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  if (!H || !F) { free(H); free(F); return ORA_ENOMEM; }
  H[0] = 0;
  F[0] = INF;
  for (int j = 1; j <= n; ++j) { H[j] = (int64_t)o + (int64_t)e * j; F[j] = INF; }
  for (int i = 1; i <= m; ++i) {
    int64_t diag = H[0];
    H[0] = (int64_t)o + (int64_t)e * i;
    F[0] = H[0];
    int64_t E = INF;
    for (int j = 1; j <= n; ++j) {
      const int64_t up_h = H[j];
      E = (E + e < H[j - 1] + o + e) ? E + e : H[j - 1] + o + e;
      F[j] = (F[j] + e < up_h + o + e) ? F[j] + e : up_h + o + e;
      int64_t best = diag + (pattern[i - 1] == text[j - 1] ? 0 : x);
      if (E < best) best = E;
      if (F[j] < best) best = F[j];
      diag = up_h;
      H[j] = best;
    }
  }
  int64_t r = H[n];
  free(H);
  free(F);
  return (int)r;
}

int64_t ora_cigar_cost(const char* ops, int len, const char* pattern, int m, const char* text, int n, int x, int o,
                       int e) {
  int v = 0, h = 0;
  int64_t cost = 0;
  char prev = 0;
  for (int i = 0; i < len; ++i) {
    const char c = ops[i];
    switch (c) {
      case 'M':
        if (v >= m || h >= n || pattern[v] != text[h]) return -1;
        ++v; ++h;
        break;
      case 'X':
        if (v >= m || h >= n || pattern[v] == text[h]) return -1;
        cost += x; ++v; ++h;
        break;
      case 'I':
        if (h >= n) return -1;
        cost += (prev == 'I') ? e : (o + e);
        ++h;
        break;
      case 'D':
        if (v >= m) return -1;
        cost += (prev == 'D') ? e : (o + e);
        ++v;
        break;
      default:
        return -1;
    }
    prev = c;
  }
  if (v != m || h != n) return -1;
  return cost;
}

int ora_ops_to_rle(const char* ops, int len, uint32_t* runs, int cap) {
  int nr = 0;
  int i = 0;
  while (i < len) {
    const char c = ops[i];
    int j = i;
    while (j < len && ops[j] == c) ++j;
    uint32_t code = c == 'M' ? 0u : c == 'I' ? 1u : c == 'D' ? 2u : 8u;
    if (nr >= cap) return -1;
    runs[nr++] = ((uint32_t)(j - i) << 4) | code;
    i = j;
  }
  return nr;
}

int ora_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static int batch_impl(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                      const int64_t* toff, const int32_t* tlen, int x, int o, int e, const ora_ends_t* ef,
                      int32_t* scores, char* ops, const int64_t* ops_off, int32_t* ops_len, int nthreads,
                      ora_stats_t* st) {
  int err = 0;
  int64_t steps = 0, cells = 0, extc = 0, extn = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(+ : steps, cells, extc, extn)
#endif
  {
    ws_t ws;
    memset(&ws, 0, sizeof(ws));
    ora_stats_t ls;
    memset(&ls, 0, sizeof(ls));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int i = 0; i < npairs; ++i) {
      char* po = ops ? ops + ops_off[i] : NULL;
      const int cap = ops ? (int)(ops_off[i + 1] - ops_off[i]) : 0;
      int len = 0;
      int r = align_ws(&ws, pat + poff[i], plen[i], txt + toff[i], tlen[i], x, o, e, ef, po, cap, &len,
                       st ? &ls : NULL);
      scores[i] = r;
      if (ops_len) ops_len[i] = ops ? len : 0;
      if (r < 0) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
        err = r;
      }
    }
    steps += ls.steps;
    cells += ls.cells;
    extc += ls.ext_chars;
    extn += ls.ext_calls;
    ws_free(&ws);
  }
  if (st) {
    st->steps = steps;
    st->cells = cells;
    st->ext_chars = extc;
    st->ext_calls = extn;
  }
  return err;
}

/* CPU-check plugin entry point: the symbol the engine's wfa_gpu command line
 * looks up in the library named by TSU_CHECK_LIB when check=1.  Computes the
 * full alignment of every pair (as the reference's WFA2-lib check does,
 * wfa_gpu.cu:154-166) and returns the scores. */
int ora_align_batch(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                    const int64_t* toff, const int32_t* tlen, int x, int o, int e, int32_t* scores, char* ops,
                    const int64_t* ops_off, int32_t* ops_len, int nthreads, ora_stats_t* st) {
  return batch_impl(npairs, pat, poff, plen, txt, toff, tlen, x, o, e, &kEndToEnd, scores, ops, ops_off, ops_len,
                    nthreads, st);
}

int ora_align_batch_ends_free(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                              const int64_t* toff, const int32_t* tlen, int x, int o, int e, const ora_ends_t* ef,
                              int32_t* scores, char* ops, const int64_t* ops_off, int32_t* ops_len, int nthreads) {
  return batch_impl(npairs, pat, poff, plen, txt, toff, tlen, x, o, e, ef ? ef : &kEndToEnd, scores, ops, ops_off,
                    ops_len, nthreads, NULL);
}

/* Gotoh DP with free ends: a start (v, 0) with v <= pattern_begin_free or
 * (0, h) with h <= text_begin_free costs nothing, and the best of the last
 * row at h >= n - text_end_free and of the last column at v >= m -
 * pattern_end_free is the score. */
int ora_gotoh_ends_free_score(const char* pattern, int m, const char* text, int n, int x, int o, int e,
                              const ora_ends_t* ef) {
  const int64_t INF = (int64_t)1 << 40;
  int64_t* H = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t* F = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  if (!H || !F) { free(H); free(F); return ORA_ENOMEM; }
  /* row 0: free up to text_begin_free, then an insertion run from there */
  int64_t E0 = INF;
  H[0] = 0;
  F[0] = INF;
  for (int j = 1; j <= n; ++j) {
    E0 = (E0 + e < H[j - 1] + o + e) ? E0 + e : H[j - 1] + o + e;
    H[j] = j <= ef->text_begin_free ? 0 : E0;
    F[j] = INF;
  }
  int64_t best_end = INF;
  if (m <= ef->pattern_end_free || m == 0)  /* last column of row 0 */
    best_end = H[n];
  for (int j = (n - ef->text_end_free > 0 ? n - ef->text_end_free : 0); j <= n && m == 0; ++j)
    if (H[j] < best_end) best_end = H[j];
  for (int i = 1; i <= m; ++i) {
    int64_t diag = H[0];
    /* column 0: free up to pattern_begin_free, then a deletion run */
    F[0] = (F[0] + e < H[0] + o + e) ? F[0] + e : H[0] + o + e;
    H[0] = i <= ef->pattern_begin_free ? 0 : F[0];
    int64_t E = INF;
    for (int j = 1; j <= n; ++j) {
      const int64_t up_h = H[j];
      E = (E + e < H[j - 1] + o + e) ? E + e : H[j - 1] + o + e;
      F[j] = (F[j] + e < up_h + o + e) ? F[j] + e : up_h + o + e;
      int64_t best = diag + (pattern[i - 1] == text[j - 1] ? 0 : x);
      if (E < best) best = E;
      if (F[j] < best) best = F[j];
      diag = up_h;
      H[j] = best;
    }
    if (i >= m - ef->pattern_end_free && H[n] < best_end) best_end = H[n];
    if (i == m)
      for (int j = (n - ef->text_end_free > 0 ? n - ef->text_end_free : 0); j <= n; ++j)
        if (H[j] < best_end) best_end = H[j];
  }
  free(H);
  free(F);
  return (int)best_end;
}

/* Cost of an operation string with free ends: a leading insertion run costs
 * gap(L - text_begin_free) beyond the free part (a leading deletion run
 * likewise with pattern_begin_free), trailing runs with the end allowances;
 * -1 if the string is not an alignment of pattern to text. */
int64_t ora_cigar_cost_ends_free(const char* ops, int len, const char* pattern, int m, const char* text, int n,
                                 int x, int o, int e, const ora_ends_t* ef) {
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
    int64_t L = j - i;
    if (c == 'I') {
      if (h + L > n) return -1;
      h += (int)L;
    } else {
      if (v + L > m) return -1;
      v += (int)L;
    }
    int64_t free_len = 0;  /* a run that is both first and last has both allowances */
    if (i == 0) free_len += c == 'I' ? ef->text_begin_free : ef->pattern_begin_free;
    if (j == len) free_len += c == 'I' ? ef->text_end_free : ef->pattern_end_free;
    if (L > free_len) cost += (int64_t)o + (int64_t)e * (L - free_len);
    i = j;
  }
  if (v != m || h != n) return -1;
  return cost;
}

int tsu_check_align_scores(int64_t n, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                           const int64_t* toff, const int32_t* tlen, int x, int o, int e, int32_t* scores,
                           int threads) {
  int err = 0;
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
#endif
  {
    ws_t ws;
    memset(&ws, 0, sizeof(ws));
    char* ops = NULL;
    int ops_cap = 0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int64_t i = 0; i < n; ++i) {
      const int need = plen[i] + tlen[i] + 1;
      if (need > ops_cap) {
        free(ops);
        ops = (char*)malloc((size_t)need);
        ops_cap = ops ? need : 0;
      }
      int len = 0;
      int r = ops ? align_ws(&ws, pat + poff[i], plen[i], txt + toff[i], tlen[i], x, o, e, &kEndToEnd, ops, ops_cap,
                             &len, NULL)
                  : ORA_ENOMEM;
      scores[i] = r;
      if (r < 0) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
        err = r;
      }
    }
    free(ops);
    ws_free(&ws);
  }
  return err;
}
