/*
 * wfa_oracle.h -- CPU oracle for gap-affine end-to-end WaveFront Alignment.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the tsunami_pact_b200
 * library, its CLI, its Python binding) links, loads or calls this code.  It
 * is used by tests/ as the parity checker, by __graft_entry__.smoke() as the
 * checker, and by bench.py's cpu_baseline / --impl reference leg as the
 * stand-in for the reference's CPU path (WFA2-lib, whose source is absent:
 * the reference's WFA2-lib/ submodule directory is empty, .gitmodules:1-3).
 *
 * What it restates:
 *   - the score semantics of the reference kernel wfa_dispatcher
 *     (wfa_gpu.cu:191-722): offsets are text positions h on diagonal
 *     k = h - v, the I/D/M recurrences of wfa_gpu.cu:616-626, the
 *     out-of-bounds nullification of wfa_gpu.cu:628-629, the end test of
 *     wfa_gpu.cu:289-300 and the end trimming of wfa_gpu.cu:636-719 --
 *     computed with int32 offsets and without the reference's indexing
 *     defects;
 *   - the published WFA2-lib gap-affine algorithm that the reference calls
 *     for its check (wfa_gpu.cu:150-166, default attributes: end-to-end,
 *     exact, high-memory, full CIGAR): wavefront limits from the sources'
 *     envelopes, nullification of only the M component, trimming of the ends
 *     of M, I and D, and the wavefront backtrace that resolves ties by the
 *     piggyback order whose numeric codes the reference copies in
 *     common.h:67-77 (bt_M=9 > D_ext=6 > D_open=5 > I_ext=2 > I_open=1).
 *
 * Parity status: scores are pinned by an independent O(mn) Gotoh DP in this
 * same file (ora_gotoh_score) -- the optimal end-to-end gap-affine score is
 * unique.  CIGAR byte-identity with WFA2-lib is UNPINNED: WFA2-lib's source
 * and tests are not available, so the tie-breaking restated here follows the
 * published algorithm and the reference's bt_type_t codes only.
 */
#ifndef TSU_WFA_ORACLE_H
#define TSU_WFA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t steps;        /* non-null score steps computed                    */
  int64_t cells;        /* sum over steps of (hi - lo + 1), compute range    */
  int64_t ext_chars;    /* characters matched by the extend step            */
  int64_t ext_calls;    /* extend calls on non-null M offsets               */
  int64_t final_score;  /* score of the last aligned pair                   */
} ora_stats_t;

/* Error codes (negative returns). */
#define ORA_EINVAL  (-1)
#define ORA_ENOMEM  (-2)
#define ORA_ECIGCAP (-3)  /* ops buffer too small */

/* Align one pair end-to-end.  Returns the score (>= 0) or a negative error.
 * When ops != NULL the WFA2-style operation string ('M','X','I','D', one char
 * per operation, pattern = vertical, text = horizontal) is written to ops
 * (no terminator) and its length to *ops_len.  ops_cap >= m + n suffices. */
int ora_align(const char* pattern, int m, const char* text, int n,
              int x, int o, int e,
              char* ops, int ops_cap, int* ops_len, ora_stats_t* st);

/* Independent Gotoh DP (O(n) memory, O(mn) time).  Returns the score. */
int ora_gotoh_score(const char* pattern, int m, const char* text, int n,
                    int x, int o, int e);

/* Cost of an operation string, or -1 if it does not transform pattern into
 * text (length mismatch or an 'M' on unequal characters / 'X' on equal). */
int64_t ora_cigar_cost(const char* ops, int len,
                       const char* pattern, int m, const char* text, int n,
                       int x, int o, int e);

/* Batch over concatenated sequences, OpenMP over pairs with nthreads threads
 * (<= 0: all available).  ops may be NULL (scores only); otherwise pair i's
 * operations go to ops + ops_off[i] (capacity ops_off[i+1] - ops_off[i])
 * and their count to ops_len[i].  Returns 0 or a negative error (first
 * failing pair's error). */
int ora_align_batch(int npairs,
                    const char* pat, const int64_t* poff, const int32_t* plen,
                    const char* txt, const int64_t* toff, const int32_t* tlen,
                    int x, int o, int e,
                    int32_t* scores, char* ops, const int64_t* ops_off,
                    int32_t* ops_len, int nthreads, ora_stats_t* st);

/* Run-length form of an operation string, BAM-style: (len << 4) | code with
 * M=0, I=1, D=2, X=8.  Returns the number of runs written, or -1 when cap is
 * too small. */
int ora_ops_to_rle(const char* ops, int len, uint32_t* runs, int cap);

int ora_max_threads(void);

/* Ends-free alignment (WFA2-lib's alignment_span = ends_free, set by
 * wavefront_aligner_set_alignment_free_ends): the alignment may start at
 * (v, 0) with v <= pattern_begin_free or (0, h) with h <= text_begin_free at
 * no cost, and end at (m, h) with h >= n - text_end_free or (v, n) with v >=
 * m - pattern_end_free.  All zero: end-to-end (ora_align).  The free end
 * gaps are part of the operation string ('I' / 'D' runs) at no cost; of
 * several ends at the optimal score the lowest diagonal k = h - v wins. */
typedef struct {
  int32_t pattern_begin_free, pattern_end_free, text_begin_free, text_end_free;
} ora_ends_t;
int ora_align_ends_free(const char* pattern, int m, const char* text, int n, int x, int o, int e,
                        const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st);
int ora_align_batch_ends_free(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                              const int64_t* toff, const int32_t* tlen, int x, int o, int e, const ora_ends_t* ef,
                              int32_t* scores, char* ops, const int64_t* ops_off, int32_t* ops_len, int nthreads);
/* Independent Gotoh DP with the same free ends, and the cost of an
 * operation string under them. */
int ora_gotoh_ends_free_score(const char* pattern, int m, const char* text, int n, int x, int o, int e,
                              const ora_ends_t* ef);
int64_t ora_cigar_cost_ends_free(const char* ops, int len, const char* pattern, int m, const char* text, int n,
                                 int x, int o, int e, const ora_ends_t* ef);

/* Dual gap-affine (two-piece) mode, wfa_oracle2.c: a gap of length L costs
 * min(o1 + e1*L, o2 + e2*L).  Same return conventions as the one-piece
 * functions above. */
int ora_align2(const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2, int e2, char* ops,
               int ops_cap, int* ops_len, ora_stats_t* st);
int ora_gotoh2_score(const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2, int e2);
int64_t ora_cigar_cost2(const char* ops, int len, const char* pattern, int m, const char* text, int n, int x, int o1,
                        int e1, int o2, int e2);
int ora_align_batch2(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                     const int64_t* toff, const int32_t* tlen, int x, int o1, int e1, int o2, int e2, int32_t* scores,
                     char* ops, const int64_t* ops_off, int32_t* ops_len, int nthreads);

/* Gap-linear mode, wfa_oracle_linear.c: a gap of length L costs e*L (edit
 * distance: x = e = 1; indel distance: x = 3, e = 1). */
int ora_align_linear(const char* pattern, int m, const char* text, int n, int x, int e, char* ops, int ops_cap,
                     int* ops_len, ora_stats_t* st);
int ora_linear_dp_score(const char* pattern, int m, const char* text, int n, int x, int e);
int ora_align_batch_linear(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                           const int64_t* toff, const int32_t* tlen, int x, int e, int32_t* scores, char* ops,
                           const int64_t* ops_off, int32_t* ops_len, int nthreads);

/* Free ends for the gap-linear and dual gap-affine oracles (same semantics
 * as ora_align_ends_free; the gap-linear scores are the gap-affine ones with
 * opening 0, so ora_gotoh_ends_free_score pins them). */
int ora_align_linear_ends_free(const char* pattern, int m, const char* text, int n, int x, int e,
                               const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st);
int ora_align_batch_linear_ends_free(int npairs, const char* pat, const int64_t* poff, const int32_t* plen,
                                     const char* txt, const int64_t* toff, const int32_t* tlen, int x, int e,
                                     const ora_ends_t* ef, int32_t* scores, char* ops, const int64_t* ops_off,
                                     int32_t* ops_len, int nthreads);
int ora_align2_ends_free(const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2, int e2,
                         const ora_ends_t* ef, char* ops, int ops_cap, int* ops_len, ora_stats_t* st);
int ora_align_batch2_ends_free(int npairs, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                               const int64_t* toff, const int32_t* tlen, int x, int o1, int e1, int o2, int e2,
                               const ora_ends_t* ef, int32_t* scores, char* ops, const int64_t* ops_off,
                               int32_t* ops_len, int nthreads);
int ora_gotoh2_ends_free_score(const char* pattern, int m, const char* text, int n, int x, int o1, int e1, int o2,
                               int e2, const ora_ends_t* ef);

/* CPU-check plugin for the wfa_gpu command line (TSU_CHECK_LIB). */
int tsu_check_align_scores(int64_t n, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                           const int64_t* toff, const int32_t* tlen, int x, int o, int e, int32_t* scores,
                           int threads);

/* Bidirectional (BiWFA-style) alignment, wfa_oracle_bidir.c: breakpoints
 * of forward and reverse wavefronts, recursion down to segments whose score
 * is at most base_score (<= 0: two of the dearest single edits), each
 * aligned by the plain WFA with its gap components.  Writes the operation
 * string to ops (no terminator), its length to *ops_len; returns 0 or a
 * negative error.  ops_cap >= m + n suffices. */
int ora_bialign(const char* pattern, int m, const char* text, int n, int x, int o, int e, int base_score,
                char* ops, int ops_cap, int* ops_len);
/* The same recursion cut by the two-ring search (forward and reverse in
 * turns, each new wavefront checked against the other side's last
 * max(x, o+e) + 1 scores for crossing offsets): what a GPU kernel with two
 * rings per pair computes. */
int ora_bialign_ring(const char* pattern, int m, const char* text, int n, int x, int o, int e, int base_score,
                     char* ops, int ops_cap, int* ops_len);
/* The two-ring breakpoint search on one segment with gap components (begin
 * and end 'M', 'I' or 'D'): the lowest crossing total *T, its component
 * *comp, forward diagonal *k and cut offset *h (text position).  Returns 1
 * when a crossing was found, 0 when none, or a negative error. */
int ora_crossing_split(const char* pattern, int m, const char* text, int n, int x, int o, int e, char begin,
                       char end, int* T, char* comp, int* k, int* h);
/* The same over a batch (OpenMP over segments): T[i] = -1 where none. */
int ora_crossing_split_batch(int64_t num, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                             const int64_t* toff, const int32_t* tlen, const char* begin, const char* end, int x,
                             int o, int e, int32_t* T, char* comp, int32_t* k, int32_t* h);
/* One segment of a bidirectional alignment by the plain WFA with gap
 * components (the recursion's base case): begin 'I'/'D' continues a gap
 * from the left (a leading run costs e per base), end 'I'/'D' requires the
 * last operation to be that gap ('M': free).  Returns the cost (>= 0) or a
 * negative error; operations as ora_align. */
int ora_align_segment(const char* pattern, int m, const char* text, int n, int x, int o, int e, char begin,
                      char end, char* ops, int ops_cap, int* ops_len);

/* The seeded pair generator (wfa_gen.c): the same pairs as the engine's
 * tsu_gen_batch for the same seed, first index and lengths/rates, without
 * the engine library.  Returns 0 or a negative error. */
int ora_gen_batch(uint64_t seed, int64_t first, int64_t count, const int32_t* lengths, const double* rates, char* pat,
                  const int64_t* pat_off, int32_t* pat_len, char* txt, const int64_t* txt_off, int32_t* txt_len);

/* CPU model of the reference's GPU kernel wfa_dispatcher, its defects
 * included (ref_kernel_model.c).  Pairs of seq_len bytes each at
 * pat0 + i * seq_len and txt0 + i * seq_len; `front` / `back` bytes are
 * readable before the first and after the last pair.  scores[i] receives the
 * kernel's int16 score, codes[i] 0 or the first violation: a wavefront index
 * outside the pair's ring, a byte read outside the buffers, or no end within
 * step_cap score steps (steps[i], nullable, receives the steps taken;
 * maxk[i], nullable, the largest |diagonal| addressed in the ring). */
#define ORA_REFK_RING  (-10)
#define ORA_REFK_SEQ   (-11)
#define ORA_REFK_STEPS (-12)
int ora_refk_batch(const char* pat0, const char* txt0, int64_t front, int64_t back, int64_t num, int seq_len, int x,
                   int o, int e, int wf_length, int step_cap, int16_t* scores, int32_t* codes, int32_t* steps,
                   int32_t* maxk);
#ifdef __cplusplus
}
#endif
#endif
