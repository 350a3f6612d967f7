/*
 * tsunami_b200.h -- C ABI of the B200-native gap-affine WaveFront Alignment
 * (WFA) engine.  Plain pointers and sizes only; every call returns a status
 * code (TSU_OK == 0) and never exits the process.
 *
 * The reference (giuliagerometta/TSUNAMI_PACT) exposes this path as
 *   - the command line `wfa_gpu mismatch gap_opening gap_extension
 *     input_file wf_length check` (wfa_gpu.cu:43-188), and
 *   - its kernel ABI `wfa_dispatcher(char* pattern_d, char* text_d,
 *     short* score_d, ...)` over fixed-stride equal-length pairs
 *     (wfa_gpu.cu:36-39, launched at wfa_gpu.cu:118-120),
 * with the CPU check through WFA2-lib's `wavefront_align`
 * (wfa_gpu.cu:154-166).  The entry points below replace those; each one
 * names the reference interface it stands in for.
 *
 * Conventions: the pattern is the vertical sequence, the text the horizontal
 * one (wfa_gpu.cu:164 passes pattern first).  Penalties: match 0, mismatch x,
 * a gap of length L costs gap_opening + gap_extension * L.  Scores are the
 * positive penalty sums (the reference prints -(cigar->score),
 * wfa_gpu.cu:165).  CIGARs are WFA2-style operation sequences (M match,
 * X mismatch, I insertion = text character, D deletion = pattern character)
 * delivered run-length encoded, one uint32 per run: (length << 4) | code,
 * code M=0, I=1, D=2, X=8.
 */
#ifndef TSUNAMI_B200_H
#define TSUNAMI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define TSU_OK 0
#define TSU_EINVAL 1    /* bad argument (penalties, lengths, null pointer)  */
#define TSU_ENOMEM 2    /* device memory budget exceeded / allocation failed */
#define TSU_EDEVICE 3   /* CUDA error (launch, copy, device lost)            */
#define TSU_ETIMEOUT 4  /* a wait ran out of time                            */
#define TSU_EOVERFLOW 5 /* caller's output buffer too small (see *_needed)   */
#define TSU_EBUSY 6     /* serving queue full / admission refused            */
#define TSU_ENOTFOUND 7 /* unknown request id                                */
#define TSU_EINTERNAL 8 /* an internal consistency check failed              */
#define TSU_EIO 9       /* file could not be opened / parsed                 */
#define TSU_EPENDING 10 /* request not finished yet (tsu_poll)               */

/* Per-pair status values written by the engine. */
#define TSU_PAIR_OK 0
#define TSU_PAIR_SCRATCH 1 /* wavefront scratch exhausted at this config     */
#define TSU_PAIR_ARENA 2   /* CIGAR arena exhausted                          */
#define TSU_PAIR_INTERNAL 3

/* Flags for the align calls. */
#define TSU_SCORE_ONLY 0x1u  /* skip the CIGAR (the reference kernel's work) */
#define TSU_ONE_WARP 0x2u    /* one warp per pair in every pass, no warp groups and
                                no longest-first order: the reference's scheduling
                                (one 32-thread block per pair, wfa_gpu.cu:113-114),
                                kept as the "plain" baseline of the benchmarks */
#define TSU_BIDIRECTIONAL 0x4u /* one-piece gap-affine or a gap-linear metric
                                  (edit, indel, gap-linear: run as gap-affine
                                  with a zero gap opening), end to end:
                                  bidirectional WFA.  Each score is the lowest total at which a
                                  forward and a reverse wavefront pass cross (the
                                  breakpoint search, two rings per pair), about
                                  half the wavefront cells of the forward pass; the
                                  same scores.  CIGARs come from the recursion on
                                  crossings down to segments of at most
                                  max(2 max(x, o+e), 256 g) (g = gcd(x, o, e)),
                                  each aligned with its full history: memory
                                  linear in the score per pair.  WFA2-lib's
                                  ultralow memory mode; the reference keeps the
                                  default mode (wfa_gpu.cu:156-160) */

typedef struct tsu_ctx tsu_ctx;

typedef struct {
  int32_t mismatch;      /* > 0  (wfa_gpu.cu:59)  */
  int32_t gap_opening;   /* >= 0 (wfa_gpu.cu:60)  */
  int32_t gap_extension; /* > 0  (wfa_gpu.cu:61)  */
} tsu_penalties;

/* Dual gap-affine ("affine 2-pieces") penalties: a gap of length L costs
 * min(gap_opening + gap_extension*L, gap_opening2 + gap_extension2*L).  The
 * reference declares the second piece (penalties_t gap_open2 / gap_ext2,
 * common.h:80-87; matrices I2 / D2, common.h:52-58; backtrace codes
 * bt_I2_* / bt_D2_*, common.h:67-77) but aligns with one piece only.  In a
 * context made by tsu_create_dual every align call uses both pieces; pattern
 * and text lengths are then limited to 2^24 - 2. */
typedef struct {
  int32_t mismatch;       /* > 0  */
  int32_t gap_opening;    /* >= 0 */
  int32_t gap_extension;  /* > 0  */
  int32_t gap_opening2;   /* >= 0 */
  int32_t gap_extension2; /* > 0  */
} tsu_penalties2;

typedef struct {
  int32_t device;        /* CUDA device ordinal                                */
  int32_t reserved0;
  size_t mem_budget;     /* bytes of device memory the context may hold;
                            0 = 80% of the device's free memory at create    */
  double max_error_hint; /* expected worst per-pair edit rate used to size
                            wavefront scratch (0 = 0.20).  Pairs that exceed
                            it are retried with larger scratch, never dropped */
} tsu_config;

/* Host-side batch: sequences are byte strings at pattern + pattern_off[i]
 * (pattern_len[i] bytes) and text + text_off[i].  Any byte values are
 * accepted; A/C/G/T-only pairs take the 2-bit packed path. */
typedef struct {
  int64_t num_pairs;
  const char* pattern;
  const int64_t* pattern_off;
  const int32_t* pattern_len;
  const char* text;
  const int64_t* text_off;
  const int32_t* text_len;
} tsu_batch;

/* Results.  score[num_pairs] is required.  For CIGARs, cigar_offset has
 * num_pairs + 1 entries and pair i's runs are
 * cigar[cigar_offset[i] .. cigar_offset[i+1]).  If cigar_capacity (in runs)
 * is too small the call returns TSU_EOVERFLOW with scores filled and
 * cigar_needed set. */
typedef struct {
  int32_t* score;
  uint32_t* cigar;
  int64_t cigar_capacity;
  int64_t* cigar_offset;
  int64_t cigar_needed; /* out */
  int32_t* pair_status; /* optional [num_pairs], TSU_PAIR_* */
} tsu_result;

/* Timing of the last align call, measured with CUDA events on the context's
 * stream (milliseconds).  A call's fixed launch sequence (packing, the first
 * pass of every length band, counter read-back) runs as one CUDA graph kept
 * by the context and updated in place from call to call; set TSU_GRAPH=0 in
 * the environment before tsu_create to queue the same launches directly. */
typedef struct {
  double h2d_ms, pack_ms, align_ms, compact_ms, d2h_ms, total_ms;
  int64_t kernel_launches; /* kernels of this library launched by the call */
  int64_t retried_pairs;   /* pairs re-run with larger scratch            */
  int64_t h2d_bytes, d2h_bytes;
  int64_t cells; /* wavefront (score, diagonal) cells computed, all passes */
  int64_t steps; /* non-null score steps computed, all passes              */
  int64_t ext_bases; /* bases matched by extend steps, all passes         */
  int64_t device_bytes; /* most device memory the context's buffers held
                           during the call (the workspace carried over from
                           earlier calls included)                        */
} tsu_timing;

/* ---- context ------------------------------------------------------------
 * Replaces the reference's per-run setup: cudaDeviceReset + 12 cudaMalloc
 * (wfa_gpu.cu:96-108).  One context = one device, one stream, one memory
 * budget.  A context is used by one host thread at a time. */
int tsu_create(const tsu_penalties* pen, const tsu_config* cfg /* nullable */, tsu_ctx** out);
/* A context whose align calls use dual gap-affine penalties (tsu_penalties2).
 * Not available through tsu_align_scores_noalloc (one piece only). */
int tsu_create_dual(const tsu_penalties2* pen, const tsu_config* cfg /* nullable */, tsu_ctx** out);

/* Distance metrics -- WFA2-lib's distance_metric_t, which the reference sets
 * to gap_affine for its check (wfa_gpu.cu:157).  penalties[] holds, in order:
 *   TSU_METRIC_INDEL          none (gaps cost 1 per base; a mismatch is never
 *                             cheaper than a deletion plus an insertion, so the
 *                             CIGAR has no X)
 *   TSU_METRIC_EDIT           none (Levenshtein: mismatch and gap base cost 1)
 *   TSU_METRIC_GAP_LINEAR     mismatch, gap_extension (a gap of L costs e*L)
 *   TSU_METRIC_GAP_AFFINE     mismatch, gap_opening, gap_extension (tsu_create)
 *   TSU_METRIC_GAP_AFFINE_2P  mismatch, gap_opening, gap_extension,
 *                             gap_opening2, gap_extension2 (tsu_create_dual)
 * Indel, edit and gap-linear contexts run kernels with the M wavefront only
 * (no I/D components); their CIGARs resolve ties mismatch > deletion >
 * insertion. */
#define TSU_METRIC_INDEL 0
#define TSU_METRIC_EDIT 1
#define TSU_METRIC_GAP_LINEAR 2
#define TSU_METRIC_GAP_AFFINE 3
#define TSU_METRIC_GAP_AFFINE_2P 4
int tsu_create_metric(int metric, const int32_t* penalties /* nullable when none */, int num_penalties,
                      const tsu_config* cfg /* nullable */, tsu_ctx** out);
int tsu_destroy(tsu_ctx* ctx);
const char* tsu_status_str(int status);
const char* tsu_last_error(const tsu_ctx* ctx);
int tsu_get_timing(const tsu_ctx* ctx, tsu_timing* out);
/* The align passes of the last call (of its last chunk), e.g.
 * "s1x2368:200000@812.3ms s16x148:3120@4410.0ms": ring mode (s shared,
 * g global), warps per pair x pairs in flight : pairs, device time.  No
 * counterpart in the reference (one fixed launch, wfa_gpu.cu:118). */
const char* tsu_pass_log(const tsu_ctx* ctx);

/* ---- pass plan ------------------------------------------------------------
 * Pairs are aligned by length band (max(m, n) < 1024, < 2048, < 4096, < 8192,
 * < 16384, >= 16384 for bands 0..5); each band starts at a rung: the wavefront
 * ring in shared memory (mode 0) or in device memory (mode 1), with 1, 2, 4,
 * 8, 16 or 32 warps per pair.  A context starts from the table compiled in
 * (tsu_tuning.h, written by the autotuner tsunami_pact_b200/tune.py); these
 * calls read and change the context's copy.  Pairs that outgrow a rung are
 * retried at the next one, so a rung never changes a result.  No
 * counterpart in the reference (one fixed launch shape, wfa_gpu.cu:113-114). */
int tsu_set_band_start(tsu_ctx* ctx, int band, int mode, int warps_per_pair);

/* Ends-free alignment: WFA2-lib's alignment_span = ends_free
 * (wavefront_aligner_set_alignment_free_ends), which the reference leaves at
 * its end-to-end default (wfa_gpu.cu:156-160).  The alignment may start at
 * (v, 0) with v <= pattern_begin_free or at (0, h) with h <= text_begin_free
 * at no cost, and end at (m, h) with h >= n - text_end_free or at (v, n) with
 * v >= m - pattern_end_free.  The free end gaps stay in the CIGAR as I / D
 * runs (costing 0); of several ends at the optimal score the lowest diagonal
 * h - v wins.  All 0 (the default): end-to-end.  Every metric (gap-affine,
 * dual gap-affine, gap-linear, edit, indel -- e.g. semi-global edit distance
 * of a read against a longer region); applies to the context's later align
 * calls. */
int tsu_set_ends_free(tsu_ctx* ctx, int32_t pattern_begin_free, int32_t pattern_end_free, int32_t text_begin_free,
                      int32_t text_end_free);
int tsu_get_ends_free(const tsu_ctx* ctx, int32_t* out4);

/* Low-memory mode for the CIGAR of long or divergent pairs (the role of
 * WFA2-lib's memory modes, wavefront_memory_*; the reference keeps its
 * default, wfa_gpu.cu:156-160).  The backtrace history normally holds one
 * 4-byte word per wavefront cell of every score (about s^2 / e words for a
 * pair of score s).  With a checkpoint interval K the score pass keeps no
 * history but saves the wavefront ring every K scores; the backtrace then
 * recomputes the history K scores at a time, from the last segment to the
 * first, and walks each.  The CIGAR is the same; device memory per pair
 * falls to about (s / K) checkpoints plus K rows, for about twice the
 * compute.  checkpoint_interval: 0 off (default), > 0 K in score steps
 * (units of gcd of the penalties), < 0 chosen per pass (K near
 * sqrt(s * checkpoint size / row size)).  Low-memory passes run with the
 * wavefront ring in device memory. */
int tsu_set_low_memory(tsu_ctx* ctx, int32_t checkpoint_interval);
int tsu_get_band_start(const tsu_ctx* ctx, int band, int* mode, int* warps_per_pair);

/* ---- batch alignment, host buffers -------------------------------------
 * Replaces H2D + wfa_dispatcher launch + D2H of the reference
 * (wfa_gpu.cu:110-128) for arbitrary-length pairs, plus the CIGARs the
 * reference's WFA2-lib check computes (wfa_gpu.cu:164). */
int tsu_align_batch(tsu_ctx* ctx, const tsu_batch* batch, tsu_result* res, uint32_t flags);

/* Fixed-stride, equal-length layout of the reference host buffers
 * (wfa_gpu.cu:75-81): pair i is pattern + i*pattern_len and
 * text + i*text_len.  Scores only (the reference kernel's output,
 * short* score_d, wfa_gpu.cu:99,128 -- int32 here). */
int tsu_align_fixed(tsu_ctx* ctx, const char* pattern, const char* text, int64_t num_couples,
                    int32_t pattern_len, int32_t text_len, int32_t* score, uint32_t flags);

/* ---- batch alignment, device-resident buffers ---------------------------
 * Same as tsu_align_batch, but every pointer in batch and res is device
 * memory (res->cigar_offset must hold num_pairs + 1 entries; pair_status is
 * optional).  Work is queued on the context's stream and the call returns
 * when it is complete.  This is the entry a caller with resident data (or
 * the benchmark's kernel-time leg) uses; no host copies of sequence data. */
int tsu_align_batch_device(tsu_ctx* ctx, const tsu_batch* dev_batch, tsu_result* dev_res, uint32_t flags);

/* ---- scores without allocating -----------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * plug-ins whose host framework owns every device allocation through its own
 * pool, and services that must not block on, or fail in, the driver's
 * allocator in the middle of a request.
 * Same inputs as tsu_align_batch_device (device pointers), scores only, work
 * queued on `stream` (a cudaStream_t; NULL = default stream); the call reads
 * small counters back from the device on that stream and waits for its work
 * before it returns.  It allocates no device memory: its scratch is a fixed
 * 32 MiB array compiled into this library, held by every GPU that loads the
 * library until the process exits.  The first call on a device looks up that
 * array's device address (driver work, once per device).  All calls share
 * the one array: calls whose GPU work
 * overlaps race on it, so serialize them per device.  Batches needing more
 * than the array holds (about 55,000 pairs of 1 kbp, fewer for longer pairs;
 * also any batch whose longest pair's HBM wavefront ring would not fit beside
 * its packed input) return TSU_EOVERFLOW before any score is written; bad
 * lengths or penalties return TSU_EINVAL. */
int tsu_align_scores_noalloc(const tsu_penalties* pen, const tsu_batch* dev_batch, int32_t* dev_score, void* stream);

/* ---- render ------------------------------------------------------------
 * Expand run-length CIGAR runs into WFA2's one-char-per-operation string
 * (cigar->operations), or into the compact text form ("12M1X3I...").
 * Return the number of chars written (no terminator), or -1 if cap is too
 * small. */
int64_t tsu_cigar_to_ops(const uint32_t* runs, int64_t nruns, char* out, int64_t cap);
int64_t tsu_cigar_to_string(const uint32_t* runs, int64_t nruns, char* out, int64_t cap);

/* ---- input format (generate_dataset.cpp:39-41,68-69; read as in
 * wfa_gpu.cu:71-81) --------------------------------------------------------
 * sequences.txt: "N\nL\nerr\n" then N x (pattern line, text line).  Lines may
 * have any length up to the header L... or longer: each line is read at its
 * own length.  tsu_file_* hold the parsed batch in host memory -- page-locked
 * when a CUDA device is present, so tsu_align_batch copies it to the GPU at
 * full link speed; the file is read with parallel preads and tokenized in
 * parallel (the reference's reader is a single-threaded fscanf). */
typedef struct tsu_file tsu_file;
int tsu_file_read(const char* path, tsu_file** out);
/* Pairs from two FASTA or FASTQ files (either format, detected per file;
 * multi-line FASTA sequences are joined): record i of pattern_path is the
 * pattern of pair i, record i of text_path its text; the files must hold
 * the same number of records.  No counterpart in the reference (its only
 * input is sequences.txt).  tsu_file_header then gives the longest
 * sequence as seq_len and 0 as error_rate. */
int tsu_file_read_pairs(const char* pattern_path, const char* text_path, tsu_file** out);
int tsu_file_batch(const tsu_file* f, tsu_batch* out); /* views into f */
int tsu_file_header(const tsu_file* f, int64_t* num, int32_t* seq_len, int32_t* error_rate);
void tsu_file_free(tsu_file* f);

/* Seeded synthetic pairs (replaces generate_dataset.cpp:11-75).  Pattern:
 * i.i.d. uniform ACGT of length L; text: pattern with E = round(L*rate)
 * edits, floor(E/3) insertions, floor(E/3) deletions and the rest
 * substitutions at distinct uniform positions.  xoshiro256** seeded by
 * splitmix64(seed ^ pair index): each pair is reproducible on its own.
 * Writes into caller buffers: pattern/text bytes at pattern_off/text_off
 * (the caller sizes them from len_fn below). */
int tsu_gen_pair(uint64_t seed, int64_t pair_index, int32_t length, double error_rate, char* pattern_out,
                 int32_t* pattern_len, char* text_out, int32_t* text_len);

/* Many pairs at once on `threads` host threads (<= 0: all cores): pair i is
 * tsu_gen_pair(seed, first + i, lengths[i], rates[i], ...).  The text of a
 * pair has the pattern's length (equal insertion and deletion counts), so
 * each output slot needs lengths[i] bytes. */
int tsu_gen_batch(uint64_t seed, int64_t first, int64_t count, const int32_t* lengths, const double* rates,
                  char* pattern, const int64_t* pattern_off, int32_t* pattern_len, char* text,
                  const int64_t* text_off, int32_t* text_len, int threads);

/* Write a batch in the sequences.txt format (generate_dataset.cpp:39-41,
 * 68-69): header num / seq_len / error_rate, then pattern and text lines. */
int tsu_file_write(const char* path, int64_t num, int32_t seq_len, int32_t error_rate, const tsu_batch* batch);

/* Multi-GPU plan for one batch (host only, no device call).  The reference
 * aligns a file on one GPU in one launch (wfa_gpu.cu:113-123); pairs are
 * independent, so a batch splits into num_shards shards that separate GPUs
 * align with no communication, the results being put back in pair order on
 * the host.  Each pair's work is predicted from its lengths and edit rate
 * (max_error_hint > 0: that rate for every pair; 0: estimated per pair from
 * shared k-mers, which needs the sequence bytes) as the square of its
 * predicted score in extension steps plus its length; pairs are placed
 * largest first on the least-loaded shard.  Writes shard_of_pair[num_pairs]
 * and, when not NULL, shard_work[num_shards] (predicted work per shard).
 * Deterministic: every rank computes the same plan from the same batch. */
int tsu_shard_plan(const tsu_penalties* pen, const tsu_batch* batch, int32_t num_shards, double max_error_hint,
                   int32_t* shard_of_pair, double* shard_work);

/* ---- request server -------------------------------------------------------
 * No counterpart in the reference (one file per process, wfa_gpu.cu:43-188).
 * Continuous batching on one device: tsu_submit copies a request (a batch of
 * any size) into the server and returns at once; a pool of workers -- engine
 * contexts with their own streams and buffers -- runs jobs through the same
 * path as tsu_align_batch, and jobs overlap on the device.  Long pairs
 * (max(m, n) >= heavy_len) run as jobs of their own; the other pairs of the
 * oldest waiting requests are merged into shared jobs.  A job starts when a
 * worker is free and its predicted device memory (inputs, CIGAR arena,
 * wavefront scratch sized by max_error_hint and bounded by the
 * penalty-derived score bound of each pair) fits in mem_budget beside the
 * memory the other workers hold.  Long and other pairs each start in
 * submission order; a request is done when all its pairs are.
 * Scores and CIGARs of a request are the same alone and in any mix.
 * submit / poll / wait / cancel / stats may be called from any threads. */
typedef struct tsu_server tsu_server;

typedef struct {
  int32_t device;
  int32_t workers;          /* jobs in flight (engine contexts, one stream
                               each); 0 = 32.  Jobs overlap on the device only
                               as far as CUDA_DEVICE_MAX_CONNECTIONS hardware
                               queues allow: tsu_server_create sets it to 32
                               when unset, which takes effect if no CUDA work
                               ran in the process before                         */
  size_t mem_budget;        /* device bytes of all workers; 0 = 80% of free      */
  double max_error_hint;    /* edit rate sizing predicted wavefront memory (0 = 0.20);
                               pairs beyond it are retried, never dropped       */
  int64_t max_queue;        /* requests waiting to start before submit says
                               TSU_EBUSY (0 = 65536)                             */
  int64_t max_job_pairs;    /* light pairs merged into one job (0 = 16384)       */
  int32_t max_job_requests; /* requests merged into one job (0 = 64; 1 = none)   */
  int32_t heavy_len;        /* pairs with max(m, n) >= heavy_len run as jobs of
                               their own (0 = 8192; < 0 = never)                  */
  int32_t heavy_workers;    /* such jobs at once (0 = workers - 2, at least 1)   */
  int32_t estimate_hint;    /* 0: size each long pair's memory by its edit rate
                               estimated from shared k-mers (x 1.3 + 0.01);
                               < 0: by max_error_hint                            */
  double watchdog_ms;       /* a job running longer fails its requests with
                               TSU_ETIMEOUT (0 = off)                             */
  size_t resident_bytes;    /* device bytes an idle worker keeps for the next job
                               (0 = mem_budget / (2 * workers))                   */
} tsu_server_config;

/* Per-request timing, from tsu_poll / tsu_wait. */
typedef struct {
  int64_t num_pairs;
  double queue_ms;       /* submit -> its job started                      */
  double latency_ms;     /* submit -> result visible to poll / wait        */
  int32_t job_requests;  /* most requests merged into a job that delivered
                            some of its pairs                              */
  int32_t attempts;      /* most jobs one of its parts took (> 1 after a
                            retry)                                         */
  int64_t job_seq;       /* number of the job that started its first pairs;
                            jobs are numbered in the order they start      */
} tsu_request_info;

/* Counters since create or the last tsu_server_reset_stats; latencies are
 * those of completed requests (submit -> result visible). */
typedef struct {
  int64_t submitted, completed, failed, rejected, cancelled, timed_out;
  int64_t queued, running; /* requests now */
  int64_t jobs, pairs_completed;
  double mean_requests_per_job;
  double p50_ms, p99_ms, p999_ms, mean_ms, max_ms;
  double elapsed_s;
  uint64_t budget_bytes, granted_bytes, peak_granted_bytes;
  int32_t workers, reserved0;
  int64_t heavy_jobs;        /* jobs of one long pair                            */
  double busy_s;             /* worker time spent in jobs (all workers)          */
  double heavy_busy_s;       /* of which in jobs of one long pair                */
} tsu_server_stats;

int tsu_server_create(const tsu_penalties* pen, const tsu_server_config* cfg /* nullable */, tsu_server** out);
/* A server whose workers align with dual gap-affine penalties, or with any
 * metric of tsu_create_metric. */
int tsu_server_create_dual(const tsu_penalties2* pen, const tsu_server_config* cfg /* nullable */,
                           tsu_server** out);
int tsu_server_create_metric(int metric, const int32_t* penalties, int num_penalties,
                             const tsu_server_config* cfg /* nullable */, tsu_server** out);
/* Queued requests are dropped; running jobs finish first. */
int tsu_server_destroy(tsu_server* srv);
/* flags: TSU_SCORE_ONLY, TSU_BIDIRECTIONAL (gap-affine and gap-linear
 * servers; on a dual gap-affine one the request fails with TSU_EINVAL),
 * both, or 0; only requests of
 * the same flags share a job.  TSU_EINVAL for bad pairs, TSU_ENOMEM when the
 * request cannot fit the budget even alone, TSU_EBUSY when the queue is
 * full.  The caller's buffers may be reused when it returns. */
int tsu_submit(tsu_server* srv, const tsu_batch* request, uint32_t flags, uint64_t* id);
/* TSU_EPENDING until the request is done; then its results are copied into
 * res (as tsu_align_batch fills it; cigar_offset has num_pairs + 1 entries),
 * the request is forgotten and its status returned.  TSU_EOVERFLOW keeps the
 * request and sets res->cigar_needed.  info is optional. */
int tsu_poll(tsu_server* srv, uint64_t id, tsu_result* res, tsu_request_info* info);
/* tsu_poll after waiting up to timeout_ms (< 0: no limit); TSU_ETIMEOUT if
 * the request is still not done. */
int tsu_wait(tsu_server* srv, uint64_t id, double timeout_ms, tsu_result* res, tsu_request_info* info);
/* Drop a request: queued ones never run, running ones' results are
 * discarded.  TSU_ENOTFOUND for unknown ids. */
int tsu_cancel(tsu_server* srv, uint64_t id);
int tsu_server_get_stats(tsu_server* srv, tsu_server_stats* out);
int tsu_server_reset_stats(tsu_server* srv);
const char* tsu_server_last_error(tsu_server* srv);

/* Device bytes tsu_align_batch(ctx, batch, flags) holds at its peak, with
 * every pair of a length band in flight (*full) or one (*min); the server
 * admits requests by this prediction. */
int tsu_predict_bytes(tsu_ctx* ctx, const tsu_batch* batch, uint32_t flags, size_t* full, size_t* min);

#ifdef __cplusplus
}
#endif
#endif
