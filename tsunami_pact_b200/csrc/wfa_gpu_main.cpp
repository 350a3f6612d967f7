// wfa_gpu_main.cpp -- drop-in for the reference's `wfa_gpu` command line
// (wfa_gpu.cu:43-188): same six positional arguments, same stdout lines.
//
//   wfa_gpu mismatch gap_opening gap_extension input_file wf_length check
//
// Differences, all on the safe side of the reference:
//   * wf_length is accepted for compatibility and ignored: wavefront
//     capacity is derived per pair (the reference overwrote neighbouring
//     slots when it was too small, wfa_gpu.cu:217,341);
//   * scores are int32 (no overflow above ~16 kbp), pairs may have unequal
//     lengths, any byte values are compared exactly;
//   * check=1 compares against a CPU aligner loaded at run time from the
//     shared library named by TSU_CHECK_LIB, which must export
//     tsu_check_align_scores (a WFA2-lib adapter, or this project's CPU
//     oracle, oracle/liboracle.so); the reference linked WFA2-lib directly
//     (wfa_gpu.cu:9-11,150-166).  Without TSU_CHECK_LIB, check=1 prints the
//     GPU lines, a message on stderr and exits with status 2.
//   * TSU_CIGAR_OUT=<path> additionally writes "score<TAB>cigar" per pair.
#include <dlfcn.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/tsunami_b200.h"

typedef int (*check_fn)(int64_t n, const char* pat, const int64_t* poff, const int32_t* plen, const char* txt,
                        const int64_t* toff, const int32_t* tlen, int x, int o, int e, int32_t* scores,
                        int threads);

int main(int argc, char const* argv[]) {
  if (argc != 7) {  // wfa_gpu.cu:45-48
    printf("ERROR! Please specify in order: mismatch, gap_opening, gap_extension, file name, wf_length, check\n");
    fprintf(stderr, "check=1 compares the GPU scores with the CPU aligner of the library named by TSU_CHECK_LIB "
                    "(exporting tsu_check_align_scores)\n");
    return 0;
  }
  const int mismatch = atoi(argv[1]);
  const int gap_opening = atoi(argv[2]);
  const int gap_extension = atoi(argv[3]);
  const char* path = argv[4];
  (void)atoi(argv[5]);  // wf_length: capacity is automatic
  const bool check = atoi(argv[6]) != 0;

  tsu_file* f = nullptr;
  int rc = tsu_file_read(path, &f);
  if (rc == TSU_EIO && !f) {
    FILE* probe = fopen(path, "r");
    if (!probe) {  // wfa_gpu.cu:66-69
      printf("ERROR: Cannot open file.\n");
      return 1;
    }
    fclose(probe);
    fprintf(stderr, "ERROR: malformed input file %s\n", path);
    return 1;
  }
  tsu_batch b;
  tsu_file_batch(f, &b);
  const int64_t n = b.num_pairs;

  tsu_penalties pen{mismatch, gap_opening, gap_extension};
  tsu_ctx* ctx = nullptr;
  rc = tsu_create(&pen, nullptr, &ctx);
  if (rc) {
    fprintf(stderr, "ERROR: tsu_create: %s\n", tsu_status_str(rc));
    tsu_file_free(f);
    return 1;
  }
  const char* cig_out = getenv("TSU_CIGAR_OUT");
  std::vector<int32_t> score((size_t)n);
  std::vector<int64_t> coff;
  std::vector<uint32_t> runs;
  tsu_result res{};
  res.score = score.data();
  uint32_t flags = TSU_SCORE_ONLY;
  if (cig_out) {
    flags = 0;
    coff.resize((size_t)n + 1);
    res.cigar_offset = coff.data();
    rc = tsu_align_batch(ctx, &b, &res, flags);
    if (rc == TSU_EOVERFLOW) {
      runs.resize((size_t)res.cigar_needed);
      res.cigar = runs.data();
      res.cigar_capacity = res.cigar_needed;
      rc = tsu_align_batch(ctx, &b, &res, flags);
    }
  } else {
    rc = tsu_align_batch(ctx, &b, &res, flags);
  }
  if (rc) {
    fprintf(stderr, "ERROR: alignment failed: %s (%s)\n", tsu_status_str(rc), tsu_last_error(ctx));
    tsu_destroy(ctx);
    tsu_file_free(f);
    return 1;
  }
  tsu_timing tm;
  tsu_get_timing(ctx, &tm);
  // Device time of the alignment work, excluding host<->device copies, as
  // the reference times launch + synchronize only (wfa_gpu.cu:116-126).
  const double gpu_s = (tm.pack_ms + tm.align_ms + tm.compact_ms) / 1e3;
  long double cells = 0;
  for (int64_t i = 0; i < n; ++i) cells += (long double)b.pattern_len[i] * (long double)b.text_len[i];
  long double gcups = cells / 1e9L / (long double)gpu_s;  // wfa_gpu.cu:130-133
  printf("GPU Time: %lf\n", gpu_s);
  printf("Estimated GCUPS GPU: : %Lf\n", gcups);
  fflush(stdout);

  if (cig_out) {
    FILE* fo = fopen(cig_out, "w");
    if (fo) {
      std::vector<char> s;
      for (int64_t i = 0; i < n; ++i) {
        const int64_t nr = coff[(size_t)i + 1] - coff[(size_t)i];
        s.resize((size_t)(nr * 12 + 1));
        int64_t w = tsu_cigar_to_string(runs.data() + coff[(size_t)i], nr, s.data(), (int64_t)s.size());
        fprintf(fo, "%d\t%.*s\n", score[(size_t)i], (int)(w < 0 ? 0 : w), s.data());
      }
      fclose(fo);
    }
  }

  int exit_code = 0;
  if (check) {
    const char* lib = getenv("TSU_CHECK_LIB");
    void* h = lib ? dlopen(lib, RTLD_NOW | RTLD_LOCAL) : nullptr;
    check_fn fn = h ? (check_fn)dlsym(h, "tsu_check_align_scores") : nullptr;
    if (!fn) {
      fprintf(stderr, "check=1 needs a CPU aligner: set TSU_CHECK_LIB to a library exporting tsu_check_align_scores%s%s\n",
              lib ? " (" : "", lib ? dlerror() : "");
      exit_code = 2;
    } else {
      std::vector<int32_t> cpu((size_t)n);
      auto t0 = std::chrono::high_resolution_clock::now();
      int crc = fn(n, b.pattern, b.pattern_off, b.pattern_len, b.text, b.text_off, b.text_len, mismatch, gap_opening,
                   gap_extension, cpu.data(), 0);
      auto t1 = std::chrono::high_resolution_clock::now();
      const double cpu_s = std::chrono::duration<double>(t1 - t0).count();
      long double gc = cells / 1e9L / (long double)cpu_s;
      printf("CPU Time: %lf\n", cpu_s);  // wfa_gpu.cu:174-175
      printf("Estimated GCUPS SW: %Lf\n", gc);
      bool equal = crc == 0;
      for (int64_t i = 0; i < n && equal; ++i)
        if (cpu[(size_t)i] != score[(size_t)i]) equal = false;
      if (equal)  // wfa_gpu.cu:183-184
        printf("\n\n                    |ALIGNEMENT FINISHED CORRECTLY|\n");
      else
        printf("\n\n |ERROR|\n");
    }
    // The plugin stays loaded until exit: unloading a library whose thread
    // pool (e.g. OpenMP workers) is still alive crashes the process.
  }
  tsu_destroy(ctx);
  tsu_file_free(f);
  return exit_code;
}
