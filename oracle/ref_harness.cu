// ref_harness.cu -- runs the reference's own GPU kernel on seeded pairs.
//
// TEST INFRASTRUCTURE ONLY: it produces reference-run scores that pin this
// project's oracle and engine to the reference (the committed fixture is
// tests/golden/ref_scores.json, written by tests/golden/make_ref_scores.py).
//
// The kernel is the reference's wfa_dispatcher, compiled unchanged from
// wfa_gpu.cu by oracle/ref_build.sh (its main is renamed so this file owns
// main).  This harness replaces the reference's host driver
// (wfa_gpu.cu:43-135) with one that keeps its launch arguments
// (max_score = max(o+e, x) + 1 ring slots, one 32-thread block per pair,
// wfa_gpu.cu:83-120) but:
//   * generates the pairs with the seeded generator (ora_gen_batch) instead
//     of reading sequences.txt, all of one length (the kernel's layout);
//   * pads the pattern and text buffers (2 * len + 256 bytes before and
//     after, filled with bytes outside ACGT that differ between pattern and
//     text) because the kernel reads past its pairs' ends;
//   * clears the limits words the kernel never initialises;
//   * runs the CPU model of the kernel (ora_refk_batch) FIRST and launches
//     nothing unless every pair is certified: all wavefront indices inside
//     the pair's ring, all reads inside the padded buffers, an end within the
//     step cap.  The kernel has no bounds checks and no step limit of its
//     own.
//
// Usage: ref_harness x o e seed first num len rate wf_length step_cap out [reps]
//   wf_length 0: 2 * (len + 3) + 2, wide enough that no access leaves its
//   slot.  Writes "pair gpu_score model_score" lines to `out` and one summary
//   line (JSON) to stdout: kernel time (CUDA events, mean of reps launches)
//   and GCUPS by the reference's formula (wfa_gpu.cu:130-133).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "wfa_oracle.h"

__global__ void wfa_dispatcher(char* pattern_d, char* text_d, short* score_d, short* mwavefronts_d,
                               short* iwavefronts_d, short* dwavefronts_d, int max_op, int num_couples,
                               bool* nullm_d, bool* nulli_d, bool* nulld_d, short* limitsm_d, short* limitsi_d,
                               short* limitsd_d, int pattern_len, int text_len, int num_wavefronts, int wf_length,
                               int max_score, short mismatch, short gap_opening, short gap_extension, int hi, int lo);

#define HCHECK(call)                                                                      \
  do {                                                                                    \
    const cudaError_t err_ = (call);                                                      \
    if (err_ != cudaSuccess) {                                                            \
      fprintf(stderr, "ref_harness: %s at %s:%d\n", cudaGetErrorString(err_), __FILE__, __LINE__); \
      return 4;                                                                           \
    }                                                                                     \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 12) {
    fprintf(stderr, "usage: ref_harness x o e seed first num len rate wf_length step_cap out [reps]\n");
    return 2;
  }
  const int x = atoi(argv[1]), o = atoi(argv[2]), e = atoi(argv[3]);
  const uint64_t seed = strtoull(argv[4], nullptr, 0);
  const int64_t first = atoll(argv[5]), num = atoll(argv[6]);
  const int len = atoi(argv[7]);
  const double rate = atof(argv[8]);
  int wf = atoi(argv[9]);
  const int step_cap = std::min(atoi(argv[10]), 32000);
  const char* out_path = argv[11];
  const int reps = argc > 12 ? std::max(1, atoi(argv[12])) : 1;
  if (num <= 0 || len <= 0 || x < 0 || o < 0 || e <= 0 || x > o + e) {
    // x > o + e: the kernel reads M[s - x] before s >= x (wfa_gpu.cu:626)
    fprintf(stderr, "ref_harness: need num, len > 0 and 0 <= x <= o + e\n");
    return 2;
  }
  if (wf <= 0) wf = 2 * (len + 3) + 2;
  const int nw = std::max(o + e, x) + 1;  // wfa_gpu.cu:83-84
  if ((int64_t)nw * wf > 32767) {
    fprintf(stderr, "ref_harness: %d slots x wf_length %d overflow the kernel's short slot base\n", nw, wf);
    return 2;
  }

  // pairs
  std::vector<int32_t> lens((size_t)num, len), plen((size_t)num), tlen((size_t)num);
  std::vector<double> rates((size_t)num, rate);
  std::vector<int64_t> off((size_t)num);
  for (int64_t i = 0; i < num; ++i) off[(size_t)i] = i * (int64_t)len;
  const int64_t pad = 2 * (int64_t)len + 256;
  const size_t bytes = (size_t)(pad + num * (int64_t)len + pad);
  std::vector<char> P(bytes, (char)1), T(bytes, (char)2);
  if (ora_gen_batch(seed, first, num, lens.data(), rates.data(), P.data() + pad, off.data(), plen.data(),
                    T.data() + pad, off.data(), tlen.data()) != 0) {
    fprintf(stderr, "ref_harness: generator failed\n");
    return 2;
  }
  for (int64_t i = 0; i < num; ++i)
    if (plen[(size_t)i] != len || tlen[(size_t)i] != len) {
      fprintf(stderr, "ref_harness: pair %lld is not %d x %d\n", (long long)i, len, len);
      return 2;
    }

  // certification by the CPU model
  std::vector<int16_t> model((size_t)num);
  std::vector<int32_t> codes((size_t)num), steps((size_t)num), maxk((size_t)num);
  if (ora_refk_batch(P.data() + pad, T.data() + pad, pad, pad, num, len, x, o, e, wf, step_cap, model.data(),
                     codes.data(), steps.data(), maxk.data()) != 0) {
    fprintf(stderr, "ref_harness: model failed\n");
    return 2;
  }
  int64_t uncertified = 0;
  for (int64_t i = 0; i < num; ++i)
    if (codes[(size_t)i]) {
      if (uncertified < 10) fprintf(stderr, "not certified: pair %lld code %d\n", (long long)i, codes[(size_t)i]);
      ++uncertified;
    }
  if (uncertified) {
    fprintf(stderr, "ref_harness: %lld pairs not certified; nothing launched\n", (long long)uncertified);
    return 3;
  }

  // the reference's launch arguments (wfa_gpu.cu:83-94,113-120)
  const int max_score = std::max(o + e, x) + 1;
  const int max_op = 2 * (len + len);
  int hi = 0, lo = 0;
  const int eff_lo = lo - (max_score + 1), eff_hi = hi + (max_score + 1);
  lo = std::min(eff_lo, 0);
  hi = std::max(eff_hi, 0);
  const size_t ring = (size_t)nw * (size_t)wf * (size_t)num;
  char *pd = nullptr, *td = nullptr;
  short *sd = nullptr, *md = nullptr, *id = nullptr, *dd = nullptr, *lmd = nullptr, *lid = nullptr, *ldd = nullptr;
  bool *nmd = nullptr, *nid = nullptr, *ndd = nullptr;
  HCHECK(cudaMalloc(&pd, bytes));
  HCHECK(cudaMalloc(&td, bytes));
  HCHECK(cudaMalloc(&sd, sizeof(short) * (size_t)num));
  HCHECK(cudaMalloc(&md, sizeof(short) * ring));
  HCHECK(cudaMalloc(&id, sizeof(short) * ring));
  HCHECK(cudaMalloc(&dd, sizeof(short) * ring));
  HCHECK(cudaMalloc(&nmd, (size_t)nw * (size_t)num));
  HCHECK(cudaMalloc(&nid, (size_t)nw * (size_t)num));
  HCHECK(cudaMalloc(&ndd, (size_t)nw * (size_t)num));
  const size_t limb = sizeof(short) * 4 * (size_t)nw * (size_t)num;
  HCHECK(cudaMalloc(&lmd, limb));
  HCHECK(cudaMalloc(&lid, limb));
  HCHECK(cudaMalloc(&ldd, limb));
  HCHECK(cudaMemcpy(pd, P.data(), bytes, cudaMemcpyHostToDevice));
  HCHECK(cudaMemcpy(td, T.data(), bytes, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  HCHECK(cudaEventCreate(&e0));
  HCHECK(cudaEventCreate(&e1));
  std::vector<int16_t> gpu((size_t)num), first_run((size_t)num);
  double total_ms = 0.0, wall_s = 0.0;
  for (int r = 0; r < reps; ++r) {
    // every launch starts from the state the model assumes
    HCHECK(cudaMemset(lmd, 0, limb));
    HCHECK(cudaMemset(lid, 0, limb));
    HCHECK(cudaMemset(ldd, 0, limb));
    HCHECK(cudaMemset(nmd, 0, (size_t)nw * (size_t)num));
    HCHECK(cudaMemset(nid, 0, (size_t)nw * (size_t)num));
    HCHECK(cudaMemset(ndd, 0, (size_t)nw * (size_t)num));
    HCHECK(cudaMemset(sd, 0, sizeof(short) * (size_t)num));
    HCHECK(cudaDeviceSynchronize());
    const auto w0 = std::chrono::high_resolution_clock::now();
    HCHECK(cudaEventRecord(e0));
    wfa_dispatcher<<<(unsigned)num, 32>>>(pd + pad, td + pad, sd, md, id, dd, max_op, (int)num, nmd, nid, ndd, lmd,
                                          lid, ldd, len, len, nw, wf, max_score, (short)x, (short)o, (short)e, hi, lo);
    HCHECK(cudaGetLastError());
    HCHECK(cudaEventRecord(e1));
    HCHECK(cudaEventSynchronize(e1));
    const auto w1 = std::chrono::high_resolution_clock::now();
    float ms = 0.f;
    HCHECK(cudaEventElapsedTime(&ms, e0, e1));
    total_ms += ms;
    wall_s += std::chrono::duration<double>(w1 - w0).count();
    HCHECK(cudaMemcpy(gpu.data(), sd, sizeof(short) * (size_t)num, cudaMemcpyDeviceToHost));
    if (r == 0) {
      first_run = gpu;
    } else if (gpu != first_run) {
      fprintf(stderr, "ref_harness: launch %d gave different scores than the first\n", r);
      return 5;
    }
  }
  FILE* f = fopen(out_path, "w");
  if (!f) {
    fprintf(stderr, "ref_harness: cannot write %s\n", out_path);
    return 2;
  }
  int64_t diff = 0;
  int32_t kmax = 0;
  for (int64_t i = 0; i < num; ++i) {
    fprintf(f, "%lld %d %d\n", (long long)i, (int)first_run[(size_t)i], (int)model[(size_t)i]);
    diff += first_run[(size_t)i] != model[(size_t)i];
    kmax = std::max(kmax, maxk[(size_t)i]);
  }
  fclose(f);
  const double ms = total_ms / reps;
  const double gcups = (double)len * (double)len * (double)num / (ms / 1e3) / 1e9;
  printf("{\"num\": %lld, \"len\": %d, \"rate\": %g, \"seed\": %llu, \"first\": %lld, \"wf_length\": %d, "
         "\"max_abs_k\": %d, \"kernel_ms\": %.4f, \"wall_s\": %.6f, \"reps\": %d, \"gcups\": %.4f, "
         "\"gpu_vs_model_diff\": %lld}\n",
         (long long)num, len, rate, (unsigned long long)seed, (long long)first, wf, kmax, ms, wall_s / reps, reps,
         gcups, (long long)diff);
  cudaFree(pd), cudaFree(td), cudaFree(sd), cudaFree(md), cudaFree(id), cudaFree(dd);
  cudaFree(nmd), cudaFree(nid), cudaFree(ndd), cudaFree(lmd), cudaFree(lid), cudaFree(ldd);
  return 0;
}
