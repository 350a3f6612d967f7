// generate_dataset_main.cpp -- drop-in for the reference's generator
// (generate_dataset.cpp:11-75): `generate_dataset N L err [seed] [mode]`
// writes sequences.txt in the current directory in the same format
// (header N, L, err, then pattern and text lines).
//
// Unlike the reference (unseeded rand(), a data race on the error index,
// substitutions only, generate_dataset.cpp:32-37,56-61) the pairs are
// reproducible: pair i depends only on (seed, i).  mode "mixed" (default)
// splits the round(L*err/100) edits into equal insertion and deletion counts
// plus substitutions, so every text keeps length L; mode "sub" makes
// floor(L*err/100) substitutions only, like generate_dataset.cpp:23,56-66.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

#include "../../include/tsunami_b200.h"

int main(int argc, char* argv[]) {
  if (argc < 4) {  // generate_dataset.cpp:14-18
    std::cout << "Required arguments: number of couples, sequences length, error rate" << std::endl;
    exit(1);
  }
  const int64_t num = atoll(argv[1]);
  const int32_t L = atoi(argv[2]);
  const int32_t err = atoi(argv[3]);
  const uint64_t seed = argc > 4 ? strtoull(argv[4], nullptr, 0) : 0x5453554E414D49ull;
  const bool sub_only = argc > 5 && strcmp(argv[5], "sub") == 0;
  if (num < 0 || L < 0 || err < 0 || err > 100) {
    std::cout << "invalid arguments" << std::endl;
    return 1;
  }
  std::vector<char> pat((size_t)(num * L)), txt((size_t)(num * L));
  std::vector<int64_t> off((size_t)num);
  std::vector<int32_t> lens((size_t)num, L), plen((size_t)num), tlen((size_t)num);
  std::vector<double> rates((size_t)num);
  for (int64_t i = 0; i < num; ++i) off[(size_t)i] = i * (int64_t)L;
  if (sub_only) {
    // floor(L*err/100) substitutions: tsu_gen_pair's edit split is 1/3 each,
    // so generate with rate 0 and substitute here deterministically.
    for (auto& r : rates) r = 0.0;
  } else {
    for (auto& r : rates) r = err / 100.0;
  }
  int rc = tsu_gen_batch(seed, 0, num, lens.data(), rates.data(), pat.data(), off.data(), plen.data(), txt.data(),
                         off.data(), tlen.data(), 0);
  if (rc) {
    std::cout << "generation failed: " << tsu_status_str(rc) << std::endl;
    return 1;
  }
  if (sub_only) {
    const int64_t ne = ((int64_t)L * err) / 100;
    static const char A[4] = {'A', 'C', 'G', 'T'};
    uint64_t x = seed ^ 0xA5A5A5A5ull;
    for (int64_t i = 0; i < num; ++i) {
      char* t = txt.data() + i * L;
      for (int64_t j = 0; j < ne && L > 0; ++j) {
        // position j*L/ne spreads edits; base chosen by a splitmix step
        x += 0x9E3779B97F4A7C15ull;
        uint64_t z = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const int64_t p = (int64_t)((j * (int64_t)L) / ne + (int64_t)(z % (uint64_t)std::max<int64_t>(1, L / ne))) % L;
        const char old = t[p];
        char c = A[z >> 62];
        if (c == old) c = A[((z >> 62) + 1) & 3];
        t[p] = c;
      }
    }
  }
  tsu_batch b{num, pat.data(), off.data(), plen.data(), txt.data(), off.data(), tlen.data()};
  rc = tsu_file_write("sequences.txt", num, L, err, &b);
  if (rc) {
    std::cout << "cannot write sequences.txt" << std::endl;
    return 1;
  }
  return 0;
}
