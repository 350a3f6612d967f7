/*
 * wfa_gen.c -- the seeded pair generator, restated for the CPU side.
 *
 * TEST INFRASTRUCTURE ONLY.  The engine library has its own generator
 * (tsu_gen_pair / tsu_gen_batch); this file gives bench.py's CPU reference
 * arm and the oracle-side fixture scripts the same pairs without loading the
 * engine library.  tests/test_readers.py checks that both produce identical
 * bytes for the same seeds.
 *
 * The data model replaces the reference's generator (generate_dataset.cpp:
 * 11-75, substitutions only, unseeded): an i.i.d. uniform ACGT pattern of
 * length L; text = pattern with E = round(L * rate) edits at distinct uniform
 * positions, floor(E/3) insertions, floor(E/3) deletions and the rest
 * substitutions (a substitution picks one of the three other bases, an
 * insertion a uniform base before the pattern base).  Randomness:
 * splitmix64-seeded xoshiro256** (Vigna, public-domain algorithms) with one
 * stream per pair index, uniform integers by Lemire's multiply-shift with
 * rejection.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "wfa_oracle.h"

static uint64_t gen_splitmix(uint64_t* x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

typedef struct {
  uint64_t s[4];
} gen_rng;

static uint64_t gen_rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

static void gen_seed(gen_rng* r, uint64_t seed) {
  uint64_t x = seed;
  for (int i = 0; i < 4; ++i) r->s[i] = gen_splitmix(&x);
}

static uint64_t gen_next(gen_rng* r) {
  uint64_t* s = r->s;
  const uint64_t out = gen_rotl(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = gen_rotl(s[3], 45);
  return out;
}

/* uniform in [0, n) */
static uint32_t gen_below(gen_rng* r, uint32_t n) {
  uint64_t m = (uint64_t)(uint32_t)(gen_next(r) >> 32) * n;
  uint32_t l = (uint32_t)m;
  if (l < n) {
    const uint32_t t = (uint32_t)(-n) % n;
    while (l < t) {
      m = (uint64_t)(uint32_t)(gen_next(r) >> 32) * n;
      l = (uint32_t)m;
    }
  }
  return (uint32_t)(m >> 32);
}

static const char gen_bases[4] = {'A', 'C', 'G', 'T'};

/* One pair; kind[] (L bytes) and pos[] (L ints) are scratch. */
static int gen_pair(uint64_t seed, int64_t idx, int32_t L, double rate, char* pat, int32_t* plen, char* txt,
                    int32_t* tlen, uint8_t* kind, int32_t* pos) {
  if (L < 0 || rate < 0 || rate > 1) return ORA_EINVAL;
  gen_rng rng;
  gen_seed(&rng, seed ^ ((uint64_t)idx * 0xD1B54A32D192ED03ull + 0x5851F42D4C957F2Dull));
  for (int32_t i = 0; i < L; i += 32) {
    const uint64_t r = gen_next(&rng);
    for (int j = 0; j < 32 && i + j < L; ++j) pat[i + j] = gen_bases[(r >> (2 * j)) & 3];
  }
  int64_t E = llround((double)L * rate);
  if (E > L) E = L;
  const int64_t ni = E / 3, nd = E / 3;
  memset(kind, 0, (size_t)L);
  int64_t np = 0;
  while (np < E) {
    const uint32_t p = gen_below(&rng, (uint32_t)L);
    if (kind[p]) continue;
    kind[p] = 1;
    pos[np++] = (int32_t)p;
  }
  for (int64_t i = np - 1; i > 0; --i) {
    const uint32_t j = gen_below(&rng, (uint32_t)(i + 1));
    const int32_t t = pos[i];
    pos[i] = pos[j];
    pos[j] = t;
  }
  for (int64_t i = 0; i < E; ++i) kind[pos[i]] = i < ni ? 2 : (i < ni + nd ? 3 : 1);
  int32_t t = 0;
  for (int32_t i = 0; i < L; ++i) {
    switch (kind[i]) {
      case 0:
        txt[t++] = pat[i];
        break;
      case 1: {
        const char c = pat[i];
        const int ci = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : 3;
        txt[t++] = gen_bases[(ci + 1 + (int)gen_below(&rng, 3)) & 3];
        break;
      }
      case 2:
        txt[t++] = gen_bases[gen_below(&rng, 4)];
        txt[t++] = pat[i];
        break;
      default:
        break;
    }
  }
  *plen = L;
  *tlen = t;
  return 0;
}

/* Pairs first .. first + count - 1 of the stream `seed`; pattern i is written
 * at pat + pat_off[i] (lengths[i] bytes), text i at txt + txt_off[i] (at most
 * lengths[i] + round(lengths[i] * rates[i]) bytes).  OpenMP over pairs. */
int ora_gen_batch(uint64_t seed, int64_t first, int64_t count, const int32_t* lengths, const double* rates, char* pat,
                  const int64_t* pat_off, int32_t* pat_len, char* txt, const int64_t* txt_off, int32_t* txt_len) {
  if (count < 0 || (count && (!lengths || !rates || !pat || !pat_off || !pat_len || !txt || !txt_off || !txt_len)))
    return ORA_EINVAL;
  int32_t lmax = 0;
  for (int64_t i = 0; i < count; ++i) {
    if (lengths[i] < 0) return ORA_EINVAL;
    if (lengths[i] > lmax) lmax = lengths[i];
  }
  int rc = 0;
#pragma omp parallel
  {
    uint8_t* kind = (uint8_t*)malloc((size_t)lmax + 1);
    int32_t* pos = (int32_t*)malloc(sizeof(int32_t) * ((size_t)lmax + 1));
    if (!kind || !pos) {
#pragma omp atomic write
      rc = ORA_ENOMEM;
    } else {
#pragma omp for schedule(dynamic, 64)
      for (int64_t i = 0; i < count; ++i) {
        const int r = gen_pair(seed, first + i, lengths[i], rates[i], pat + pat_off[i], &pat_len[i], txt + txt_off[i],
                               &txt_len[i], kind, pos);
        if (r) {
#pragma omp atomic write
          rc = r;
        }
      }
    }
    free(kind);
    free(pos);
  }
  return rc;
}
