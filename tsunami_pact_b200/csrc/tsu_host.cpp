// tsu_host.cpp -- host-side formats of the WFA engine: the sequences.txt
// reader (reference wfa_gpu.cu:71-81, format generate_dataset.cpp:39-41,
// 68-69) and the seeded synthetic pair generator that replaces
// generate_dataset.cpp:11-75.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/tsunami_b200.h"

struct tsu_file {
  int64_t num = 0;
  int32_t seq_len = 0, err = 0;
  std::vector<char> buf;  // file contents, tokens NUL-separated in place
  std::vector<int64_t> poff, toff;
  std::vector<int32_t> plen, tlen;
};

namespace {

inline bool is_space(unsigned char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == '\v' || c == '\f'; }

// Next whitespace-delimited token starting at *pos (like fscanf "%s").
bool next_token(const std::vector<char>& b, size_t* pos, size_t* start, size_t* len) {
  size_t i = *pos;
  const size_t n = b.size();
  while (i < n && is_space((unsigned char)b[i])) ++i;
  if (i >= n) return false;
  size_t j = i;
  while (j < n && !is_space((unsigned char)b[j])) ++j;
  *start = i;
  *len = j - i;
  *pos = j;
  return true;
}

bool parse_int(const std::vector<char>& b, size_t* pos, int64_t* out) {
  size_t s, l;
  if (!next_token(b, pos, &s, &l)) return false;
  char tmp[32];
  if (l >= sizeof tmp) return false;
  memcpy(tmp, &b[s], l);
  tmp[l] = 0;
  char* end = nullptr;
  long long v = strtoll(tmp, &end, 10);
  if (!end || *end) return false;
  *out = v;
  return true;
}

// splitmix64 / xoshiro256** (Vigna; public-domain reference algorithms).
inline uint64_t splitmix64(uint64_t* x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
struct Xoshiro {
  uint64_t s[4];
  explicit Xoshiro(uint64_t seed) {
    uint64_t x = seed;
    for (auto& v : s) v = splitmix64(&x);
  }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform in [0, n) by rejection (Lemire's multiply-shift)
  uint32_t below(uint32_t n) {
    uint64_t m = (uint64_t)(uint32_t)(next() >> 32) * n;
    uint32_t l = (uint32_t)m;
    if (l < n) {
      uint32_t t = (uint32_t)(-n) % n;
      while (l < t) {
        m = (uint64_t)(uint32_t)(next() >> 32) * n;
        l = (uint32_t)m;
      }
    }
    return (uint32_t)(m >> 32);
  }
};

const char kBases[4] = {'A', 'C', 'G', 'T'};

}  // namespace

static int tsu_gen_pair_impl(uint64_t seed, int64_t idx, int32_t L, double rate, char* pat, int32_t* plen, char* txt,
                      int32_t* tlen, std::vector<uint8_t>& kind) {
  if (L < 0 || rate < 0 || rate > 1 || !pat || !txt) return TSU_EINVAL;
  Xoshiro rng(seed ^ ((uint64_t)idx * 0xD1B54A32D192ED03ull + 0x5851F42D4C957F2Dull));
  for (int32_t i = 0; i < L; i += 32) {
    uint64_t r = rng.next();
    for (int j = 0; j < 32 && i + j < L; ++j) pat[i + j] = kBases[(r >> (2 * j)) & 3];
  }
  const int64_t E = std::min<int64_t>(L, (int64_t)std::llround((double)L * rate));
  const int64_t ni = E / 3, nd = E / 3;
  // E distinct positions: partial Fisher-Yates over kind[] used as a marker
  // array (0 = untouched, 1 = sub, 2 = ins, 3 = del).
  kind.assign((size_t)L, 0);
  std::vector<int32_t> pos;
  pos.reserve((size_t)E);
  while ((int64_t)pos.size() < E) {
    uint32_t p = rng.below((uint32_t)L);
    if (kind[p]) continue;
    kind[p] = 1;
    pos.push_back((int32_t)p);
  }
  // kinds shuffled over the positions: the first ni get ins, next nd del
  for (int64_t i = (int64_t)pos.size() - 1; i > 0; --i) {
    uint32_t j = rng.below((uint32_t)(i + 1));
    std::swap(pos[(size_t)i], pos[j]);
  }
  for (int64_t i = 0; i < E; ++i) kind[(size_t)pos[(size_t)i]] = i < ni ? 2 : (i < ni + nd ? 3 : 1);
  int32_t t = 0;
  for (int32_t i = 0; i < L; ++i) {
    switch (kind[(size_t)i]) {
      case 0: txt[t++] = pat[i]; break;
      case 1: {  // substitution: uniform among the 3 other bases
        const char c = pat[i];
        int ci = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : 3;
        txt[t++] = kBases[(ci + 1 + rng.below(3)) & 3];
        break;
      }
      case 2:  // insertion before pattern base i
        txt[t++] = kBases[rng.below(4)];
        txt[t++] = pat[i];
        break;
      case 3: break;  // deletion
    }
  }
  *plen = L;
  *tlen = t;
  return TSU_OK;
}

extern "C" {

int tsu_gen_pair(uint64_t seed, int64_t idx, int32_t L, double rate, char* pat, int32_t* plen, char* txt,
                 int32_t* tlen) {
  std::vector<uint8_t> kind;
  return tsu_gen_pair_impl(seed, idx, L, rate, pat, plen, txt, tlen, kind);
}

int tsu_gen_batch(uint64_t seed, int64_t first, int64_t count, const int32_t* lengths, const double* rates,
                  char* pat, const int64_t* pat_off, int32_t* pat_len, char* txt, const int64_t* txt_off,
                  int32_t* txt_len, int threads) {
  if (count < 0 || (count && (!lengths || !rates || !pat || !pat_off || !pat_len || !txt || !txt_off || !txt_len)))
    return TSU_EINVAL;
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  threads = (int)std::min<int64_t>(threads, std::max<int64_t>(count / 64, 1));
  std::vector<int> rcs((size_t)threads, TSU_OK);
  auto work = [&](int tid) {
    std::vector<uint8_t> kind;
    for (int64_t i = tid; i < count; i += threads) {
      int r = tsu_gen_pair_impl(seed, first + i, lengths[i], rates[i], pat + pat_off[i], &pat_len[i], txt + txt_off[i],
                                &txt_len[i], kind);
      if (r) rcs[(size_t)tid] = r;
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < threads; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& t : th) t.join();
  for (int r : rcs)
    if (r) return r;
  return TSU_OK;
}

int tsu_file_read(const char* path, tsu_file** out) {
  if (!path || !out) return TSU_EINVAL;
  *out = nullptr;
  FILE* fp = fopen(path, "rb");
  if (!fp) return TSU_EIO;
  auto* f = new tsu_file();
  if (fseek(fp, 0, SEEK_END) == 0) {
    long sz = ftell(fp);
    if (sz > 0) {
      f->buf.resize((size_t)sz);
      fseek(fp, 0, SEEK_SET);
      if (fread(f->buf.data(), 1, (size_t)sz, fp) != (size_t)sz) {
        fclose(fp);
        delete f;
        return TSU_EIO;
      }
    }
  }
  fclose(fp);
  size_t pos = 0;
  int64_t num = 0, len = 0, err = 0;
  if (!parse_int(f->buf, &pos, &num) || !parse_int(f->buf, &pos, &len) || !parse_int(f->buf, &pos, &err) || num < 0 ||
      len < 0) {
    delete f;
    return TSU_EIO;
  }
  f->num = num;
  f->seq_len = (int32_t)len;
  f->err = (int32_t)err;
  f->poff.resize((size_t)num);
  f->toff.resize((size_t)num);
  f->plen.resize((size_t)num);
  f->tlen.resize((size_t)num);
  for (int64_t i = 0; i < num; ++i) {
    size_t s, l;
    if (!next_token(f->buf, &pos, &s, &l) || l > (1u << 26)) {
      delete f;
      return TSU_EIO;
    }
    f->poff[(size_t)i] = (int64_t)s;
    f->plen[(size_t)i] = (int32_t)l;
    if (!next_token(f->buf, &pos, &s, &l) || l > (1u << 26)) {
      delete f;
      return TSU_EIO;
    }
    f->toff[(size_t)i] = (int64_t)s;
    f->tlen[(size_t)i] = (int32_t)l;
  }
  *out = f;
  return TSU_OK;
}

int tsu_file_batch(const tsu_file* f, tsu_batch* out) {
  if (!f || !out) return TSU_EINVAL;
  out->num_pairs = f->num;
  out->pattern = f->buf.data();
  out->pattern_off = f->poff.data();
  out->pattern_len = f->plen.data();
  out->text = f->buf.data();
  out->text_off = f->toff.data();
  out->text_len = f->tlen.data();
  return TSU_OK;
}

int tsu_file_header(const tsu_file* f, int64_t* num, int32_t* seq_len, int32_t* error_rate) {
  if (!f) return TSU_EINVAL;
  if (num) *num = f->num;
  if (seq_len) *seq_len = f->seq_len;
  if (error_rate) *error_rate = f->err;
  return TSU_OK;
}

void tsu_file_free(tsu_file* f) { delete f; }

int tsu_file_write(const char* path, int64_t num, int32_t seq_len, int32_t error_rate, const tsu_batch* b) {
  if (!path || !b) return TSU_EINVAL;
  FILE* fp = fopen(path, "wb");
  if (!fp) return TSU_EIO;
  std::vector<char> io(1 << 20);
  setvbuf(fp, io.data(), _IOFBF, io.size());
  fprintf(fp, "%lld\n%d\n%d\n", (long long)num, seq_len, error_rate);
  for (int64_t i = 0; i < num; ++i) {
    fwrite(b->pattern + b->pattern_off[i], 1, (size_t)b->pattern_len[i], fp);
    fputc('\n', fp);
    fwrite(b->text + b->text_off[i], 1, (size_t)b->text_len[i], fp);
    fputc('\n', fp);
  }
  int bad = ferror(fp);
  fclose(fp);
  return bad ? TSU_EIO : TSU_OK;
}

}  // extern "C"
