// tsu_host.cpp -- host-side formats of the WFA engine: the sequences.txt
// reader (reference wfa_gpu.cu:71-81, format generate_dataset.cpp:39-41,
// 68-69), a FASTA/FASTQ pair reader, and the seeded synthetic pair
// generator that replaces generate_dataset.cpp:11-75.
//
// The reference reads its input with a single-threaded fscanf into pageable
// memory.  Here a file is read with parallel pread calls straight into
// page-locked memory (when a CUDA device is present: the engine's copies to
// the GPU then run at full link speed) and tokenized in parallel chunks.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/tsunami_b200.h"
#include "tsu_estimate.h"

namespace {

// Host bytes: page-locked when a CUDA device is present, else malloc'ed.
struct HostBytes {
  char* p = nullptr;
  size_t n = 0;
  bool pinned = false;
  HostBytes() = default;
  HostBytes(const HostBytes&) = delete;
  HostBytes& operator=(const HostBytes&) = delete;
  ~HostBytes() { reset(); }
  void reset() {
    if (p) {
      if (pinned)
        cudaFreeHost(p);
      else
        free(p);
    }
    p = nullptr;
    n = 0;
    pinned = false;
  }
  bool alloc(size_t bytes) {
    reset();
    const size_t b = std::max<size_t>(bytes, 1);
    int dev = 0;
    if (cudaGetDeviceCount(&dev) == cudaSuccess && dev > 0 &&
        cudaHostAlloc(reinterpret_cast<void**>(&p), b, cudaHostAllocPortable) == cudaSuccess) {
      pinned = true;
    } else {
      cudaGetLastError();
      p = static_cast<char*>(malloc(b));
      if (!p) return false;
    }
    n = bytes;
    return true;
  }
};

int reader_threads() {
  const unsigned h = std::thread::hardware_concurrency();
  return (int)std::min<unsigned>(std::max<unsigned>(h, 1), 32);
}

// Run fn(t) for t in [0, T) on T threads (the caller's thread runs t = 0).
template <class F>
void parallel(int T, F&& fn) {
  std::vector<std::thread> th;
  for (int t = 1; t < T; ++t) th.emplace_back([&, t] { fn(t); });
  fn(0);
  for (auto& x : th) x.join();
}

// Whole file into b (parallel preads).
bool read_file(const char* path, HostBytes* b) {
  const int fd = open(path, O_RDONLY);
  if (fd < 0) return false;
  struct stat stt {};
  if (fstat(fd, &stt) != 0 || stt.st_size < 0) {
    close(fd);
    return false;
  }
  const size_t size = (size_t)stt.st_size;
  if (!b->alloc(size)) {
    close(fd);
    return false;
  }
  const int T = size < (8u << 20) ? 1 : reader_threads();
  std::vector<char> ok((size_t)T, 1);
  parallel(T, [&](int t) {
    size_t off = size * (size_t)t / (size_t)T;
    const size_t end = size * (size_t)(t + 1) / (size_t)T;
    while (off < end) {
      const ssize_t r = pread(fd, b->p + off, end - off, (off_t)off);
      if (r <= 0) {
        ok[(size_t)t] = 0;
        return;
      }
      off += (size_t)r;
    }
  });
  close(fd);
  for (char v : ok)
    if (!v) return false;
  return true;
}

}  // namespace

struct tsu_file {
  int64_t num = 0;
  int32_t seq_len = 0, err = 0;
  HostBytes buf;  // file contents (sequences.txt) or the sequences themselves (FASTA/FASTQ)
  std::vector<int64_t> poff, toff;
  std::vector<int32_t> plen, tlen;
};

namespace {

inline bool is_space(unsigned char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == '\v' || c == '\f'; }

// Next whitespace-delimited token starting at *pos (like fscanf "%s").
bool next_token(const HostBytes& b, size_t* pos, size_t* start, size_t* len) {
  size_t i = *pos;
  const size_t n = b.n;
  while (i < n && is_space((unsigned char)b.p[i])) ++i;
  if (i >= n) return false;
  size_t j = i;
  while (j < n && !is_space((unsigned char)b.p[j])) ++j;
  *start = i;
  *len = j - i;
  *pos = j;
  return true;
}

bool parse_int(const HostBytes& b, size_t* pos, int64_t* out) {
  size_t s, l;
  if (!next_token(b, pos, &s, &l)) return false;
  char tmp[32];
  if (l >= sizeof tmp) return false;
  memcpy(tmp, b.p + s, l);
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
  auto* f = new tsu_file();
  if (!read_file(path, &f->buf)) {
    delete f;
    return TSU_EIO;
  }
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
  // Tokens after the header, found in parallel: chunk t lists the tokens
  // that start in its byte range; the chunks' lists in order are the file's.
  const char* p = f->buf.p;
  const size_t size = f->buf.n;
  const int T = size - pos < (8u << 20) ? 1 : reader_threads();
  std::vector<std::vector<std::pair<int64_t, int64_t>>> toks((size_t)T);
  parallel(T, [&](int t) {
    size_t i = pos + (size - pos) * (size_t)t / (size_t)T;
    const size_t end = pos + (size - pos) * (size_t)(t + 1) / (size_t)T;
    // a token starts at i when i follows whitespace: skip the tail of a token
    // begun in the previous chunk
    if (t > 0)
      while (i < end && !is_space((unsigned char)p[i - 1])) ++i;
    auto& v = toks[(size_t)t];
    while (i < end) {
      while (i < end && is_space((unsigned char)p[i])) ++i;
      if (i >= end) break;
      size_t j = i;
      while (j < size && !is_space((unsigned char)p[j])) ++j;  // a token may run past the chunk
      v.emplace_back((int64_t)i, (int64_t)(j - i));
      i = j;
    }
  });
  size_t have = 0;
  for (auto& v : toks) have += v.size();
  if (have < 2 * (size_t)num) {
    delete f;
    return TSU_EIO;
  }
  f->poff.resize((size_t)num);
  f->toff.resize((size_t)num);
  f->plen.resize((size_t)num);
  f->tlen.resize((size_t)num);
  size_t k = 0;  // token index: pair i is tokens 2i, 2i + 1 (exactly N pairs are read, as the reference does)
  for (auto& v : toks)
    for (auto& tk : v) {
      if (k >= 2 * (size_t)num) break;
      if (tk.second > (1 << 26)) {
        delete f;
        return TSU_EIO;
      }
      const size_t i = k >> 1;
      if (k & 1) {
        f->toff[i] = tk.first;
        f->tlen[i] = (int32_t)tk.second;
      } else {
        f->poff[i] = tk.first;
        f->plen[i] = (int32_t)tk.second;
      }
      ++k;
    }
  *out = f;
  return TSU_OK;
}

namespace {

// Records of a FASTA or FASTQ file: [start, end) of each record's sequence
// lines (line breaks included), in file order.  FASTA: a '>' header line,
// then sequence lines up to the next '>' at the start of a line.  FASTQ: an
// '@' header line, one sequence line, a '+' line, a quality line.  False on
// a malformed file.
bool index_records(const HostBytes& b, std::vector<std::pair<int64_t, int64_t>>* recs) {
  const char* p = b.p;
  const size_t n = b.n;
  size_t i = 0;
  while (i < n && is_space((unsigned char)p[i])) ++i;
  if (i >= n) return true;  // empty file: no records
  const char kind = p[i];
  if (kind != '>' && kind != '@') return false;
  auto line_end = [&](size_t a) {
    if (a >= n) return n;
    return (size_t)(std::find(p + a, p + n, '\n') - p);
  };
  if (kind == '@') {
    while (i < n) {
      if (p[i] != '@') return false;
      const size_t s0 = std::min(line_end(i) + 1, n), s1 = line_end(s0);
      const size_t plus = std::min(s1 + 1, n);
      if (plus >= n || p[plus] != '+') return false;
      const size_t q0 = std::min(line_end(plus) + 1, n), q1 = line_end(q0);
      recs->emplace_back((int64_t)s0, (int64_t)s1);
      i = std::min(q1 + 1, n);
      while (i < n && is_space((unsigned char)p[i])) ++i;
    }
    return true;
  }
  // FASTA records start at a '>' that begins a line; found in parallel
  const int T = n - i < (8u << 20) ? 1 : reader_threads();
  std::vector<std::vector<int64_t>> starts((size_t)T);
  parallel(T, [&](int t) {
    const size_t a = i + (n - i) * (size_t)t / (size_t)T, e = i + (n - i) * (size_t)(t + 1) / (size_t)T;
    for (size_t k = a; k < e; ++k)
      if (p[k] == '>' && (k == i || p[k - 1] == '\n')) starts[(size_t)t].push_back((int64_t)k);
  });
  std::vector<int64_t> all;
  for (auto& v : starts) all.insert(all.end(), v.begin(), v.end());
  for (size_t r = 0; r < all.size(); ++r) {
    const size_t s0 = std::min(line_end((size_t)all[r]) + 1, n);
    const size_t s1 = r + 1 < all.size() ? (size_t)all[r + 1] : n;
    recs->emplace_back((int64_t)s0, (int64_t)std::max(s0, s1));
  }
  return true;
}

// Each record's sequence without whitespace: lengths and offsets (from
// base) into len/off; with out, the bytes too (in parallel).
bool pack_records(const HostBytes& src, const std::vector<std::pair<int64_t, int64_t>>& recs, char* out,
                  int64_t base, std::vector<int64_t>* off, std::vector<int32_t>* len) {
  const size_t R = recs.size();
  off->resize(R);
  len->resize(R);
  std::vector<int64_t> l(R);
  const int T = R < 1024 ? 1 : reader_threads();
  parallel(T, [&](int t) {
    for (size_t r = R * (size_t)t / (size_t)T; r < R * (size_t)(t + 1) / (size_t)T; ++r) {
      int64_t c = 0;
      for (int64_t k = recs[r].first; k < recs[r].second; ++k) c += !is_space((unsigned char)src.p[k]);
      l[r] = c;
    }
  });
  int64_t acc = base;
  for (size_t r = 0; r < R; ++r) {
    if (l[r] > (1 << 26)) return false;
    (*off)[r] = acc;
    (*len)[r] = (int32_t)l[r];
    acc += l[r];
  }
  if (!out) return true;
  parallel(T, [&](int t) {
    for (size_t r = R * (size_t)t / (size_t)T; r < R * (size_t)(t + 1) / (size_t)T; ++r) {
      char* d = out + (*off)[r];
      for (int64_t k = recs[r].first; k < recs[r].second; ++k)
        if (!is_space((unsigned char)src.p[k])) *d++ = src.p[k];
    }
  });
  return true;
}

}  // namespace

int tsu_file_read_pairs(const char* pattern_path, const char* text_path, tsu_file** out) {
  if (!pattern_path || !text_path || !out) return TSU_EINVAL;
  *out = nullptr;
  HostBytes pf, tf;
  if (!read_file(pattern_path, &pf) || !read_file(text_path, &tf)) return TSU_EIO;
  std::vector<std::pair<int64_t, int64_t>> pr, tr;
  if (!index_records(pf, &pr) || !index_records(tf, &tr) || pr.size() != tr.size()) return TSU_EIO;
  auto* f = new tsu_file();
  std::vector<int64_t> po, to;
  std::vector<int32_t> pl, tl;
  // sizes first, then one buffer holding the patterns, then the texts
  if (!pack_records(pf, pr, nullptr, 0, &po, &pl)) {
    delete f;
    return TSU_EIO;
  }
  const int64_t pbytes = pr.empty() ? 0 : po.back() + pl.back();
  if (!pack_records(tf, tr, nullptr, pbytes, &to, &tl)) {
    delete f;
    return TSU_EIO;
  }
  const int64_t total = tr.empty() ? pbytes : to.back() + tl.back();
  if (!f->buf.alloc((size_t)total) || !pack_records(pf, pr, f->buf.p, 0, &po, &pl) ||
      !pack_records(tf, tr, f->buf.p, pbytes, &to, &tl)) {
    delete f;
    return TSU_EIO;
  }
  f->num = (int64_t)pr.size();
  int32_t longest = 0;
  for (size_t i = 0; i < pl.size(); ++i) longest = std::max({longest, pl[i], tl[i]});
  f->seq_len = longest;
  f->err = 0;
  f->poff = std::move(po);
  f->toff = std::move(to);
  f->plen = std::move(pl);
  f->tlen = std::move(tl);
  *out = f;
  return TSU_OK;
}

int tsu_file_batch(const tsu_file* f, tsu_batch* out) {
  if (!f || !out) return TSU_EINVAL;
  out->num_pairs = f->num;
  out->pattern = f->buf.p;
  out->pattern_off = f->poff.data();
  out->pattern_len = f->plen.data();
  out->text = f->buf.p;
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

// Predicted work of every pair, then longest-processing-time-first
// placement: pairs in decreasing work (ties by index) each go to the shard
// with the least work so far (ties to the lowest shard).  The result depends
// only on the inputs, so every rank that calls this gets the same plan.
int tsu_shard_plan(const tsu_penalties* pen, const tsu_batch* b, int32_t num_shards, double max_error_hint,
                   int32_t* shard_of_pair, double* shard_work) {
  if (!pen || !b || num_shards < 1 || b->num_pairs < 0 || !(max_error_hint >= 0.0) || max_error_hint > 2.0)
    return TSU_EINVAL;
  if (pen->mismatch <= 0 || pen->gap_opening < 0 || pen->gap_extension <= 0) return TSU_EINVAL;
  const int64_t n = b->num_pairs;
  if (n && (!shard_of_pair || !b->pattern_len || !b->text_len)) return TSU_EINVAL;
  const bool estimate = max_error_hint == 0.0;
  if (n && estimate && (!b->pattern || !b->pattern_off || !b->text || !b->text_off)) return TSU_EINVAL;
  for (int64_t i = 0; i < n; ++i)
    if (b->pattern_len[i] < 0 || b->text_len[i] < 0) return TSU_EINVAL;

  const double x = pen->mismatch, o = pen->gap_opening, e = pen->gap_extension;
  const double dear = std::max(x, o + e);  // dearest one-base edit
  std::vector<double> work((size_t)n);
  auto predict = [&](int64_t i) {
    const double m = b->pattern_len[i], t = b->text_len[i];
    // upper bound of the optimal score: mismatches plus one gap for the
    // length difference, or delete everything and insert everything
    const double ub = std::min(x * std::min(m, t) + (m != t ? o + e * std::fabs(m - t) : 0.0),
                               (m > 0 ? o + e * m : 0.0) + (t > 0 ? o + e * t : 0.0));
    double rate = max_error_hint;
    if (estimate) {
      rate = tsu::estimate_edit_rate(b->pattern + b->pattern_off[i], b->pattern_len[i], b->text + b->text_off[i],
                                     b->text_len[i]);
      if (rate < 0.0) rate = 0.1;  // too short to estimate: small either way
    }
    const double s = std::min(ub, rate * std::max(m, t) * dear);
    // wavefront cells grow with the square of the score (the envelope widens
    // by one diagonal per extension step); the packed sequences are read once
    const double steps = s / e + 1.0;
    work[(size_t)i] = steps * steps + (m + t) / 16.0;
  };
  int threads = estimate ? (int)std::max(1u, std::thread::hardware_concurrency()) : 1;
  threads = (int)std::min<int64_t>(threads, std::max<int64_t>(n / 256, 1));
  {
    std::vector<std::thread> th;
    auto run = [&](int tid) {
      for (int64_t i = tid; i < n; i += threads) predict(i);
    };
    for (int t = 1; t < threads; ++t) th.emplace_back(run, t);
    run(0);
    for (auto& t : th) t.join();
  }

  std::vector<int64_t> order((size_t)n);
  for (int64_t i = 0; i < n; ++i) order[(size_t)i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int64_t a, int64_t c) { return work[(size_t)a] > work[(size_t)c]; });
  // min-heap of (load, shard)
  std::vector<std::pair<double, int32_t>> heap;
  for (int32_t s = 0; s < num_shards; ++s) heap.emplace_back(0.0, s);
  auto later = [](const std::pair<double, int32_t>& a, const std::pair<double, int32_t>& c) {
    return a.first != c.first ? a.first > c.first : a.second > c.second;
  };
  std::make_heap(heap.begin(), heap.end(), later);
  std::vector<double> load((size_t)num_shards, 0.0);
  for (int64_t i : order) {
    std::pop_heap(heap.begin(), heap.end(), later);
    auto& top = heap.back();
    shard_of_pair[i] = top.second;
    top.first += work[(size_t)i];
    load[(size_t)top.second] = top.first;
    std::push_heap(heap.begin(), heap.end(), later);
  }
  if (shard_work)
    for (int32_t s = 0; s < num_shards; ++s) shard_work[s] = load[(size_t)s];
  return TSU_OK;
}

}  // extern "C"
