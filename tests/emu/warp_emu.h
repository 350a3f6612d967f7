// warp_emu.h -- runs the engine's CUDA kernel source on the CPU (test
// infrastructure).  Each lane is a std::thread; every warp collective
// (__syncwarp, __shfl_sync, __shfl_xor_sync, __reduce_*_sync, __any_sync,
// __ballot_sync) is a barrier over the lanes of that warp.  Dynamic shared memory and all
// buffers are exact-size heap blocks, so AddressSanitizer reports any access
// outside them.  Used to check the kernels' index arithmetic without a GPU.
#pragma once

#include <algorithm>
#include <barrier>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#define TSU_WARP_EMU 1
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __align__(x) alignas(x)

struct int2 {
  int x, y;
};
inline int2 make_int2(int a, int b) { return int2{a, b}; }
struct emu_dim3 {
  unsigned x = 0, y = 1, z = 1;
};

namespace emu {
inline thread_local emu_dim3 tid, bid;
inline emu_dim3 bdim, gdim;
inline unsigned char* smem_block = nullptr;

// Lane exchange slots, double-buffered by collective parity: a collective
// writes its lane's slot of the current parity, waits once, and reads.  A
// lane writes that parity again only two collectives later, after the
// barrier of the next collective, which no lane reaches before it has read
// this one -- so one barrier per collective suffices.  Every lane of a warp
// runs the same sequence of collectives (converged code), so the lanes'
// parities agree.
struct Warp {
  std::barrier<> bar{32};
  uint64_t slot[2][32];
};
inline std::vector<std::unique_ptr<Warp>> warps;
inline thread_local unsigned coll_parity = 0;

inline Warp& W() { return *warps[tid.x >> 5]; }
inline int lane() { return (int)(tid.x & 31); }
inline void syncwarp() { W().bar.arrive_and_wait(); }
// Publish this lane's value and wait for the warp; returns the slots of this
// collective.
inline const uint64_t* exchange(uint64_t v) {
  Warp& w = W();
  const unsigned p = coll_parity;
  coll_parity ^= 1u;
  w.slot[p][lane()] = v;
  w.bar.arrive_and_wait();
  return w.slot[p];
}
template <class T>
inline T shfl(T v, int src) {
  uint64_t b = 0;
  std::memcpy(&b, &v, sizeof(T));
  const uint64_t r = exchange(b)[src & 31];
  T out;
  std::memcpy(&out, &r, sizeof(T));
  return out;
}
template <class F>
inline uint64_t all_reduce(uint64_t v, F f) {
  const uint64_t* s = exchange(v);
  uint64_t acc = s[0];
  for (int i = 1; i < 32; ++i) acc = f(acc, s[i]);
  return acc;
}
inline int reduce_min(int v) {
  return (int)(int64_t)all_reduce((uint64_t)(int64_t)v, [](uint64_t a, uint64_t b) {
    return (uint64_t)std::min((int64_t)a, (int64_t)b);
  });
}
inline int reduce_max(int v) {
  return (int)(int64_t)all_reduce((uint64_t)(int64_t)v, [](uint64_t a, uint64_t b) {
    return (uint64_t)std::max((int64_t)a, (int64_t)b);
  });
}
inline unsigned reduce_add(unsigned v) {
  return (unsigned)all_reduce((uint64_t)v, [](uint64_t a, uint64_t b) { return (uint64_t)(uint32_t)(a + b); });
}
// the value of lane (this lane ^ m)
template <class T>
inline T shfl_xor(T v, int m) {
  uint64_t b = 0;
  std::memcpy(&b, &v, sizeof(T));
  const uint64_t r = exchange(b)[(lane() ^ m) & 31];
  T out;
  std::memcpy(&out, &r, sizeof(T));
  return out;
}
inline unsigned ballot(bool p) {
  const uint64_t* s = exchange(p ? 1u : 0u);
  unsigned r = 0;
  for (int i = 0; i < 32; ++i) r |= (s[i] ? 1u : 0u) << i;
  return r;
}
inline unsigned char* dyn_smem() { return smem_block; }

// Named barriers of the block (bar.sync id, nthreads): one std::barrier per
// (id, group of threads) -- the kernels use id = 1 + group index and the
// group's thread count, so the key is the id alone.
struct Named {
  std::unique_ptr<std::barrier<>> bar[16];
};
inline std::unique_ptr<Named> named;
inline void named_bar(int id, int nthreads) {
  static std::mutex mu;
  std::barrier<>* b;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto& slot = named->bar[id & 15];
    if (!slot) slot.reset(new std::barrier<>(nthreads));
    b = slot.get();
  }
  b->arrive_and_wait();
}

// Launch body() on blocks x threads lanes, block after block.
template <class F>
void launch(int blocks, int threads, size_t smem_bytes, F body) {
  gdim.x = (unsigned)blocks;
  bdim.x = (unsigned)threads;
  for (int b = 0; b < blocks; ++b) {
    unsigned char* sm = smem_bytes ? static_cast<unsigned char*>(std::malloc(smem_bytes)) : nullptr;
    if (sm) std::memset(sm, 0xA5, smem_bytes);
    smem_block = sm;
    warps.clear();
    for (int w = 0; w < threads / 32; ++w) warps.emplace_back(new Warp());
    named.reset(new Named());
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
      th.emplace_back([=] {
        tid.x = (unsigned)t;
        bid.x = (unsigned)b;
        body();
      });
    for (auto& x : th) x.join();
    std::free(sm);
    smem_block = nullptr;
  }
}
}  // namespace emu

#define threadIdx (emu::tid)
#define blockIdx (emu::bid)
#define blockDim (emu::bdim)
#define gridDim (emu::gdim)
#define __syncwarp(...) emu::syncwarp()
#define __shfl_sync(mask, v, src) emu::shfl((v), (src))
#define __shfl_xor_sync(mask, v, m) emu::shfl_xor((v), (m))
#define __reduce_min_sync(mask, v) emu::reduce_min(v)
#define __reduce_max_sync(mask, v) emu::reduce_max(v)
#define __reduce_add_sync(mask, v) emu::reduce_add(v)
#define __any_sync(mask, p) (emu::ballot(p) != 0u)
#define __ballot_sync(mask, p) emu::ballot(p)

inline unsigned atomicAdd(unsigned* p, unsigned v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
  return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
template <class T>
inline T __ldg(const T* p) {
  return *p;
}
inline uint32_t __funnelshift_r(uint32_t lo, uint32_t hi, uint32_t sh) {
  return (uint32_t)(((((uint64_t)hi) << 32) | lo) >> (sh & 31u));
}
inline int __ffs(int x) { return __builtin_ffs(x); }
inline int __ffs(uint32_t x) { return __builtin_ffs((int)x); }
inline int __ffsll(long long x) { return __builtin_ffsll(x); }
using std::max;
using std::min;
