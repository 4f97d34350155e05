// Host emulation of the CUDA execution model, for CPU tests of the library's
// device functions (test infrastructure; never linked into the library).
//
// Every thread of an emulated block is a host thread (of a reused pool).  __syncthreads is a
// barrier over the block; a warp intrinsic is an exchange through a per-warp
// buffer between two barriers over the warp's 32 threads, so every lane must
// take part (the library only uses full-warp masks).  Shared-memory variables
// become function statics, which is correct while one block runs at a time.
// Atomics are GCC __atomic builtins on host memory.
#pragma once

#include <atomic>
#include <barrier>
#include <cassert>
#include <cstdint>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define __noinline__
#define __launch_bounds__(...)
#define __shared__ static
#define __align__(n) alignas(n)

struct uint4 {
  uint32_t x, y, z, w;
};
struct ulonglong2 {
  unsigned long long x, y;
};
struct dim3 {
  unsigned x = 1, y = 1, z = 1;
};

inline thread_local dim3 threadIdx, blockIdx;
inline dim3 blockDim, gridDim;

namespace emu {

struct Block {
  std::unique_ptr<std::barrier<>> bar;
  std::vector<std::unique_ptr<std::barrier<>>> warp_bar;
  std::vector<uint64_t> buf;  // 32 words per warp
  std::atomic<int> or_flag{0};  // __syncthreads_or
};

inline thread_local Block* blk = nullptr;

inline uint64_t* wbuf() { return &blk->buf[(threadIdx.x >> 5) * 32]; }
inline void wsync() { blk->warp_bar[threadIdx.x >> 5]->arrive_and_wait(); }

template <class T>
inline uint64_t to64(T v) {
  static_assert(sizeof(T) <= 8, "warp exchange of at most 8 bytes");
  uint64_t r = 0;
  std::memcpy(&r, &v, sizeof(T));
  return r;
}
template <class T>
inline T from64(uint64_t r) {
  T v;
  std::memcpy(&v, &r, sizeof(T));
  return v;
}

// A pool of host threads, created once and reused for every block (creating
// a block's threads afresh per block dominated the run time under
// AddressSanitizer).  Worker t runs the posted block's f() as threadIdx.x = t.
class Pool {
 public:
  static Pool& get() {
    static Pool p;
    return p;
  }
  void run(unsigned nthreads, unsigned block, Block* b, const std::function<void()>& f) {
    std::unique_lock<std::mutex> lk(mu_);
    while (workers_.size() < nthreads) {
      const unsigned t = (unsigned)workers_.size();
      // gen_ is still the previous block's: the new worker takes this block
      workers_.emplace_back([this, t, g = gen_] { loop(t, g); });
    }
    job_ = &f;
    blk_ = b;
    block_ = block;
    active_ = nthreads;
    left_ = nthreads;
    ++gen_;
    start_.notify_all();
    done_.wait(lk, [this] { return left_ == 0; });
    job_ = nullptr;
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      ++gen_;
    }
    start_.notify_all();
    for (auto& w : workers_) w.join();
  }

 private:
  void loop(unsigned t, uint64_t seen) {
    for (;;) {
      const std::function<void()>* f;
      {
        std::unique_lock<std::mutex> lk(mu_);
        start_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
        if (t >= active_) continue;
        f = job_;
        threadIdx.x = t;
        blockIdx.x = block_;
        blk = blk_;
      }
      (*f)();
      std::lock_guard<std::mutex> lk(mu_);
      if (--left_ == 0) done_.notify_one();
    }
  }
  std::mutex mu_;
  std::condition_variable start_, done_;
  std::vector<std::thread> workers_;
  const std::function<void()>* job_ = nullptr;
  Block* blk_ = nullptr;
  unsigned block_ = 0, active_ = 0, left_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

// Runs f() on every thread of one block of `nthreads` (a multiple of 32).
template <class F>
void run_block(unsigned nthreads, unsigned block, unsigned nblocks, F&& f) {
  assert(nthreads % 32 == 0 && nthreads <= 1024);
  Block b;
  b.bar = std::make_unique<std::barrier<>>(nthreads);
  for (unsigned w = 0; w < nthreads / 32; ++w)
    b.warp_bar.push_back(std::make_unique<std::barrier<>>(32));
  b.buf.assign(nthreads, 0);
  blockDim.x = nthreads;
  gridDim.x = nblocks;
  const std::function<void()> job = [&] { f(); };
  Pool::get().run(nthreads, block, &b, job);
}

}  // namespace emu

inline void __syncthreads() { emu::blk->bar->arrive_and_wait(); }
inline int __syncthreads_or(int pred) {
  emu::Block* b = emu::blk;
  if (pred) b->or_flag.store(1);
  b->bar->arrive_and_wait();
  const int r = b->or_flag.load();
  b->bar->arrive_and_wait();
  if (threadIdx.x == 0) b->or_flag.store(0);
  b->bar->arrive_and_wait();
  return r;
}
inline void __threadfence() { __atomic_thread_fence(__ATOMIC_SEQ_CST); }
inline void __threadfence_block() { __atomic_thread_fence(__ATOMIC_SEQ_CST); }
inline void __nanosleep(unsigned) { std::this_thread::yield(); }

template <class T>
inline T __shfl_sync(unsigned mask, T v, int src) {
  assert(mask == 0xFFFFFFFFu);
  uint64_t* b = emu::wbuf();
  b[threadIdx.x & 31] = emu::to64(v);
  emu::wsync();
  const T r = emu::from64<T>(b[src & 31]);
  emu::wsync();
  return r;
}

template <class T>
inline T __shfl_up_sync(unsigned mask, T v, unsigned d) {
  assert(mask == 0xFFFFFFFFu);
  const unsigned lane = threadIdx.x & 31;
  uint64_t* b = emu::wbuf();
  b[lane] = emu::to64(v);
  emu::wsync();
  const T r = lane >= d ? emu::from64<T>(b[lane - d]) : v;
  emu::wsync();
  return r;
}

inline unsigned __ballot_sync(unsigned mask, int pred) {
  assert(mask == 0xFFFFFFFFu);
  uint64_t* b = emu::wbuf();
  b[threadIdx.x & 31] = pred ? 1 : 0;
  emu::wsync();
  unsigned r = 0;
  for (unsigned l = 0; l < 32; ++l) r |= (unsigned)(b[l] & 1) << l;
  emu::wsync();
  return r;
}

template <class T>
inline unsigned __match_any_sync(unsigned mask, T v) {
  assert(mask == 0xFFFFFFFFu);
  uint64_t* b = emu::wbuf();
  const uint64_t me = emu::to64(v);
  b[threadIdx.x & 31] = me;
  emu::wsync();
  unsigned r = 0;
  for (unsigned l = 0; l < 32; ++l) r |= (unsigned)(b[l] == me) << l;
  emu::wsync();
  return r;
}

namespace emu {
template <class Op>
inline unsigned reduce(unsigned mask, unsigned v, Op op) {
  assert(mask == 0xFFFFFFFFu);
  uint64_t* b = wbuf();
  b[threadIdx.x & 31] = v;
  wsync();
  unsigned r = (unsigned)b[0];
  for (unsigned l = 1; l < 32; ++l) r = op(r, (unsigned)b[l]);
  wsync();
  return r;
}
}  // namespace emu

inline unsigned __reduce_min_sync(unsigned m, unsigned v) {
  return emu::reduce(m, v, [](unsigned a, unsigned b) { return a < b ? a : b; });
}
inline unsigned __reduce_max_sync(unsigned m, unsigned v) {
  return emu::reduce(m, v, [](unsigned a, unsigned b) { return a > b ? a : b; });
}
inline unsigned __reduce_add_sync(unsigned m, unsigned v) {
  return emu::reduce(m, v, [](unsigned a, unsigned b) { return a + b; });
}

inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline unsigned __vcmpeq4(unsigned a, unsigned b) {
  unsigned r = 0;
  for (int i = 0; i < 4; ++i)
    if (((a >> (8 * i)) & 0xFF) == ((b >> (8 * i)) & 0xFF)) r |= 0xFFu << (8 * i);
  return r;
}
template <class T>
inline T min(T a, T b) {
  return a < b ? a : b;
}
template <class T>
inline T max(T a, T b) {
  return a > b ? a : b;
}

// The value operand converts to the pointee type, as CUDA's overloads do.
template <class T, class U>
inline T atomicAdd(T* p, U v) {
  return __atomic_fetch_add(p, (T)v, __ATOMIC_SEQ_CST);
}
template <class T, class U>
inline T atomicSub(T* p, U v) {
  return __atomic_fetch_sub(p, (T)v, __ATOMIC_SEQ_CST);
}
template <class T, class U>
inline T atomicAnd(T* p, U v) {
  return __atomic_fetch_and(p, (T)v, __ATOMIC_SEQ_CST);
}
template <class T, class U>
inline T atomicOr(T* p, U v) {
  return __atomic_fetch_or(p, (T)v, __ATOMIC_SEQ_CST);
}
template <class T, class U>
inline T atomicXor(T* p, U v) {
  return __atomic_fetch_xor(p, (T)v, __ATOMIC_SEQ_CST);
}
template <class T, class U>
inline T atomicExch(T* p, U v) {
  return __atomic_exchange_n(p, (T)v, __ATOMIC_SEQ_CST);
}
template <class T, class U, class V>
inline T atomicCAS(T* p, U cmp_in, V v) {
  T cmp = (T)cmp_in;
  __atomic_compare_exchange_n(p, &cmp, (T)v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return cmp;
}
template <class T, class U>
inline T atomicMin(T* p, U v_in) {
  const T v = (T)v_in;
  T cur = __atomic_load_n(p, __ATOMIC_SEQ_CST);
  while (v < cur && !__atomic_compare_exchange_n(p, &cur, v, false, __ATOMIC_SEQ_CST,
                                                 __ATOMIC_SEQ_CST)) {
  }
  return cur;
}
template <class T, class U>
inline T atomicMax(T* p, U v_in) {
  const T v = (T)v_in;
  T cur = __atomic_load_n(p, __ATOMIC_SEQ_CST);
  while (v > cur && !__atomic_compare_exchange_n(p, &cur, v, false, __ATOMIC_SEQ_CST,
                                                 __ATOMIC_SEQ_CST)) {
  }
  return cur;
}
