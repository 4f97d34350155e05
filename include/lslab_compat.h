// Source-compatible C++ front of the lsb C-ABI for callers written against
// depaulmillz/lslab's host API.  It covers the batched methods of
//   lslab::map<uint64_t, uint64_t>   (include/lslab/map.h:24-234)
//   lslab::set<uint32_t>             (include/lslab/set.h:21-134)
// with the same names, template block-size parameter, argument order and
// stream-ordered asynchronous behaviour, so code such as the reference's
// benchmark (benchmark/benchmark.cu:56-175) compiles against it unchanged.
//
// Differences a caller can observe:
//  * errors are reported: host-visible failures throw lslab::lsb_error
//    (the reference exits or traps, include/lslab/lslab.h:28-41);
//  * get() writes value 0 on a miss (the reference leaves it unwritten);
//  * a batch behaves as if its ops ran one at a time in index order (the
//    reference orders same-key ops only within a warp);
//  * the block_size template parameter is accepted and ignored: launch shapes
//    come from the table's tuning (lsb_map_set_tuning / the autotuner);
//  * the object owns its device memory and frees it on destruction (the
//    reference leaks, include/lslab/map.h:85-86), and it is not copyable
//    into kernels: there is no per-warp device API on this class.
#ifndef LSLAB_COMPAT_H
#define LSLAB_COMPAT_H

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

#include "lsb.h"

#if __has_include(<cuda/std/utility>)
#include <cuda/std/utility>
#define LSLAB_COMPAT_HAS_CUDA_PAIR 1
#endif

namespace lslab {

struct lsb_error : std::runtime_error {
  int code;
  lsb_error(int c, const char* what)
      : std::runtime_error(std::string(what) + ": " + lsb_error_string(c)), code(c) {}
};

inline void lsb_check(int code, const char* what) {
  if (code != LSB_OK) throw lsb_error(code, what);
}

// Overflow pool size for the constructor; the reference passes an allocator
// (device_allocator(stack_size), include/lslab/device_allocator.h:16).
struct pool_slabs {
  uint64_t count;
};

template <typename K, typename V>
class map;

template <>
class map<uint64_t, uint64_t> {
 public:
  map() : map(10) {}
  explicit map(unsigned n_log_2) : map(n_log_2, pool_slabs{0}) {}
  map(unsigned n_log_2, pool_slabs pool) {
    lsb_check(lsb_map_create(n_log_2, pool.count, &m_), "lsb_map_create");
  }
  ~map() {
    if (m_) lsb_map_destroy(m_);
  }
  map(const map&) = delete;
  map& operator=(const map&) = delete;
  map(map&& o) noexcept : m_(o.m_) { o.m_ = nullptr; }
  map& operator=(map&& o) noexcept {
    std::swap(m_, o.m_);
    return *this;
  }

#ifdef LSLAB_COMPAT_HAS_CUDA_PAIR
  // map.h:189-192
  template <int block_size = 256>
  void put(cuda::std::pair<uint64_t, uint64_t>* operations, uint64_t* output, size_t size,
           cudaStream_t stream = 0x0) {
    static_assert(sizeof(cuda::std::pair<uint64_t, uint64_t>) == sizeof(lsb_kv), "pair layout");
    lsb_check(lsb_map_put_pairs(m_, reinterpret_cast<const lsb_kv*>(operations), output, size,
                                stream),
              "lsb_map_put_pairs");
  }

  // map.h:208-211
  template <int block_size = 256>
  void get(uint64_t* operations, cuda::std::pair<bool, uint64_t>* output, size_t size,
           cudaStream_t stream = 0x0) {
    static_assert(sizeof(cuda::std::pair<bool, uint64_t>) == sizeof(lsb_result), "pair layout");
    lsb_check(lsb_map_get(m_, operations, reinterpret_cast<lsb_result*>(output), size, stream),
              "lsb_map_get");
  }
#endif

  // map.h:198-201
  template <int block_size = 256>
  void put(uint64_t* operations_keys, uint64_t* operations_values, uint64_t* output, size_t size,
           cudaStream_t stream = 0x0) {
    lsb_check(lsb_map_put(m_, operations_keys, operations_values, output, size, stream),
              "lsb_map_put");
  }

  template <int block_size = 256>
  void get(uint64_t* operations, lsb_result* output, size_t size, cudaStream_t stream = 0x0) {
    lsb_check(lsb_map_get(m_, operations, output, size, stream), "lsb_map_get");
  }

  // The REMOVE branch of detail::traverse (traverse.h:88-91), not exposed by
  // the reference map.
  template <int block_size = 256>
  void remove(uint64_t* operations, lsb_result* output, size_t size, cudaStream_t stream = 0x0) {
    lsb_check(lsb_map_remove(m_, operations, output, size, stream), "lsb_map_remove");
  }

  // map.h:225-227
  unsigned buckets() const { return lsb_map_buckets(m_); }

  lsb_map* handle() const { return m_; }

 private:
  lsb_map* m_ = nullptr;
};

template <typename K>
class set;

template <>
class set<uint32_t> {
 public:
  set() : set(10) {}
  explicit set(unsigned n_log_2) : set(n_log_2, pool_slabs{0}) {}
  set(unsigned n_log_2, pool_slabs pool) {
    lsb_check(lsb_set_create(n_log_2, pool.count, &s_), "lsb_set_create");
  }
  ~set() {
    if (s_) lsb_set_destroy(s_);
  }
  set(const set&) = delete;
  set& operator=(const set&) = delete;
  set(set&& o) noexcept : s_(o.s_) { o.s_ = nullptr; }
  set& operator=(set&& o) noexcept {
    std::swap(s_, o.s_);
    return *this;
  }

  // set.h:92-95
  template <int block_size = 256>
  void contains(const uint32_t* keys, bool* output, size_t size, cudaStream_t stream = 0x0) {
    lsb_check(lsb_set_contains(s_, keys, output, size, stream), "lsb_set_contains");
  }

  // set.h:103-106
  template <int block_size = 256>
  void insert(const uint32_t* keys, bool* output, size_t size, cudaStream_t stream = 0x0) {
    lsb_check(lsb_set_insert(s_, keys, output, size, stream), "lsb_set_insert");
  }

  // set.h:114-117
  template <int block_size = 256>
  void remove(const uint32_t* keys, bool* output, size_t size, cudaStream_t stream = 0x0) {
    lsb_check(lsb_set_remove(s_, keys, output, size, stream), "lsb_set_remove");
  }

  // set.h:125-127
  unsigned buckets() const { return lsb_set_buckets(s_); }

  lsb_set* handle() const { return s_; }

 private:
  lsb_set* s_ = nullptr;
};

}  // namespace lslab

#endif  // LSLAB_COMPAT_H
