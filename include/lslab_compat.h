// Source-compatible C++ front of the lsb C-ABI for callers written against
// depaulmillz/lslab's host API.  It covers the batched methods of
//   lslab::map<K, V>   (include/lslab/map.h:24-234), K a 64-bit unsigned
//                      integer, V a 32- or 64-bit unsigned integer;
//   lslab::set<K>      (include/lslab/set.h:21-134), K a 32-bit unsigned
//                      integer, including the thrust::device_vector overloads
//                      (set.h:97-123) when compiled by nvcc with thrust;
// with the same names, template block-size parameter, argument order and
// stream-ordered asynchronous behaviour, the constructors map(n_log_2) and
// map(n_log_2, Allocator&&) (map.h:43-66; device_allocator(stack_size) gives
// the overflow pool's size), and the gpuErrchk macro (lslab.h:28-41).  The
// headers under include/compat/lslab/ map the reference's include paths
// (<lslab/map.h>, <lslab/set.h>, ...) here, so a caller such as the
// reference's own benchmark (benchmark/benchmark.cu) compiles against this
// library unchanged with -I include/compat.
//
// Differences a caller can observe:
//  * errors are reported: host-visible failures throw lslab::lsb_error
//    (the reference exits or traps, include/lslab/lslab.h:28-41);
//  * get() writes value 0 on a miss (the reference leaves it unwritten);
//  * update() is update-if-present returning {present, old value} (the
//    reference's batched update calls put, detail/map_kernels.h:85);
//  * a batch behaves as if its ops ran one at a time in index order (the
//    reference orders same-key ops only within a warp);
//  * the block_size template parameter is accepted and ignored, and so are
//    the Allocator and Hash types beyond the pool size: launch shapes come
//    from the table's tuning and the hash is the library's own;
//  * the object owns its device memory and frees it on destruction (the
//    reference leaks, include/lslab/map.h:85-86), and it is not copyable
//    into kernels: there is no per-warp device API on this class.
#ifndef LSLAB_COMPAT_H
#define LSLAB_COMPAT_H

#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include "lsb.h"

#if __has_include(<cuda/std/utility>)
#include <cuda/std/utility>
#define LSLAB_COMPAT_HAS_CUDA_PAIR 1
#endif
#if defined(__CUDACC__) && __has_include(<thrust/device_vector.h>)
#include <thrust/device_vector.h>
#define LSLAB_COMPAT_HAS_THRUST 1
#endif

// lslab.h:28-41: abort with a message on a failed CUDA runtime call.
#ifndef gpuErrchk
#define gpuErrchk(ans) \
  { lslab::gpuAssert_slab((ans), __FILE__, __LINE__); }
#endif

namespace lslab {

inline void gpuAssert_slab(cudaError_t code, const char* file, int line, bool abort = true) {
  if (code != cudaSuccess) {
    std::fprintf(stderr, "GPUassert: %s %s %d\n", cudaGetErrorString(code), file, line);
    if (abort) std::exit(code);
  }
}

struct lsb_error : std::runtime_error {
  int code;
  lsb_error(int c, const char* what)
      : std::runtime_error(std::string(what) + ": " + lsb_error_string(c)), code(c) {}
};

inline void lsb_check(int code, const char* what) {
  if (code != LSB_OK) throw lsb_error(code, what);
}

namespace detail {
// Names the reference's allocator is instantiated with
// (device_allocator<detail::slab_node<K, V>>); only the names are needed.
template <typename K, typename V>
struct slab_node;
template <typename K>
struct set_node;
}  // namespace detail

// include/lslab/device_allocator.h:13-34: here only the pool size it
// carries, in slabs (the reference's default is 10000).
template <typename T>
struct device_allocator {
  explicit device_allocator(size_t stack_size_ = 10000) : stack_size(stack_size_) {}
  size_t stack_size;
};

// include/lslab/hash.h:10-15; accepted for source compatibility, unused.
template <typename T>
struct hash {
  size_t operator()(T x) const { return static_cast<size_t>(x); }
};

// Overflow pool size for the constructor without the reference's allocator type.
struct pool_slabs {
  uint64_t count;
};

template <typename K, typename V,
          typename Allocator = device_allocator<detail::slab_node<K, V>>,
          typename Hash = hash<K>>
class map {
  static_assert(std::is_integral<K>::value && std::is_unsigned<K>::value && sizeof(K) == 8,
                "lsb maps take 64-bit unsigned integer keys");
  static_assert(std::is_integral<V>::value && std::is_unsigned<V>::value &&
                    (sizeof(V) == 8 || sizeof(V) == 4),
                "lsb maps take 32- or 64-bit unsigned integer values");
  static constexpr bool kV32 = sizeof(V) == 4;
  using R = typename std::conditional<kV32, lsb_result32, lsb_result>::type;
  using KV = typename std::conditional<kV32, lsb_kv32, lsb_kv>::type;

  static const uint64_t* K64(const K* p) { return reinterpret_cast<const uint64_t*>(p); }

 public:
  using this_t = map<K, V, Allocator, Hash>;

  map() : map(10) {}
  explicit map(unsigned n_log_2) : map(n_log_2, pool_slabs{0}) {}
  map(unsigned n_log_2, Allocator&& a) : map(n_log_2, pool_slabs{a.stack_size}) {}
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
  void put(cuda::std::pair<K, V>* operations, V* output, size_t size, cudaStream_t stream = 0x0) {
    static_assert(sizeof(cuda::std::pair<K, V>) == sizeof(KV), "pair layout");
    const KV* ops = reinterpret_cast<const KV*>(operations);
    if constexpr (kV32)
      lsb_check(lsb_map_put_pairs_v32(m_, ops, reinterpret_cast<uint32_t*>(output), size, stream),
                "lsb_map_put_pairs_v32");
    else
      lsb_check(lsb_map_put_pairs(m_, ops, reinterpret_cast<uint64_t*>(output), size, stream),
                "lsb_map_put_pairs");
  }

  // map.h:208-211
  template <int block_size = 256>
  void get(K* operations, cuda::std::pair<bool, V>* output, size_t size,
           cudaStream_t stream = 0x0) {
    static_assert(sizeof(cuda::std::pair<bool, V>) == sizeof(R), "pair layout");
    get<block_size>(operations, reinterpret_cast<R*>(output), size, stream);
  }

  // map.h:217-220 (update-if-present)
  template <int block_size = 256>
  void update(cuda::std::pair<K, V>* operations, cuda::std::pair<bool, V>* output, size_t size,
              cudaStream_t stream = 0x0) {
    const KV* ops = reinterpret_cast<const KV*>(operations);
    R* out = reinterpret_cast<R*>(output);
    if constexpr (kV32)
      lsb_check(lsb_map_update_v32(m_, ops, out, size, stream), "lsb_map_update_v32");
    else
      lsb_check(lsb_map_update(m_, ops, out, size, stream), "lsb_map_update");
  }
#endif

  // map.h:198-201
  template <int block_size = 256>
  void put(K* operations_keys, V* operations_values, V* output, size_t size,
           cudaStream_t stream = 0x0) {
    if constexpr (kV32)
      lsb_check(lsb_map_put_v32(m_, K64(operations_keys),
                                reinterpret_cast<const uint32_t*>(operations_values),
                                reinterpret_cast<uint32_t*>(output), size, stream),
                "lsb_map_put_v32");
    else
      lsb_check(lsb_map_put(m_, K64(operations_keys),
                            reinterpret_cast<const uint64_t*>(operations_values),
                            reinterpret_cast<uint64_t*>(output), size, stream),
                "lsb_map_put");
  }

  template <int block_size = 256>
  void get(K* operations, R* output, size_t size, cudaStream_t stream = 0x0) {
    if constexpr (kV32)
      lsb_check(lsb_map_get_v32(m_, K64(operations), output, size, stream), "lsb_map_get_v32");
    else
      lsb_check(lsb_map_get(m_, K64(operations), output, size, stream), "lsb_map_get");
  }

  // The REMOVE branch of detail::traverse (traverse.h:88-91), not exposed by
  // the reference map; 64-bit values only.
  template <int block_size = 256>
  void remove(K* operations, lsb_result* output, size_t size, cudaStream_t stream = 0x0) {
    static_assert(!kV32, "remove reports 64-bit values");
    lsb_check(lsb_map_remove(m_, K64(operations), output, size, stream), "lsb_map_remove");
  }

  // map.h:225-227
  unsigned buckets() const { return lsb_map_buckets(m_); }

  lsb_map* handle() const { return m_; }

 private:
  lsb_map* m_ = nullptr;
};

template <typename K, typename Allocator = device_allocator<detail::set_node<K>>,
          typename Hash = hash<K>>
class set {
  static_assert(std::is_integral<K>::value && std::is_unsigned<K>::value && sizeof(K) == 4,
                "lsb sets take 32-bit unsigned integer keys");
  static const uint32_t* K32(const K* p) { return reinterpret_cast<const uint32_t*>(p); }

 public:
  using this_t = set<K, Allocator, Hash>;

  set() : set(10) {}
  explicit set(unsigned n_log_2) : set(n_log_2, pool_slabs{0}) {}
  set(unsigned n_log_2, Allocator&& a) : set(n_log_2, pool_slabs{a.stack_size}) {}
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
  void contains(const K* keys, bool* output, size_t size, cudaStream_t stream = 0x0) {
    lsb_check(lsb_set_contains(s_, K32(keys), output, size, stream), "lsb_set_contains");
  }

  // set.h:103-106
  template <int block_size = 256>
  void insert(const K* keys, bool* output, size_t size, cudaStream_t stream = 0x0) {
    lsb_check(lsb_set_insert(s_, K32(keys), output, size, stream), "lsb_set_insert");
  }

  // set.h:114-117
  template <int block_size = 256>
  void remove(const K* keys, bool* output, size_t size, cudaStream_t stream = 0x0) {
    lsb_check(lsb_set_remove(s_, K32(keys), output, size, stream), "lsb_set_remove");
  }

#ifdef LSLAB_COMPAT_HAS_THRUST
  // set.h:97-101, 108-112, 119-123
  template <int block_size = 256>
  void contains(const thrust::device_vector<K>& keys, thrust::device_vector<bool>& output,
                cudaStream_t stream = 0x0) {
    contains<block_size>(keys.data().get(), output.data().get(), keys.size(), stream);
  }
  template <int block_size = 256>
  void insert(const thrust::device_vector<K>& keys, thrust::device_vector<bool>& output,
              cudaStream_t stream = 0x0) {
    insert<block_size>(keys.data().get(), output.data().get(), keys.size(), stream);
  }
  template <int block_size = 256>
  void remove(const thrust::device_vector<K>& keys, thrust::device_vector<bool>& output,
              cudaStream_t stream = 0x0) {
    remove<block_size>(keys.data().get(), output.data().get(), keys.size(), stream);
  }
#endif

  // set.h:125-127
  unsigned buckets() const { return lsb_set_buckets(s_); }

  lsb_set* handle() const { return s_; }

 private:
  lsb_set* s_ = nullptr;
};

}  // namespace lslab

#endif  // LSLAB_COMPAT_H
