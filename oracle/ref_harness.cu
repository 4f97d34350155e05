// Test infrastructure, not product code.
//
// C-ABI harness around the reference library's OWN containers and kernels
// (lslab::map<uint64_t,uint64_t>, lslab::set<uint32_t>), compiled for sm_100a
// from the reference headers where they lie (include path given by the
// Makefile beside this file).  Nothing here re-implements the reference: every
// get/put/insert/contains/remove below runs lslab's stock device code.  The
// built library lands in oracle/_ref/ and is used only by tests (golden vectors,
// GPU parity) and by bench.py's reference arm.
//
// What the harness adds around the stock code, and why:
//  * an explicit slab pool size, through the public constructor
//    map(n_log_2, Allocator&&) (include/lslab/map.h:57-66) with
//    device_allocator(stack_size) (include/lslab/device_allocator.h:16,
//    include/lslab/detail/device_allocator.h:9-14); the caller sizes it from an
//    upper bound on the slabs the workload can need, so the allocator's
//    overflow path (printf + __trap, include/lslab/detail/device_allocator.h:63-70)
//    is never reached;
//  * the pool is zeroed after construction: lslab placement-news overflow slabs
//    (include/lslab/detail/traverse.h:116-117) which leaves key[]/value[]
//    indeterminate, so a put of a new key into a fresh overflow slab would
//    return whatever cudaMalloc left there; zeroing makes "absent => 0" hold;
//  * map remove: lslab has no public map remove.  The REMOVE branch of the
//    generic traversal (include/lslab/detail/traverse.h:88-91) is reached by a
//    harness kernel that calls detail::traverse<Alloc, REMOVE> on the map's own
//    arrays, with a functor that reports the old value and zeroes the slot
//    (so a later insert into the freed slot again returns 0 for a new key);
//  * a host-side dump of the final (key,value) contents that walks the bucket
//    array and the pool exactly as the traversal does (valid bitmap, next link
//    in lane 31's slot).
//
// The containers keep their members private; the harness needs the lock
// table, bucket array and allocator for remove and for the dump, so the
// private section is opened for this translation unit only.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>

#define private public
#include <lslab/map.h>
#include <lslab/set.h>
#undef private

namespace {

using MapT = lslab::map<uint64_t, uint64_t>;
using MapSlab = lslab::detail::slab_node<uint64_t, uint64_t>;
using MapAlloc = lslab::device_allocator<MapSlab>;
using SetT = lslab::set<uint32_t>;
using SetSlab = lslab::detail::set_node<uint32_t>;
using SetAlloc = lslab::device_allocator<SetSlab>;

struct GetPair {      // layout of cuda::std::pair<bool, uint64_t>
  bool first;
  uint64_t second;
};
static_assert(sizeof(cuda::std::pair<bool, uint64_t>) == 16, "pair layout");
static_assert(sizeof(GetPair) == 16, "pair layout");

int check(cudaError_t e) { return e == cudaSuccess ? 0 : (int)e; }

// Remove functor: report the old value, then zero the slot.
struct RemoveFn {
  __device__ void operator()(uint64_t& v) {
    found = true;
    old = v;
    v = 0;
  }
  bool found;
  uint64_t old;
};

__global__ void map_remove_kernel(lslab::warp_mutex* lt, MapSlab* buckets, unsigned n_log_2,
                                  MapAlloc alloc, const uint64_t* keys, GetPair* out,
                                  size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool active = i < n;
  uint64_t key = active ? keys[i] : 0;
  RemoveFn fn{false, 0};
  unsigned bucket = (unsigned)(lslab::hash<uint64_t>{}(key) & ((1ull << n_log_2) - 1));
  lslab::detail::traverse<MapAlloc, lslab::detail::OPERATION_TYPE::REMOVE>{}(
      lt, buckets, key, fn, alloc, bucket, active);
  if (active) {
    out[i].first = fn.found;
    out[i].second = fn.found ? fn.old : 0;
  }
}

template <typename Slab, typename F>
size_t walk_pool(const std::vector<Slab>& heads, const Slab* pool_dev_base,
                 const std::vector<Slab>& pool, F&& emit) {
  size_t count = 0;
  for (size_t b = 0; b < heads.size(); ++b) {
    const Slab* s = &heads[b];
    while (s) {
      for (int lane = 0; lane < 31; ++lane) {
        if ((s->valid >> lane) & 1u) {
          emit(*s, lane);
          ++count;
        }
      }
      if (s->next == nullptr) break;
      size_t idx = (size_t)(s->next - pool_dev_base);
      if (idx >= pool.size()) {
        fprintf(stderr, "lslab_ref: next pointer outside the pool\n");
        return (size_t)-1;
      }
      s = &pool[idx];
    }
  }
  return count;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- map
void* lref_map_create(unsigned log2_buckets, uint64_t pool_slabs) {
  MapT* m = new MapT(log2_buckets, MapAlloc(pool_slabs));
  if (check(cudaMemset(m->alloc.mempool, 0, sizeof(MapSlab) * pool_slabs)) ||
      check(cudaDeviceSynchronize())) {
    delete m;
    return nullptr;
  }
  return m;
}

void lref_map_destroy(void* h) {
  MapT* m = static_cast<MapT*>(h);
  if (!m) return;
  cudaFree(m->lock_table);
  cudaFree(m->buckets_array);
  cudaFree(m->alloc.loc);
  cudaFree(m->alloc.mempool);
  delete m;
}

int lref_map_put(void* h, const uint64_t* keys, const uint64_t* vals, uint64_t* old_out,
                 size_t n, void* stream) {
  MapT* m = static_cast<MapT*>(h);
  if (n == 0) return 0;
  // the reference's put kernel stores every op's old value unconditionally
  // (include/lslab/detail/map_kernels.h:47-49): a null output is refused here
  if (!keys || !vals || !old_out) return -2;
  m->put<256>(const_cast<uint64_t*>(keys), const_cast<uint64_t*>(vals), old_out, n,
              (cudaStream_t)stream);
  return check(cudaGetLastError());
}

int lref_map_get(void* h, const uint64_t* keys, void* out, size_t n, void* stream) {
  MapT* m = static_cast<MapT*>(h);
  if (n == 0) return 0;
  if (!keys || !out) return -2;  // the kernel writes every result
  m->get<256>(const_cast<uint64_t*>(keys), static_cast<cuda::std::pair<bool, uint64_t>*>(out),
              n, (cudaStream_t)stream);
  return check(cudaGetLastError());
}

int lref_map_remove(void* h, const uint64_t* keys, void* out, size_t n, void* stream) {
  if (n && (!keys || !out)) return -2;  // the kernel writes every result
  MapT* m = static_cast<MapT*>(h);
  if (n == 0) return 0;
  unsigned blocks = (unsigned)((n + 255) / 256);
  map_remove_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(
      m->lock_table, m->buckets_array, m->number_of_buckets_log_2, m->alloc, keys,
      static_cast<GetPair*>(out), n);
  return check(cudaGetLastError());
}

uint64_t lref_map_pool_used(void* h) {
  MapT* m = static_cast<MapT*>(h);
  uint64_t used = 0;
  cudaMemcpy(&used, m->alloc.loc, sizeof(used), cudaMemcpyDeviceToHost);
  return used;
}

uint64_t lref_map_pool_capacity(void* h) { return static_cast<MapT*>(h)->alloc.stack_size; }

size_t lref_slab_bytes_map(void) { return sizeof(MapSlab); }
size_t lref_slab_bytes_set(void) { return sizeof(SetSlab); }

// Writes up to `cap` pairs (unsorted) and returns the number of live entries,
// or (size_t)-1 on a CUDA error / corrupt link.
size_t lref_map_dump(void* h, uint64_t* keys_out, uint64_t* vals_out, size_t cap) {
  MapT* m = static_cast<MapT*>(h);
  if (check(cudaDeviceSynchronize())) return (size_t)-1;
  size_t nb = (size_t)1 << m->number_of_buckets_log_2;
  std::vector<MapSlab> heads(nb);
  if (check(cudaMemcpy(heads.data(), m->buckets_array, nb * sizeof(MapSlab),
                       cudaMemcpyDeviceToHost)))
    return (size_t)-1;
  uint64_t used = lref_map_pool_used(h);
  used = std::min<uint64_t>(used, m->alloc.stack_size);
  std::vector<MapSlab> pool(used);
  if (used && check(cudaMemcpy(pool.data(), m->alloc.mempool, used * sizeof(MapSlab),
                               cudaMemcpyDeviceToHost)))
    return (size_t)-1;
  size_t w = 0;
  return walk_pool(heads, m->alloc.mempool, pool, [&](const MapSlab& s, int lane) {
    if (w < cap) {
      keys_out[w] = s.key[lane];
      vals_out[w] = s.value[lane];
    }
    ++w;
  });
}

// ---------------------------------------------------------------- set
void* lref_set_create(unsigned log2_buckets, uint64_t pool_slabs) {
  SetT* s = new SetT(log2_buckets, SetAlloc(pool_slabs));
  if (check(cudaMemset(s->alloc.mempool, 0, sizeof(SetSlab) * pool_slabs)) ||
      check(cudaDeviceSynchronize())) {
    delete s;
    return nullptr;
  }
  return s;
}

void lref_set_destroy(void* h) {
  SetT* s = static_cast<SetT*>(h);
  if (!s) return;
  cudaFree(s->lock_table);
  cudaFree(s->buckets_array);
  cudaFree(s->alloc.loc);
  cudaFree(s->alloc.mempool);
  delete s;
}

int lref_set_insert(void* h, const uint32_t* keys, bool* out, size_t n, void* stream) {
  if (n == 0) return 0;
  if (!keys || !out) return -2;  // the kernel writes every result
  static_cast<SetT*>(h)->insert<256>(keys, out, n, (cudaStream_t)stream);
  return check(cudaGetLastError());
}

int lref_set_contains(void* h, const uint32_t* keys, bool* out, size_t n, void* stream) {
  if (n == 0) return 0;
  if (!keys || !out) return -2;  // the kernel writes every result
  static_cast<SetT*>(h)->contains<256>(keys, out, n, (cudaStream_t)stream);
  return check(cudaGetLastError());
}

int lref_set_remove(void* h, const uint32_t* keys, bool* out, size_t n, void* stream) {
  if (n == 0) return 0;
  if (!keys || !out) return -2;  // the kernel writes every result
  static_cast<SetT*>(h)->remove<256>(keys, out, n, (cudaStream_t)stream);
  return check(cudaGetLastError());
}

uint64_t lref_set_pool_used(void* h) {
  SetT* s = static_cast<SetT*>(h);
  uint64_t used = 0;
  cudaMemcpy(&used, s->alloc.loc, sizeof(used), cudaMemcpyDeviceToHost);
  return used;
}

size_t lref_set_dump(void* h, uint32_t* keys_out, size_t cap) {
  SetT* s = static_cast<SetT*>(h);
  if (check(cudaDeviceSynchronize())) return (size_t)-1;
  size_t nb = (size_t)1 << s->number_of_buckets_log_2;
  std::vector<SetSlab> heads(nb);
  if (check(cudaMemcpy(heads.data(), s->buckets_array, nb * sizeof(SetSlab),
                       cudaMemcpyDeviceToHost)))
    return (size_t)-1;
  uint64_t used = std::min<uint64_t>(lref_set_pool_used(h), s->alloc.stack_size);
  std::vector<SetSlab> pool(used);
  if (used && check(cudaMemcpy(pool.data(), s->alloc.mempool, used * sizeof(SetSlab),
                               cudaMemcpyDeviceToHost)))
    return (size_t)-1;
  size_t w = 0;
  return walk_pool(heads, s->alloc.mempool, pool, [&](const SetSlab& sl, int lane) {
    if (w < cap) keys_out[w] = sl.key[lane];
    ++w;
  });
}

}  // extern "C"
