// Per-warp device API: map and set operations called from inside a caller's
// own kernels, the counterpart of the reference's device methods
//   map::get / put / update (include/lslab/map.h:92-183)
//   set::contains / insert / remove (include/lslab/set.h:64-90)
// Like those, every function is warp-collective: all 32 lanes of the warp
// call it together, and `thread_mask` says which lanes have an op.  Lanes
// whose keys are equal are served in lane order (the reference serves a
// warp's ops one lane at a time, include/lslab/detail/traverse.h:45-48);
// lanes with different keys run at once.  Ops of different warps are
// linearizable per key: writers hold the bucket's writer lock, readers are
// lock-free (reader locks in LSB_LOCK_RW tables).
//
// Use: get a view of a table on the host with lsb_map_device_view /
// lsb_set_device_view (include/lsb.h), pass it to the kernel by value, wrap
// it in lsb_dev::map_ref / set_ref.  Build with -I <repo>/include and
// -I <repo>/lslab_b200/csrc (the slab layout) for sm_100a, and link
// liblsb.so for the host calls.
//
// Rules: a kernel that writes through this API is a mutating call on the
// table: it must not overlap other calls on the table (order it on one
// stream with them); kernels that only read may overlap read-only calls.
// Writers here never give one key's removed slot to another key (concurrent
// lock-free readers could otherwise match the old key), so the batch calls'
// compaction (lsb_map_compact) is what reclaims those slots.
#pragma once

#include <cstdint>

#include "lsb.h"
#include "lsb_core.cuh"

namespace lsb_dev {

__device__ __forceinline__ lsb::TableView to_view(const lsb_table_view& v) {
  lsb::TableView t;
  t.slabs = static_cast<uint8_t*>(v.slabs);
  t.locks = v.locks;
  t.status = v.status;
  t.pool = v.pool;
  t.free_stack = v.free_stack;
  t.mask = v.mask;
  t.lock_mode = v.lock_mode;
  t.chunk = v.chunk;
  return t;
}

// Run op() for every active lane, lanes of equal keys one after another in
// lane order; the warp is converged between rounds.
template <class K, class Op>
__device__ __forceinline__ void in_lane_order(K key, bool active, Op op) {
  const unsigned act = __ballot_sync(0xFFFFFFFFu, active);
  const unsigned lane = threadIdx.x & 31u;
  const unsigned peers = __match_any_sync(0xFFFFFFFFu, key) & act;
  const unsigned rank = __popc(peers & ((1u << lane) - 1u));
  const unsigned rounds = __reduce_max_sync(0xFFFFFFFFu, active ? rank + 1 : 0u);
  for (unsigned r = 0; r < rounds; ++r) {
    if (active && rank == r) op();
    __syncwarp();
  }
}

// Lock-free lookup through L2 (other SMs write concurrently): tags, then the
// candidate slot after a fence, so a slot whose live tag was seen is read
// with the contents its writer stored before the tag.
template <class Tr>
__device__ bool find(const lsb::TableView& t, typename Tr::Key key, uint64_t* val) {
  using namespace lsb;
  const uint64_t h = Tr::hash(key);
  const uint32_t rep = (0x80u | fingerprint(h)) * 0x01010101u;
  uint32_t s = (uint32_t)h & t.mask;
  for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
    const uint8_t* slab = slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes);
    const Meta m = load_meta<false>(slab);
    uint32_t cand = tag_match(m, rep);
    if (cand) __threadfence();
    while (cand) {
      const int slot = __ffs(cand) - 1;
      cand &= cand - 1;
      if constexpr (Tr::kHasValue) {
        const ulonglong2 kv = ld_cg_v2u64(slab + kMetaBytes + slot * Tr::kSlotBytes);
        if (kv.x == (uint64_t)key) {
          *val = kv.y;
          return true;
        }
      } else if (ld_cg_u32(slab + kMetaBytes + slot * Tr::kSlotBytes) == (uint32_t)key) {
        *val = 0;
        return true;
      }
    }
    if (m.next == 0) break;
    s = m.next;
  }
  *val = 0;
  return false;
}

enum : int { kPut = 0, kUpdate = 1, kRemove = 2 };

// One write under the bucket's writer lock; returns whether the key was
// present before and its value then (*old, 0 when absent).  put inserts an
// absent key (a removed slot of the same key first, else an empty slot, else
// a new slab at the tail); update changes only a present key; remove clears
// a present key's tag.
template <class Tr>
__device__ bool write(const lsb::TableView& t, typename Tr::Key key, int op, uint64_t val,
                      uint64_t* old) {
  using namespace lsb;
  const uint64_t h = Tr::hash(key);
  const uint32_t bucket = (uint32_t)h & t.mask;
  const uint32_t fp = fingerprint(h);
  *old = 0;
  if (!lock_writer(t, bucket)) return false;
  ScanResult r;
  r.found_slot = -1;
  r.free_slot = -1;
  const bool found = scan_chain<Tr, false>(t, key, h, r, bucket);
  bool existed = false;
  if (found) {
    uint8_t* slab = slab_ptr(t.slabs, r.found_slab, Tr::kSlabBytes);
    uint8_t* slot = slab + kMetaBytes + r.found_slot * Tr::kSlotBytes;
    existed = r.found_live;
    if constexpr (Tr::kHasValue) {
      if (existed) *old = ld_cg_u64(slot + 8);
    }
    if (op == kRemove) {
      if (existed) atomicAnd(tag_word(slab, r.found_slot), ~(0x80u << (8 * (r.found_slot & 3))));
    } else if (op == kPut || existed) {
      if constexpr (Tr::kHasValue) st_cg_u64(slot + 8, val);
      if (!existed) {  // revive the key's own removed slot
        __threadfence();
        atomicOr(tag_word(slab, r.found_slot), 0x80u << (8 * (r.found_slot & 3)));
      }
    }
  } else if (op == kPut) {
    if (r.free_slot >= 0) {
      uint8_t* slab = slab_ptr(t.slabs, r.free_slab, Tr::kSlabBytes);
      key_store<Tr>(slab + kMetaBytes + r.free_slot * Tr::kSlotBytes, key, val);
      __threadfence();
      atomicOr(tag_word(slab, r.free_slot), (0x80u | fp) << (8 * (r.free_slot & 3)));
    } else {
      const uint32_t n = pool_alloc(t);
      if (n != 0) {
        uint8_t* slab = slab_ptr(t.slabs, n, Tr::kSlabBytes);
        key_store<Tr>(slab + kMetaBytes, key, val);
        st_cg_u8(slab + 4, (uint8_t)(0x80u | fp));
        __threadfence();
        st_cg_u32(slab_ptr(t.slabs, r.tail, Tr::kSlabBytes), n);
      }
    }
  }
  unlock_writer(t, bucket);
  return existed;
}

// lslab::map<uint64_t, uint64_t>'s device methods over a table view.
struct map_ref {
  lsb::TableView t;
  __device__ explicit map_ref(const lsb_table_view& v) : t(to_view(v)) {}

  // map::get (map.h:105-119): true and the value when present.
  __device__ bool get(uint64_t key, uint64_t& value, bool thread_mask = true) const {
    bool found = false;
    uint64_t v = 0;
    in_lane_order(key, thread_mask, [&] {
      const uint32_t bucket = (uint32_t)lsb::MapTraits::hash(key) & t.mask;
      if (t.lock_mode == lsb::kLockRW) {
        if (!lsb::lock_reader(t, bucket)) return;
        found = find<lsb::MapTraits>(t, key, &v);
        lsb::unlock_reader(t, bucket);
      } else {
        found = find<lsb::MapTraits>(t, key, &v);
      }
    });
    if (thread_mask) value = v;
    return found;
  }

  // map::put (map.h:136-152): stores the value, returns the prior one (0 if
  // the key was absent).
  __device__ uint64_t put(uint64_t key, uint64_t value, bool thread_mask = true) const {
    uint64_t old = 0;
    in_lane_order(key, thread_mask,
                  [&] { write<lsb::MapTraits>(t, key, kPut, value, &old); });
    return old;
  }

  // map::update (map.h:167-183) with the semantics it intends: a present
  // key takes the value and {true, old value} is returned; an absent key
  // stays absent and {false, 0} is returned.
  __device__ lsb_result update(uint64_t key, uint64_t value, bool thread_mask = true) const {
    lsb_result r{};
    in_lane_order(key, thread_mask, [&] {
      uint64_t old = 0;
      r.found = write<lsb::MapTraits>(t, key, kUpdate, value, &old) ? 1 : 0;
      r.value = old;
    });
    return r;
  }

  // remove (the REMOVE branch of traverse.h:88-91): {true, old value} when
  // the key was present.
  __device__ lsb_result remove(uint64_t key, bool thread_mask = true) const {
    lsb_result r{};
    in_lane_order(key, thread_mask, [&] {
      uint64_t old = 0;
      r.found = write<lsb::MapTraits>(t, key, kRemove, 0, &old) ? 1 : 0;
      r.value = old;
    });
    return r;
  }
};

// lslab::set<uint32_t>'s device methods over a table view.
struct set_ref {
  lsb::TableView t;
  __device__ explicit set_ref(const lsb_table_view& v) : t(to_view(v)) {}

  // set::contains (set.h:64-72)
  __device__ bool contains(uint32_t key, bool thread_mask = true) const {
    bool found = false;
    in_lane_order(key, thread_mask, [&] {
      uint64_t v;
      const uint32_t bucket = (uint32_t)lsb::SetTraits::hash(key) & t.mask;
      if (t.lock_mode == lsb::kLockRW) {
        if (!lsb::lock_reader(t, bucket)) return;
        found = find<lsb::SetTraits>(t, key, &v);
        lsb::unlock_reader(t, bucket);
      } else {
        found = find<lsb::SetTraits>(t, key, &v);
      }
    });
    return found;
  }

  // set::insert (set.h:74-81): true for a new and for an existing key, as
  // the reference returns (traverse.h:204-212,226-232).
  __device__ bool insert(uint32_t key, bool thread_mask = true) const {
    in_lane_order(key, thread_mask, [&] {
      uint64_t old;
      write<lsb::SetTraits>(t, key, kPut, 0, &old);
    });
    return thread_mask;
  }

  // set::remove (set.h:83-90): whether the key was present.
  __device__ bool remove(uint32_t key, bool thread_mask = true) const {
    bool had = false;
    in_lane_order(key, thread_mask, [&] {
      uint64_t old;
      had = write<lsb::SetTraits>(t, key, kRemove, 0, &old);
    });
    return had;
  }
};

}  // namespace lsb_dev
