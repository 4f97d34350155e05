// Device building blocks of the slab-list table: layout, hashing, the
// thread-per-op probe, the single-writer apply, the slab pool and the bounded
// grid barrier.  sm_100a only.
//
// Layout (one slab, both containers)
//   bytes 0..31   meta sector: u32 next (slab index, 0 = none), 28 tag bytes
//   bytes 32..    28 slots: map = {u64 key, u64 value} (16 B), set = u32 key
//   map slab 480 B (15 sectors), set slab 160 B (5 sectors, 16 B spare)
// Slab indices [0, 2^n) are the bucket heads, [2^n, 2^n + pool) the overflow
// pool, so index 0 (a head) never appears as a link and means "none".
//
// Tag byte: 0x00 empty (never used), 0x80 busy (being claimed), 0x80|fp live,
// fp dead (removed; key kept so a later insert of the same key revives it).
// fp in 1..127 comes from the high half of the hash; the bucket from the low.
//
// Reference counterparts: slab_node/set_node (include/lslab/detail/slab_node.h:13-35:
// 31 keys + valid bitmap + next in lane 31's slot, values in a second array),
// traverse (include/lslab/detail/traverse.h:27-264), warp_mutex
// (include/lslab/warp_mutex.h:13-138), device_allocator
// (include/lslab/detail/device_allocator.h:63-73), hash (include/lslab/hash.h:10-15).
#pragma once

#include <cstdint>
#ifndef LSB_HOST_EMU
#include <cuda_runtime.h>
#endif

namespace lsb {

constexpr int kSlots = 28;
constexpr uint32_t kMetaBytes = 32;

enum : uint32_t {
  kStatusOOM = 0x1u,
  kStatusTimeout = 0x2u,
  kStatusChain = 0x4u,
  kStatusBarrier = 0x8u,
  kStatusScratch = 0x10u,
};

// get/contains, put/insert, remove, update (map only: overwrite the value of
// a present key, leave an absent one absent)
enum : uint8_t { kOpRead = 0, kOpWrite = 1, kOpRemove = 2, kOpUpdate = 3 };

enum : uint32_t { kLockWriter = 0, kLockFree = 1, kLockRW = 2 };

// Bounded waits: a lock or barrier wait gives up after this many polls and
// raises kStatusTimeout / kStatusBarrier instead of spinning forever.
constexpr uint32_t kLockPolls = 1u << 22;
constexpr uint32_t kBarrierPolls = 1u << 24;
constexpr uint32_t kMaxHops = 1u << 22;

// ------------------------------------------------------------------ hashing
// MurmurHash3's 64-bit finaliser (Appleby, public domain): a bijection on
// u64, so distinct keys never collide before the bucket mask.  Replaces the
// reference's identity hash (include/lslab/hash.h:12-14), which maps
// sequential keys to sequential buckets and structured keys to few buckets.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

__device__ __forceinline__ uint32_t fingerprint(uint64_t h) {
  return 1u + (uint32_t)(((h >> 32) * 127ull) >> 32);  // 1..127
}

// ------------------------------------------------------------- memory ops
#ifdef LSB_HOST_EMU
// CPU tests compile this header for the host with a thread-per-lane
// emulation of a block; it supplies these helpers (and sm_id) as plain
// atomic loads and stores.
#include "emu_mem_ops.h"
#else
// Table reads go to L2 (.cg / .relaxed.gpu): the persistent kernel reads
// slabs that other SMs wrote earlier in the same launch, and L1 is not
// coherent across SMs.
__device__ __forceinline__ uint4 ld_cg_v4(const void* p) {
  uint4 r;
  asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p));
  return r;
}

__device__ __forceinline__ ulonglong2 ld_cg_v2u64(const void* p) {
  ulonglong2 r;
  asm volatile("ld.global.cg.v2.u64 {%0,%1}, [%2];" : "=l"(r.x), "=l"(r.y) : "l"(p));
  return r;
}

__device__ __forceinline__ uint32_t ld_cg_u32(const void* p) {
  uint32_t r;
  asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(r) : "l"(p));
  return r;
}

__device__ __forceinline__ uint64_t ld_cg_u64(const void* p) {
  uint64_t r;
  asm volatile("ld.global.cg.u64 %0, [%1];" : "=l"(r) : "l"(p));
  return r;
}

// L1-cached loads for the read-only probe.  Safe because no table write runs
// concurrently with a probe (calls that mutate a table are stream-ordered;
// inside the persistent kernel probes and writes are separated by grid
// barriers whose acquire fence makes the SM's L1 observe earlier writes).
// Hot Zipf keys then hit each SM's L1 instead of queueing at one L2 slice.
// The loads also carry an L2 evict_last policy, and the streaming batch
// inputs/outputs an evict_first one, so the table's hot sectors outlive the
// batch data in L2 across calls.
__device__ __forceinline__ uint64_t l2_keep() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint4 ld_ca_v4(const void* p) {
  uint4 r;
  asm volatile("ld.global.ca.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p), "l"(l2_keep()));
  return r;
}

__device__ __forceinline__ ulonglong2 ld_ca_v2u64(const void* p) {
  ulonglong2 r;
  asm volatile("ld.global.ca.L2::cache_hint.v2.u64 {%0,%1}, [%2], %3;"
               : "=l"(r.x), "=l"(r.y)
               : "l"(p), "l"(l2_keep()));
  return r;
}

__device__ __forceinline__ uint32_t ld_ca_u32(const void* p) {
  uint32_t r;
  asm volatile("ld.global.ca.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(r) : "l"(p), "l"(l2_keep()));
  return r;
}

// Streaming (read-once / write-once) batch data: evict-first in L1 and L2.
__device__ __forceinline__ uint64_t ld_cs_u64(const void* p) {
  uint64_t r;
  asm volatile("ld.global.cs.u64 %0, [%1];" : "=l"(r) : "l"(p));
  return r;
}

__device__ __forceinline__ uint32_t ld_cs_u32(const void* p) {
  uint32_t r;
  asm volatile("ld.global.cs.u32 %0, [%1];" : "=r"(r) : "l"(p));
  return r;
}

__device__ __forceinline__ uint8_t ld_cs_u8(const void* p) {
  unsigned short r;
  asm volatile("ld.global.cs.u8 %0, [%1];" : "=h"(r) : "l"(p));
  return (uint8_t)r;
}

__device__ __forceinline__ void st_cs_u64(void* p, uint64_t v) {
  asm volatile("st.global.cs.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_cs_u32(void* p, uint32_t v) {
  asm volatile("st.global.cs.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void st_cs_u8(void* p, uint8_t v) {
  asm volatile("st.global.cs.u8 [%0], %1;" ::"l"(p), "h"((unsigned short)v) : "memory");
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t r;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(r) : "l"(p) : "memory");
  return r;
}

__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
  uint64_t r;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(r) : "l"(p) : "memory");
  return r;
}

__device__ __forceinline__ void st_cg_u8(void* p, uint8_t v) {
  asm volatile("st.global.cg.u8 [%0], %1;" ::"l"(p), "h"((unsigned short)v) : "memory");
}

__device__ __forceinline__ void st_cg_u32(void* p, uint32_t v) {
  asm volatile("st.global.cg.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void st_cg_u64(void* p, uint64_t v) {
  asm volatile("st.global.cg.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_cg_v2u64(void* p, uint64_t a, uint64_t b) {
  asm volatile("st.global.cg.v2.u64 [%0], {%1,%2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}

// Acquire-release: the block that arrives last at a grid barrier reads the
// other blocks' arrivals with this add and then proceeds without polling, so
// the add itself must acquire (a release-only add would let that block read
// stale copies of data the others wrote before arriving).
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ uint32_t sm_id() {
  uint32_t smid;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
  return smid;
}
#endif  // LSB_HOST_EMU

// Grid-wide warp index with consecutive warps in different blocks (warp w
// of block b is number w * gridDim.x + b), and the matching thread index
// (lanes stay consecutive, so a warp's 32 items stay contiguous).  A grid-
// stride loop over a small range then spreads over many SMs instead of
// filling the first few blocks.
__device__ __forceinline__ uint32_t spread_warp() {
  return (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
}
__device__ __forceinline__ uint32_t spread_tid() {
  return (threadIdx.x & 31u) + 32u * spread_warp();
}

__device__ __forceinline__ void raise_status(uint32_t* status, uint32_t bits) {
  atomicOr(status, bits);
}

// ---------------------------------------------------------------- meta
struct Meta {
  uint32_t next;
  uint32_t tag[7];  // 28 tag bytes, slot s in byte (s & 3) of word s >> 2
};

template <bool kL1 = false>
__device__ __forceinline__ Meta load_meta(const uint8_t* slab) {
  uint4 a = kL1 ? ld_ca_v4(slab) : ld_cg_v4(slab);
  uint4 b = kL1 ? ld_ca_v4(slab + 16) : ld_cg_v4(slab + 16);
  Meta m;
  m.next = a.x;
  m.tag[0] = a.y; m.tag[1] = a.z; m.tag[2] = a.w;
  m.tag[3] = b.x; m.tag[4] = b.y; m.tag[5] = b.z; m.tag[6] = b.w;
  return m;
}

// Bit s set iff tag byte s equals the byte replicated in rep4.
__device__ __forceinline__ uint32_t tag_match(const Meta& m, uint32_t rep4) {
  uint32_t mask = 0;
#pragma unroll
  for (int w = 0; w < 7; ++w) {
    uint32_t eq = __vcmpeq4(m.tag[w], rep4);  // 0xFF per equal byte
    // gather one bit per byte: byte j -> bit j
    uint32_t b = (eq >> 7) & 0x01010101u;     // bits 0, 8, 16, 24
    b = b | (b >> 7);                          // + bits 1 (byte 1), 17 (byte 3)
    b = (b | (b >> 14)) & 0xFu;                // bits 16, 17 -> 2, 3
    mask |= b << (4 * w);
  }
  return mask;
}

__device__ __forceinline__ uint8_t* slab_ptr(uint8_t* base, uint32_t idx, uint32_t bytes) {
  return base + (size_t)idx * bytes;
}
__device__ __forceinline__ const uint8_t* slab_ptr(const uint8_t* base, uint32_t idx,
                                                   uint32_t bytes) {
  return base + (size_t)idx * bytes;
}

// -------------------------------------------------------------- traits
struct MapTraits {
  using Key = uint64_t;
  static constexpr uint32_t kSlabBytes = 480;
  static constexpr uint32_t kSlotBytes = 16;
  static constexpr bool kHasValue = true;
  // Without the bucket lock (LSB_LOCK_FREE) a dead slot may be reused only by
  // its own key: a reader that matched the old key could otherwise read the
  // new key's value.  Locked inserts reuse any dead slot (scan_chain).
  static constexpr bool kReuseDead = false;
  __device__ static uint64_t hash(Key k) { return mix64(k); }
};

struct SetTraits {
  using Key = uint32_t;
  static constexpr uint32_t kSlabBytes = 160;
  static constexpr uint32_t kSlotBytes = 4;
  static constexpr bool kHasValue = false;
  // Without values a reader only ever compares the key itself, so any dead
  // slot can take a new key.
  static constexpr bool kReuseDead = true;
  __device__ static uint64_t hash(Key k) { return mix64((uint64_t)k); }
};

// Device view of one table; passed by value to kernels.
struct TableView {
  uint8_t* slabs;      // (buckets + pool) slabs
  int32_t* locks;      // one per bucket (reference encoding: 0 free, -1 writer, >0 readers)
  uint32_t* status;    // device status bits
  uint64_t* pool;      // [0] global cursor, [1] limit, [2 .. 2+kPoolSlots) per-SM ranges,
                       // [kPoolTop] free-stack top (signed; <= 0: empty)
  uint32_t* free_stack;  // slabs returned by compaction, taken before the bump pool
  uint32_t mask;       // buckets - 1
  uint32_t lock_mode;
  uint32_t chunk;      // slabs per per-SM refill (smaller for small pools)
};

// ------------------------------------------------------------ slab pool
// Slabs that compaction returned sit on a free stack (zeroed); pool_alloc
// pops from it before it bumps.  Compaction pushes only while it owns the
// table, so pops never race a push: a pop that finds the stack empty leaves
// the top below zero, and the next compaction clamps it back to zero first.
// Per-SM bump ranges refilled in chunks from one global cursor.  A range is
// one u64 {end:32 | cur:32}; atomicAdd on it hands out cur.  Exactly one
// thread sees cur == end when a range is spent: it takes a fresh chunk from
// the global cursor and installs it.  Threads that arrive while it does so
// (cur > end) take single slabs from the global cursor, so no chunk is ever
// abandoned half used.  The chunk shrinks with the pool (down to 1 slab,
// i.e. a plain global bump).  Pool memory is zeroed at creation and slabs
// are never returned, so a slab is always empty when handed out.  Replaces
// the reference's single global fetch_add with __trap on overflow
// (include/lslab/detail/device_allocator.h:63-70): here exhaustion returns 0
// and raises kStatusOOM, and only once every slab is handed out: when the
// global cursor is spent, the slabs still left in other SMs' ranges are taken
// (pool_alloc_leftover), so a caller that counts free slabs as the cursor's
// remainder plus the ranges' leftovers (pool_free_slabs) never sees an OOM
// within that count.
constexpr int kPoolSlots = 256;
constexpr int kPoolTop = 2 + kPoolSlots;
constexpr int kPoolWords = kPoolTop + 1;
constexpr uint32_t kPoolChunkMax = 32;

inline __device__ __noinline__ uint32_t pool_alloc_leftover(const TableView& t, uint32_t smid) {
  for (int k = 0; k < kPoolSlots; ++k) {
    unsigned long long* range =
        (unsigned long long*)&t.pool[2 + ((smid + (uint32_t)k) & (kPoolSlots - 1))];
    unsigned long long v = ld_relaxed_u64((const uint64_t*)range);
    for (;;) {
      const uint32_t cur = (uint32_t)v, end = (uint32_t)(v >> 32);
      if (cur >= end) break;
      const unsigned long long prev = atomicCAS(range, v, v + 1ull);
      if (prev == v) return cur;
      v = prev;
    }
  }
  raise_status(t.status, kStatusOOM);
  return 0;
}

__device__ __forceinline__ uint32_t pool_alloc(const TableView& t) {
  if ((long long)ld_relaxed_u64(&t.pool[kPoolTop]) > 0) {
    const long long top = (long long)atomicAdd((unsigned long long*)&t.pool[kPoolTop], ~0ull);
    if (top > 0) return t.free_stack[top - 1];
  }
  const uint32_t smid = sm_id();
  unsigned long long* range = (unsigned long long*)&t.pool[2 + (smid & (kPoolSlots - 1))];
  const unsigned long long old = atomicAdd(range, 1ull);
  const uint32_t cur = (uint32_t)old, end = (uint32_t)(old >> 32);
  if (cur < end) return cur;
  const unsigned long long limit = t.pool[1];
  const unsigned long long take = cur == end ? t.chunk : 1ull;  // refill, or a single slab
  const unsigned long long base = atomicAdd((unsigned long long*)&t.pool[0], take);
  if (base >= limit) return pool_alloc_leftover(t, smid);
  if (cur == end) {
    const unsigned long long stop = base + take < limit ? base + take : limit;
    atomicExch(range, (stop << 32) | (base + 1));  // base + 1 == stop: spent again
  }
  return (uint32_t)base;
}

// --------------------------------------------------------------- locks
__device__ __forceinline__ bool lock_writer(const TableView& t, uint32_t bucket) {
  int32_t* l = &t.locks[bucket];
  for (uint32_t it = 0; it < kLockPolls; ++it) {
    if (atomicCAS(l, 0, -1) == 0) {
      __threadfence();
      return true;
    }
    __nanosleep(it < 16 ? 32 : 256);
  }
  raise_status(t.status, kStatusTimeout);
  return false;
}

__device__ __forceinline__ void unlock_writer(const TableView& t, uint32_t bucket) {
  __threadfence();
  atomicExch(&t.locks[bucket], 0);
}

// Reference-style shared lock (include/lslab/warp_mutex.h:33-53), taken per
// op only in LSB_LOCK_RW mode, for the locking comparison.
__device__ __forceinline__ bool lock_reader(const TableView& t, uint32_t bucket) {
  int32_t* l = &t.locks[bucket];
  for (uint32_t it = 0; it < kLockPolls; ++it) {
    int32_t p = *(volatile int32_t*)l;
    if (p >= 0 && atomicCAS(l, p, p + 1) == p) {
      __threadfence();
      return true;
    }
  }
  raise_status(t.status, kStatusTimeout);
  return false;
}

__device__ __forceinline__ void unlock_reader(const TableView& t, uint32_t bucket) {
  __threadfence();
  atomicSub(&t.locks[bucket], 1);
}

// ---------------------------------------------------------------- probe
// Thread-per-op lookup: per slab one 32-B meta sector, then one slot load per
// fingerprint candidate.  A hit also reports where the key lives, packed as
// kLocLive | slab << 8 | slot, so the op's later write can go straight there.
constexpr uint64_t kLocLive = 1ull << 63;

__device__ __forceinline__ uint32_t loc_slab(uint64_t loc) { return (uint32_t)(loc >> 8); }
__device__ __forceinline__ int loc_slot(uint64_t loc) { return (int)(loc & 0xFFu); }

// Continue a lookup in slab `s`, trying its candidate slots `cand`, then
// the chain from `next` (s's link).  Takes the link rather than the whole
// meta sector so that callers need not keep the tag words live.
template <class Tr>
__device__ __noinline__ bool find_rest(const TableView& t, typename Tr::Key key, uint32_t rep,
                                       uint32_t s, uint32_t next, uint32_t cand, uint64_t* val,
                                       uint64_t* loc) {
  for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
    const uint8_t* slab = slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes);
    while (cand) {
      int slot = __ffs(cand) - 1;
      cand &= cand - 1;
      if constexpr (Tr::kHasValue) {
        ulonglong2 kv = ld_ca_v2u64(slab + kMetaBytes + slot * Tr::kSlotBytes);
        if (kv.x == (uint64_t)key) {
          *val = kv.y;
          *loc = kLocLive | ((uint64_t)s << 8) | (uint64_t)slot;
          return true;
        }
      } else {
        if (ld_ca_u32(slab + kMetaBytes + slot * Tr::kSlotBytes) == (uint32_t)key) {
          *loc = kLocLive | ((uint64_t)s << 8) | (uint64_t)slot;
          return true;
        }
      }
    }
    s = next;
    if (s == 0) return false;
    const Meta m = load_meta<true>(slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes));
    cand = tag_match(m, rep);
    next = m.next;
  }
  raise_status(t.status, kStatusChain);
  return false;
}

template <class Tr>
__device__ __forceinline__ bool table_find(const TableView& t, typename Tr::Key key, uint64_t h,
                                           uint64_t* val, uint64_t* loc) {
  const uint32_t s = (uint32_t)h & t.mask;
  const uint32_t rep = (0x80u | fingerprint(h)) * 0x01010101u;
  Meta m = load_meta<true>(slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes));
  return find_rest<Tr>(t, key, rep, s, m.next, tag_match(m, rep), val, loc);
}

// The lean single lookup of the read-only paths (k_read, and the fused
// kernel's read loop): the head meta sector, the first candidate slot inline,
// the rest of the chain in find_rest.  Few registers: it runs in kernels
// bounded to 32 a thread.
template <class Tr>
__device__ __forceinline__ bool read_lookup(const TableView& t, typename Tr::Key key,
                                            uint64_t* val) {
  const uint64_t h = Tr::hash(key);
  const uint32_t s = (uint32_t)h & t.mask;
  const uint32_t rep = (0x80u | fingerprint(h)) * 0x01010101u;
  const uint8_t* slab = slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes);
  const Meta m = load_meta<true>(slab);
  uint32_t cand = tag_match(m, rep);
  *val = 0;
  bool found = false;
  if (cand) {
    const int slot = __ffs(cand) - 1;
    cand &= cand - 1;
    if constexpr (Tr::kHasValue) {
      const ulonglong2 kv = ld_ca_v2u64(slab + kMetaBytes + slot * Tr::kSlotBytes);
      found = kv.x == (uint64_t)key;
      *val = found ? kv.y : 0ull;
    } else {
      found = ld_ca_u32(slab + kMetaBytes + slot * Tr::kSlotBytes) == (uint32_t)key;
    }
  }
  if (!found && (cand || m.next != 0)) {
    uint64_t loc;
    found = find_rest<Tr>(t, key, rep, s, m.next, cand, val, &loc);
    if (!found) *val = 0;
  }
  return found;
}

// P independent lookups issued together: all head meta sectors first, then
// all first-candidate slots, so a thread keeps up to P loads in flight.  The
// rare rest (second candidate, longer chain) falls back to find_rest.
template <class Tr, int P>
__device__ __forceinline__ void table_find_n(const TableView& t, const typename Tr::Key* key,
                                             const uint64_t* h, const bool* want, bool* found,
                                             uint64_t* val, uint64_t* loc) {
  Meta m[P];
  uint32_t rep[P], s[P], cand[P], next[P];
  const uint8_t* base = (const uint8_t*)t.slabs;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    s[j] = (uint32_t)h[j] & t.mask;
    rep[j] = (0x80u | fingerprint(h[j])) * 0x01010101u;
    if (want[j]) m[j] = load_meta<true>(slab_ptr(base, s[j], Tr::kSlabBytes));
  }
  uint64_t k0[P], v0[P];
  int slot0[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    cand[j] = want[j] ? tag_match(m[j], rep[j]) : 0u;
    next[j] = want[j] ? m[j].next : 0u;
    slot0[j] = cand[j] ? __ffs(cand[j]) - 1 : -1;
    if (slot0[j] >= 0) {
      const uint8_t* sp = slab_ptr(base, s[j], Tr::kSlabBytes) + kMetaBytes + slot0[j] * Tr::kSlotBytes;
      if constexpr (Tr::kHasValue) {
        ulonglong2 kv = ld_ca_v2u64(sp);
        k0[j] = kv.x;
        v0[j] = kv.y;
      } else {
        k0[j] = ld_ca_u32(sp);
        v0[j] = 0;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < P; ++j) {
    found[j] = false;
    val[j] = 0;
    loc[j] = 0;
    if (!want[j]) continue;
    if (slot0[j] >= 0 && k0[j] == (uint64_t)key[j]) {
      found[j] = true;
      val[j] = v0[j];
      loc[j] = kLocLive | ((uint64_t)s[j] << 8) | (uint64_t)slot0[j];
    } else if (cand[j] & (cand[j] - 1) || next[j] != 0) {
      found[j] = find_rest<Tr>(t, key[j], rep[j], s[j], next[j],
                               slot0[j] >= 0 ? cand[j] & (cand[j] - 1) : cand[j], &val[j],
                               &loc[j]);
    }
  }
}

// ---------------------------------------------------------------- apply
// Make the table hold `key` (present) with `val`, or not hold it (!present).
// Exactly one thread applies a given key at a time (the batch engine groups
// same-key ops and lets only the group's last op write), so a key's slot is
// only ever written by that thread.  Different keys of one bucket are kept
// apart by the bucket lock (kLockWriter / kLockRW) or by CAS on the tag and
// link words (kLockFree).  Order of writes for an insert: slot contents,
// fence, tag byte (or link word): a lock-free reader that sees the live tag
// sees the slot.
template <class Tr>
__device__ __forceinline__ void key_store(uint8_t* slot_ptr, typename Tr::Key key, uint64_t val) {
  if constexpr (Tr::kHasValue)
    st_cg_v2u64(slot_ptr, (uint64_t)key, val);
  else
    st_cg_u32(slot_ptr, (uint32_t)key);
}

template <class Tr>
__device__ __forceinline__ typename Tr::Key key_load(const uint8_t* slot_ptr) {
  if constexpr (Tr::kHasValue)
    return (typename Tr::Key)ld_cg_u64(slot_ptr);
  else
    return (typename Tr::Key)ld_cg_u32(slot_ptr);
}

struct ScanResult {
  uint32_t found_slab;  // slab holding the key (live or dead); valid if found_slot >= 0
  int found_slot;
  bool found_live;
  uint32_t free_slab;  // first reusable slot in chain order; valid if free_slot >= 0
  int free_slot;
  uint32_t tail;       // last slab of the chain
};

// kReuse: a dead slot of another key counts as free (the set always; the
// map only under the bucket lock: a lock-free map reader that matched the
// old key could otherwise read the new key's value, whereas the batch engine
// never runs a reader while a locked writer runs).
template <class Tr, bool kReuse>
__device__ __forceinline__ bool scan_chain(const TableView& t, typename Tr::Key key, uint64_t h,
                                           ScanResult& r, uint32_t start) {
  const uint32_t fp = fingerprint(h);
  const uint32_t live4 = (0x80u | fp) * 0x01010101u;
  const uint32_t dead4 = fp * 0x01010101u;
  uint32_t s = start;
  for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
    const uint8_t* slab = slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes);
    Meta m = load_meta(slab);
    uint32_t live = tag_match(m, live4);
    uint32_t cand = live | tag_match(m, dead4);
    while (cand) {
      int slot = __ffs(cand) - 1;
      cand &= cand - 1;
      if (key_load<Tr>(slab + kMetaBytes + slot * Tr::kSlotBytes) == key) {
        r.found_slab = s;
        r.found_slot = slot;
        r.found_live = (live >> slot) & 1u;
        r.tail = s;
        return true;
      }
    }
    if (r.free_slot < 0) {
      uint32_t fr = tag_match(m, 0u);  // empty
      if constexpr (kReuse) {
        // dead tags: nonzero with the top bit clear
#pragma unroll
        for (int w = 0; w < 7; ++w) {
          uint32_t x = m.tag[w];
          uint32_t nz = ((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x;  // top bit set iff byte != 0
          uint32_t dead = nz & ~x & 0x80808080u;                // nonzero and top bit clear
          uint32_t b = (dead >> 7) & 0x01010101u;
          b = (b | (b >> 7));
          b = (b | (b >> 14)) & 0xFu;
          fr |= b << (4 * w);
        }
      }
      fr &= (1u << kSlots) - 1u;
      if (fr) {
        r.free_slab = s;
        r.free_slot = __ffs(fr) - 1;
      }
    }
    r.tail = s;
    if (m.next == 0) return false;
    s = m.next;
  }
  raise_status(t.status, kStatusChain);
  return false;
}

__device__ __forceinline__ uint32_t* tag_word(uint8_t* slab, int slot) {
  return (uint32_t*)(slab + 4 + 4 * (slot >> 2));
}

template <class Tr>
__device__ void table_apply_locked(const TableView& t, typename Tr::Key key, uint64_t h,
                                   bool present, uint64_t val) {
  const uint32_t bucket = (uint32_t)h & t.mask;
  if (!lock_writer(t, bucket)) return;
  const uint32_t fp = fingerprint(h);
  ScanResult r;
  r.found_slot = -1;
  r.free_slot = -1;
  bool found = scan_chain<Tr, true>(t, key, h, r, bucket);
  if (found) {
    uint8_t* slab = slab_ptr(t.slabs, r.found_slab, Tr::kSlabBytes);
    uint8_t* tagp = slab + 4 + r.found_slot;
    if (present) {
      if constexpr (Tr::kHasValue)
        st_cg_u64(slab + kMetaBytes + r.found_slot * Tr::kSlotBytes + 8, val);
      if (!r.found_live) {
        __threadfence();
        st_cg_u8(tagp, (uint8_t)(0x80u | fp));
      }
    } else if (r.found_live) {
      st_cg_u8(tagp, (uint8_t)fp);
    }
  } else if (present) {
    if (r.free_slot >= 0) {
      uint8_t* slab = slab_ptr(t.slabs, r.free_slab, Tr::kSlabBytes);
      key_store<Tr>(slab + kMetaBytes + r.free_slot * Tr::kSlotBytes, key, val);
      __threadfence();
      st_cg_u8(slab + 4 + r.free_slot, (uint8_t)(0x80u | fp));
    } else {
      uint32_t n = pool_alloc(t);
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
}

template <class Tr>
__device__ void table_apply_lockfree(const TableView& t, typename Tr::Key key, uint64_t h,
                                     bool present, uint64_t val) {
  const uint32_t bucket = (uint32_t)h & t.mask;
  const uint32_t fp = fingerprint(h);
  // Slots are claimed with CAS on the tag words (no lock).  Growing a full
  // chain is serialized on the bucket's lock word: the holder re-reads the
  // tail's link and, if it is still empty, links one zeroed slab; every other
  // insert that found the chain full rescans from the tail once the lock is
  // released.  (Linking without it, each racer would link or drop a slab of
  // its own: hundreds of concurrent inserts into one bucket exhausted the
  // pool that way.)
  uint32_t start = bucket;
  for (uint32_t attempt = 0; attempt < kLockPolls; ++attempt) {
    ScanResult r;
    r.found_slot = -1;
    r.free_slot = -1;
    bool found = scan_chain<Tr, Tr::kReuseDead>(t, key, h, r, start);
    if (found) {
      uint8_t* slab = slab_ptr(t.slabs, r.found_slab, Tr::kSlabBytes);
      uint32_t* tw = tag_word(slab, r.found_slot);
      const uint32_t sh = 8 * (r.found_slot & 3);
      if (present) {
        if constexpr (Tr::kHasValue)
          st_cg_u64(slab + kMetaBytes + r.found_slot * Tr::kSlotBytes + 8, val);
        if (!r.found_live) {
          __threadfence();
          // Revive dead -> live by CAS on our own dead tag: where dead slots
          // are reusable (kReuseDead) another key may have claimed this slot
          // since the scan, and an unconditional OR would then mark its busy
          // claim live and lose this insert.  Other bytes of the word may
          // change meanwhile (retry); if ours no longer reads dead with our
          // fingerprint, the slot is gone and the insert starts over.
          uint32_t cur = ld_cg_u32(tw);
          bool revived = false;
          while (((cur >> sh) & 0xFFu) == fp) {
            const uint32_t prev = atomicCAS(tw, cur, cur | (0x80u << sh));
            if (prev == cur) {
              revived = true;
              break;
            }
            cur = prev;
          }
          if (!revived) {
            start = bucket;
            continue;
          }
        }
      } else if (r.found_live) {
        atomicAnd(tw, ~(0x80u << sh));
      }
      return;
    }
    if (!present) return;
    if (r.free_slot >= 0) {
      uint8_t* slab = slab_ptr(t.slabs, r.free_slab, Tr::kSlabBytes);
      uint32_t* tw = tag_word(slab, r.free_slot);
      const uint32_t sh = 8 * (r.free_slot & 3);
      uint32_t cur = ld_cg_u32(tw);
      uint32_t byte = (cur >> sh) & 0xFFu;
      bool reusable = (byte == 0) || (Tr::kReuseDead && byte != 0x80u && !(byte & 0x80u));
      if (reusable) {
        uint32_t claimed = (cur & ~(0xFFu << sh)) | (0x80u << sh);
        if (atomicCAS(tw, cur, claimed) == cur) {
          key_store<Tr>(slab + kMetaBytes + r.free_slot * Tr::kSlotBytes, key, val);
          __threadfence();
          atomicXor(tw, (0x80u ^ (0x80u | fp)) << sh);  // busy -> live
          return;
        }
      }
      start = bucket;  // lost the race: rescan from the head
      continue;
    }
    // the chain is full: grow it by one slab under the bucket's lock word
    if (!lock_writer(t, bucket)) return;  // timeout raised
    uint32_t* link = (uint32_t*)slab_ptr(t.slabs, r.tail, Tr::kSlabBytes);
    bool oom = false;
    if (ld_cg_u32(link) == 0) {
      const uint32_t n = pool_alloc(t);  // zeroed: every slot empty
      if (n != 0) {
        __threadfence();
        atomicExch(link, n);
      } else {
        oom = true;  // raised by pool_alloc
      }
    }
    unlock_writer(t, bucket);
    if (oom) return;
    start = r.tail;  // rescan from the old tail: its successor now exists
  }
  raise_status(t.status, kStatusTimeout);
}

template <class Tr>
__device__ __forceinline__ void table_apply(const TableView& t, typename Tr::Key key, uint64_t h,
                                            bool present, uint64_t val) {
  if (t.lock_mode == kLockFree)
    table_apply_lockfree<Tr>(t, key, h, present, val);
  else
    table_apply_locked<Tr>(t, key, h, present, val);
}

// Write the final state of a key whose live slot is known from this window's
// probe (loc has kLocLive).  Only this thread writes that key, and a live
// slot keeps its key until its own key's writer tombstones it, so neither a
// lock nor a rescan is needed: an update is one value store, a removal clears
// the live bit of the tag with an atomic (other bytes of the word may be
// changing under other writers).  Absent keys take table_apply.
template <class Tr>
__device__ __forceinline__ void table_apply_known(const TableView& t, typename Tr::Key key,
                                                  uint64_t h, uint64_t loc, bool present,
                                                  uint64_t val) {
  if (!(loc & kLocLive)) {
    if (present) table_apply<Tr>(t, key, h, true, val);
    return;
  }
  // the location was read back from window scratch: check it before use
  if (((loc & ~kLocLive) >> 8) >= ld_cg_u64(&t.pool[1]) || loc_slot(loc) >= kSlots) {
    raise_status(t.status, kStatusScratch);
    return;
  }
  uint8_t* slab = slab_ptr(t.slabs, loc_slab(loc), Tr::kSlabBytes);
  const int slot = loc_slot(loc);
  if (present) {
    if constexpr (Tr::kHasValue) st_cg_u64(slab + kMetaBytes + slot * Tr::kSlotBytes + 8, val);
  } else {
    // An atomic on the tag word: a locked insert of another key may be
    // writing a neighbouring tag byte of the same word at the same time.
    atomicAnd(tag_word(slab, slot), ~(0x80u << (8 * (slot & 3))));
  }
}

// ----------------------------------------------------------- compaction
__device__ __forceinline__ uint32_t live_mask(const Meta& m) {
  uint32_t mask = 0;
#pragma unroll
  for (int w = 0; w < 7; ++w) {
    // live: top bit set and not the busy marker 0x80
    const uint32_t x = m.tag[w];
    const uint32_t busy = __vcmpeq4(x, 0x80808080u);
    const uint32_t lv = x & ~busy & 0x80808080u;
    uint32_t b = (lv >> 7) & 0x01010101u;
    b = b | (b >> 7);
    b = (b | (b >> 14)) & 0xFu;
    mask |= b << (4 * w);
  }
  return mask;
}

// Tag words with every non-live byte cleared to empty.
__device__ __forceinline__ void clear_dead(Meta& m) {
#pragma unroll
  for (int w = 0; w < 7; ++w) {
    const uint32_t x = m.tag[w];
    const uint32_t busy = __vcmpeq4(x, 0x80808080u);
    const uint32_t lv = x & ~busy & 0x80808080u;  // top bit of each live byte
    m.tag[w] = x & ((lv >> 7) * 0xFFu);
  }
}

__device__ __forceinline__ void store_meta(uint8_t* slab, const Meta& m) {
  st_cg_u32(slab, m.next);
#pragma unroll
  for (int w = 0; w < 7; ++w) st_cg_u32(slab + 4 + 4 * w, m.tag[w]);
}

// Compaction of bucket b's chain; the caller owns the whole table (no other
// kernel uses it).  The chain's live entries move into its first
// need = ceil(live / kSlots) slabs (entries of later slabs fill the free
// slots of earlier ones in chain order), every removed slot of the kept
// slabs becomes empty, and the later slabs are zeroed, unlinked and pushed
// on the pool's free stack.  One thread per bucket; returns the slabs freed.
template <class Tr>
__device__ uint32_t compact_bucket(const TableView& t, uint32_t b) {
  uint8_t* base = t.slabs;
  uint32_t live = 0;
  for (uint32_t s = b, hop = 0; hop < kMaxHops; ++hop) {
    const Meta m = load_meta(slab_ptr(base, s, Tr::kSlabBytes));
    live += __popc(live_mask(m));
    if (m.next == 0) break;
    s = m.next;
  }
  const uint32_t need = live ? (live + kSlots - 1) / kSlots : 1u;
  // front: the kept slabs, whose free slots take the moved entries
  uint32_t fs = b;
  Meta fm = load_meta(slab_ptr(base, fs, Tr::kSlabBytes));
  clear_dead(fm);
  uint32_t ffree = ~live_mask(fm) & ((1u << kSlots) - 1u);
  // back: the slabs from chain position `need` on
  uint32_t last_kept = b, bs = fm.next;
  for (uint32_t k = 1; k < need && bs != 0; ++k) {
    last_kept = bs;
    bs = ld_cg_u32(slab_ptr(base, bs, Tr::kSlabBytes));
  }
  uint32_t freed = 0;
  while (bs != 0) {
    uint8_t* bp = slab_ptr(base, bs, Tr::kSlabBytes);
    const Meta bm = load_meta(bp);
    for (uint32_t lm = live_mask(bm); lm; lm &= lm - 1) {
      const int j = __ffs(lm) - 1;
      // next kept slab with a free slot; the kept slabs have room for every
      // live entry, so the front never passes last_kept
      while (ffree == 0 && fs != last_kept) {
        store_meta(slab_ptr(base, fs, Tr::kSlabBytes), fm);
        fs = fm.next;
        fm = load_meta(slab_ptr(base, fs, Tr::kSlabBytes));
        clear_dead(fm);
        ffree = ~live_mask(fm) & ((1u << kSlots) - 1u);
      }
      if (ffree == 0) {  // cannot happen (see above): keep the chain as it is
        raise_status(t.status, kStatusScratch);
        store_meta(slab_ptr(base, fs, Tr::kSlabBytes), fm);
        return freed;
      }
      const int i = __ffs(ffree) - 1;
      ffree &= ffree - 1;
      uint8_t* fp = slab_ptr(base, fs, Tr::kSlabBytes);
      if constexpr (Tr::kHasValue) {
        const ulonglong2 kv = ld_cg_v2u64(bp + kMetaBytes + j * Tr::kSlotBytes);
        st_cg_v2u64(fp + kMetaBytes + i * Tr::kSlotBytes, kv.x, kv.y);
      } else {
        st_cg_u32(fp + kMetaBytes + i * Tr::kSlotBytes,
                  ld_cg_u32(bp + kMetaBytes + j * Tr::kSlotBytes));
      }
      const uint32_t tag = (bm.tag[j >> 2] >> (8 * (j & 3))) & 0xFFu;
      fm.tag[i >> 2] = (fm.tag[i >> 2] & ~(0xFFu << (8 * (i & 3)))) | (tag << (8 * (i & 3)));
    }
    const uint32_t next = bm.next;
    for (uint32_t o = 0; o < Tr::kSlabBytes; o += 16) st_cg_v2u64(bp + o, 0ull, 0ull);
    // the stack holds at most the pool's slabs: each is either linked, on the
    // stack, or not yet handed out (checked anyway before the store)
    const unsigned long long at = atomicAdd((unsigned long long*)&t.pool[kPoolTop], 1ull);
    if (at < t.pool[1] - (uint64_t)t.mask - 1ull)
      t.free_stack[at] = bs;
    else
      raise_status(t.status, kStatusScratch);
    ++freed;
    bs = next;
  }
  if (fs == last_kept) fm.next = 0;
  store_meta(slab_ptr(base, fs, Tr::kSlabBytes), fm);
  // the kept slabs after the front cursor: removed slots become empty
  for (uint32_t s = fs; s != last_kept;) {
    s = ld_cg_u32(slab_ptr(base, s, Tr::kSlabBytes));
    uint8_t* sp = slab_ptr(base, s, Tr::kSlabBytes);
    Meta m = load_meta(sp);
    clear_dead(m);
    if (s == last_kept) m.next = 0;
    store_meta(sp, m);
  }
  return freed;
}

// -------------------------------------------------------- grid barrier
// Monotonic-count barrier for a cooperative (co-resident) grid: barrier k of
// a launch completes when the arrival counter reaches (k + 1) * nblocks, so
// nothing is reset between barriers.  One thread per block arrives with an
// acquire-release add and polls with acquire loads; the block's other threads are
// ordered by __syncthreads on both sides.  Each wait polls at most `limit`
// times (kBarrierPolls unless the caller knows a block may legitimately be
// late for longer); on timeout it raises kStatusBarrier and returns false so
// the caller can leave the kernel.
struct GridBarrier {
  uint32_t count;  // arrivals in this launch (zero when a launch starts)
  uint32_t exits;  // blocks that have left the launch (see release_counters)
};

__device__ __forceinline__ bool grid_barrier(GridBarrier* b, uint32_t nblocks, uint32_t* status,
                                             uint32_t& seq, uint32_t limit = kBarrierPolls) {
  __shared__ int ok;
  __syncthreads();
  ++seq;
  if (threadIdx.x == 0) {
    ok = 1;
    const uint32_t target = seq * nblocks;
    if (atom_add_acq_rel(&b->count, 1u) + 1 != target) {
      uint32_t it = 0;
      while ((int32_t)(ld_acquire_u32(&b->count) - target) < 0) {
        if (++it > limit || (*(volatile uint32_t*)status & kStatusBarrier)) {
          raise_status(status, kStatusBarrier);
          ok = 0;
          break;
        }
        if (it > 256) __nanosleep(64);
      }
    }
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace lsb
