// The batch engine: runs a window of ops (reads and mutations, any mix, any
// key repetition) with results equal to running them one at a time in index
// order.
//
// Phases of one window (grid-stride passes; a grid-wide barrier or a kernel
// boundary between them):
//   A probe    every op reads the table (pre-window state, P lookups in flight
//              per thread) and writes that as its tentative result.  Each
//              mutation joins its key's group in a scratch hash table
//              (epoch-tagged slots, never cleared) and gets a position in it;
//              positions 0..7 are stored inline in the group, later ones in
//              32-entry chunks found through a second small hash table.  The
//              mutation also records where its key lives (the probe's slot).
//   D sort     only groups with more than 8 mutations: one block gathers the
//              group, orders it by op index, stores the sorted list and every
//              member's predecessor.  Skipped when no such group exists.
//   E resolve  a mutation takes its result from its predecessor in index
//              order (that op's post-state: put -> {1, value}, remove ->
//              {0, 0}); the group's last mutation writes the final state (a
//              value store or tag flip at the recorded slot, or a locked
//              insert for a key that was absent).  A read after the window's
//              first mutation finds its key's group and, if a mutation of that
//              key precedes it, takes that mutation's post-state.
// Only phase E writes the table and only one thread per key does, so no probe
// races a same-key write.
//
// The reference runs each op under a per-bucket warp lock in lane order within
// a warp and in lock-acquisition order across warps
// (include/lslab/detail/traverse.h:39-143); the engine fixes the order by op
// index instead and keeps locks off the read path.
#pragma once

#include "lsb_core.cuh"

namespace lsb {

constexpr uint32_t kInline = 8;        // group members stored inline
constexpr uint32_t kChunk = 32;        // members per overflow chunk
constexpr uint32_t kPredLast = 0x80000000u;
constexpr uint32_t kPredMask = 0x7FFFFFFFu;  // predecessor op index + 1; 0 = none
constexpr uint32_t kWarpSort = 64;    // groups up to this size are ordered by one warp
constexpr uint32_t kSortSmall = 4096;  // members a shared-memory sort holds
// groups of more than kHugeMin members are ordered by many blocks (the huge_*
// steps); smaller big groups by one block or one warp
constexpr uint32_t kHugeMin = 4096;
constexpr uint32_t kSortChunkWords = 2048;  // bitmap words per counting-sort pass
// shared memory of the sort: kSortSmall members + kSortSmall sorted + bitmap
// + prefix words
constexpr uint32_t kSortSmemBytes = (2 * kSortSmall + 2 * kSortChunkWords) * 4;

// Group-table slot: bits 0..23 owner (op index + 1), 24..47 count, 48..63 epoch.
__device__ __forceinline__ uint32_t g_owner(uint64_t v) { return (uint32_t)(v & 0xFFFFFFu); }
__device__ __forceinline__ uint32_t g_count(uint64_t v) { return (uint32_t)((v >> 24) & 0xFFFFFFu); }
__device__ __forceinline__ uint32_t g_epoch(uint64_t v) { return (uint32_t)(v >> 48); }

// All counters start at zero, so a set is reset with a plain memset.
struct WinCounters {
  uint32_t mut_count;
  uint32_t seg_cursor;
  uint32_t big_count;
  uint32_t clist_count;    // entries of the compacted mutation list
  uint32_t inv_first_mut;  // ~(lowest mutation index); 0 = no mutation
  uint32_t probe_cursor;   // next op to hand out when the probe claims chunks
  uint32_t large_count;    // groups with more than kWarpSort members
  uint32_t tiles_done;     // mutation-list tiles probed (reads fill in meanwhile)
  uint32_t late_cursor;    // next late read handed out in the fused sort pass
  uint32_t huge_count;     // groups with more than kHugeMin members
  uint32_t run_count;      // runs of huge groups (each sorted by one block)
  uint32_t upd_count;      // updates among the window's mutations
  uint32_t pad[4];
};

__device__ inline void win_counters_reset(WinCounters* c) {
  c->mut_count = 0;
  c->seg_cursor = 0;
  c->big_count = 0;
  c->clist_count = 0;
  c->inv_first_mut = 0;
  c->probe_cursor = 0;
  c->large_count = 0;
  c->late_cursor = 0;
  c->tiles_done = 0;
  c->huge_count = 0;
  c->run_count = 0;
  c->upd_count = 0;
}

// Scratch owned by a table, sized for max_window ops.
struct Scratch {
  uint64_t* gtab;   // group table, gmask + 1 slots
  uint32_t* ginl;   // kInline members per group slot
  uint64_t* ctab;   // overflow chunk table: epoch:16 | group slot:24 | chunk:24
  uint32_t* cdat;   // kChunk members per chunk slot
  uint32_t gmask;
  uint32_t cmask;
  uint32_t max_window;
  uint32_t pad;
  uint64_t* minfo;  // per mutation: group slot << 32 | position in group
  uint64_t* mloc;   // per mutation: the key's slot from the probe (0 = absent)
  uint32_t* pred;   // per member of a big group: predecessor + 1 | kPredLast
  uint32_t* goff;   // per big group slot: offset of its sorted list in seg
  uint32_t* seg;    // sorted member lists of big groups
  uint32_t* mlist;  // mutation op indices
  uint32_t* big;    // group slots with more than kInline members
  uint32_t* large;  // group slots with more than kWarpSort members
  WinCounters* cnt; // two sets, used by alternate windows
  uint8_t* obin;    // per op: table region (binned probing)
  uint32_t* perm;   // probe position -> op index (binned probing)
  // groups of more than kHugeMin members (hot keys), ordered over several
  // grid steps by many blocks: see the huge_* phases
  uint32_t* hlist;  // group slots, hcap entries
  uint32_t* hrec;   // per huge group: seg offset, stored members, first run, runs
  uint32_t* hbins;  // per huge group: kHugeBins range counts, then cursors
  uint32_t* hrun;   // per huge group and range: its run
  uint32_t* runs;   // per run: seg begin, seg end, info, 1 + largest member
  uint32_t hcap;
  uint32_t rcap;
  uint32_t* clist;  // compacted mutation indices, clist_cap(max_window) entries
  uint32_t* status; // the table's device status word
  // windows with updates: an update's effect depends on whether its key is
  // present just before it, i.e. on the last earlier member of its group
  // that is not an update
  uint32_t* lnu;    // per member of a group of > kInline: that member + 1, 0 = none
  uint32_t* rnu;    // per run of a huge group: 1 + its largest non-update member
};

// Result arrays: kOutResult {u8 found, pad, u64 value} (16 B), kOutOld u64,
// kOutBool u8, and for maps with 32-bit values kOutResult32 {u8 found, pad,
// u32 value} (8 B, the layout of cuda::std::pair<bool, uint32_t>) and
// kOutOld32 u32.
enum : uint32_t {
  kOutNone = 0, kOutResult = 1, kOutOld = 2, kOutBool = 3, kOutResult32 = 4, kOutOld32 = 5
};

__host__ __device__ constexpr uint32_t out_bytes(uint32_t kind) {
  return kind == kOutResult ? 16 : kind == kOutOld || kind == kOutResult32 ? 8
       : kind == kOutOld32 ? 4 : kind == kOutBool ? 1 : 0;
}

template <class Tr>
struct Window {
  const uint8_t* types;  // null: every op has type `uniform`
  const typename Tr::Key* keys;
  const uint64_t* vals;  // map puts and updates (u32 elements when v32)
  void* out;
  uint32_t kstride;      // elements between consecutive keys (2 for AoS pairs)
  uint32_t vstride;      // elements between consecutive values
  uint32_t n;
  uint32_t epoch;        // 1..65535
  uint8_t uniform;
  uint8_t out_kind;
  uint8_t v32;           // values are 32-bit (stored zero-extended)
  WinCounters* cnt;
};

template <class Tr>
__device__ __forceinline__ uint8_t op_type(const Window<Tr>& w, uint32_t i) {
  return w.types ? w.types[i] : w.uniform;
}

template <class Tr>
__device__ __forceinline__ typename Tr::Key key_of(const Window<Tr>& w, uint32_t i) {
  return w.keys[(size_t)i * w.kstride];
}

template <class Tr>
__device__ __forceinline__ uint64_t val_of(const Window<Tr>& w, uint32_t i) {
  if (w.v32) return reinterpret_cast<const uint32_t*>(w.vals)[(size_t)i * w.vstride];
  return w.vals[(size_t)i * w.vstride];
}

// First (streaming) read of op i's type and key in the probe phase.
template <class Tr>
__device__ __forceinline__ uint8_t op_type_stream(const Window<Tr>& w, uint32_t i) {
  return w.types ? ld_cs_u8(w.types + i) : w.uniform;
}

template <class Tr>
__device__ __forceinline__ typename Tr::Key key_stream(const Window<Tr>& w, uint32_t i) {
  if constexpr (sizeof(typename Tr::Key) == 8)
    return (typename Tr::Key)ld_cs_u64(w.keys + (size_t)i * w.kstride);
  else
    return (typename Tr::Key)ld_cs_u32(w.keys + (size_t)i * w.kstride);
}

// Result of op i given the key's state just before it.
template <class Tr>
__device__ __forceinline__ void write_result(const Window<Tr>& w, uint32_t i, uint8_t type,
                                             bool found, uint64_t value) {
  switch (w.out_kind) {
    case kOutResult: {
      // two 8-byte stores: lsb_result arrays are only 8-byte aligned in C
      uint64_t* p = (uint64_t*)w.out + 2 * (size_t)i;
      st_cs_u64(p, found ? 1ull : 0ull);
      st_cs_u64(p + 1, found ? value : 0ull);
      break;
    }
    case kOutOld:
      st_cs_u64((uint64_t*)w.out + i, found ? value : 0ull);
      break;
    case kOutResult32:  // one 8-byte store: found in byte 0, the value in bytes 4..7
      st_cs_u64((uint64_t*)w.out + i, found ? (1ull | (value << 32)) : 0ull);
      break;
    case kOutOld32:
      st_cs_u32((uint32_t*)w.out + i, found ? (uint32_t)value : 0u);
      break;
    case kOutBool:
      st_cs_u8((uint8_t*)w.out + i, (type == kOpWrite) ? 1 : (found ? 1 : 0));
      break;
    default:
      break;
  }
}

__device__ __forceinline__ uint32_t lane_id() {
#ifdef LSB_HOST_EMU
  return threadIdx.x & 31u;
#else
  uint32_t l;
  asm("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
#endif
}

__device__ __forceinline__ uint32_t gslot_of(uint64_t h, uint32_t gmask) {
  return (uint32_t)(h >> 20) & gmask;
}

// --------------------------------------------------------- overflow chunks
__device__ __forceinline__ uint32_t chunk_hash(uint32_t gslot, uint32_t k) {
  uint32_t x = gslot * 0x9E3779B1u ^ (k + 0x7F4A7C15u) * 0x85EBCA77u;
  x ^= x >> 15;
  x *= 0x2C1B3C6Du;
  return x ^ (x >> 12);
}

// Slot of chunk k of group gslot in this window; claims it if new.
__device__ __forceinline__ uint32_t chunk_claim(const Scratch& sc, uint32_t epoch, uint32_t gslot,
                                                uint32_t k) {
  const uint64_t key = ((uint64_t)epoch << 48) | ((uint64_t)gslot << 24) | k;
  uint32_t s = chunk_hash(gslot, k) & sc.cmask;
  for (uint32_t probe = 0; probe <= sc.cmask; ++probe) {
    uint64_t v = ld_relaxed_u64(&sc.ctab[s]);
    while ((uint32_t)(v >> 48) != epoch) {  // stale: try to claim
      uint64_t prev = atomicCAS((unsigned long long*)&sc.ctab[s], v, key);
      if (prev == v) return s;
      v = prev;
    }
    if (v == key) return s;
    s = (s + 1) & sc.cmask;
  }
  return 0xFFFFFFFFu;
}

__device__ __forceinline__ uint32_t chunk_find(const Scratch& sc, uint32_t epoch, uint32_t gslot,
                                               uint32_t k) {
  const uint64_t key = ((uint64_t)epoch << 48) | ((uint64_t)gslot << 24) | k;
  uint32_t s = chunk_hash(gslot, k) & sc.cmask;
  for (uint32_t probe = 0; probe <= sc.cmask; ++probe) {
    uint64_t v = ld_relaxed_u64(&sc.ctab[s]);
    if (v == key) return s;
    if ((uint32_t)(v >> 48) != epoch) return 0xFFFFFFFFu;
    s = (s + 1) & sc.cmask;
  }
  return 0xFFFFFFFFu;
}

// Member j (0-based position) of group gslot.
__device__ __forceinline__ uint32_t member_at(const Scratch& sc, uint32_t epoch, uint32_t gslot,
                                              uint32_t j) {
  if (j < kInline) return ld_cg_u32(&sc.ginl[(size_t)gslot * kInline + j]);
  const uint32_t q = j - kInline;
  const uint32_t cs = chunk_find(sc, epoch, gslot, q / kChunk);
  return cs == 0xFFFFFFFFu ? 0xFFFFFFFFu : ld_cg_u32(&sc.cdat[(size_t)cs * kChunk + q % kChunk]);
}

// ---------------------------------------------------------------- phase A
// Store member i at position pos of group `slot` (inline or in a chunk).
template <class Tr>
__device__ __forceinline__ void group_store(const Scratch& sc, const Window<Tr>& w, uint32_t slot,
                                            uint32_t pos, uint32_t i, uint64_t loc) {
  sc.minfo[i] = ((uint64_t)slot << 32) | pos;
  sc.mloc[i] = loc;
  if (pos >= sc.max_window) return;  // no group (cannot happen: the table has 2x room)
  if (pos < kInline) {
    sc.ginl[(size_t)slot * kInline + pos] = i;
  } else {
    const uint32_t q = pos - kInline;
    const uint32_t cs = chunk_claim(sc, w.epoch, slot, q / kChunk);
    if (cs != 0xFFFFFFFFu) sc.cdat[(size_t)cs * kChunk + q % kChunk] = i;
    if (pos == kInline) sc.big[atomicAdd(&w.cnt->big_count, 1u)] = slot;
    if (pos == kWarpSort) sc.large[atomicAdd(&w.cnt->large_count, 1u)] = slot;
    if (pos == kHugeMin) {
      const uint32_t h = atomicAdd(&w.cnt->huge_count, 1u);
      if (h < sc.hcap) sc.hlist[h] = slot;
    }
  }
}

// Join `cnt` mutations of `key` (op indices carried by the caller's peer
// lanes) to the key's group; returns the group slot and the position of the
// first of them.  The group's owner (first joiner) claims the slot by CAS.
template <class Tr>
__device__ __forceinline__ uint32_t group_join(const Scratch& sc, const Window<Tr>& w, uint32_t i,
                                               typename Tr::Key key, uint64_t h, uint32_t cnt,
                                               uint32_t* pos_out) {
  uint32_t slot = gslot_of(h, sc.gmask);
  const uint64_t mine =
      ((uint64_t)w.epoch << 48) | ((uint64_t)cnt << 24) | (uint64_t)(i + 1);
  for (uint32_t probe = 0; probe <= sc.gmask; ++probe) {
    uint64_t v = ld_relaxed_u64(&sc.gtab[slot]);
    while (g_epoch(v) != w.epoch) {  // stale slot: try to claim it
      uint64_t prev = atomicCAS((unsigned long long*)&sc.gtab[slot], v, mine);
      if (prev == v) {
        *pos_out = 0;
        return slot;
      }
      v = prev;
    }
    if (key_of(w, g_owner(v) - 1) == key) {
      *pos_out = g_count(atomicAdd((unsigned long long*)&sc.gtab[slot], (uint64_t)cnt << 24));
      return slot;
    }
    slot = (slot + 1) & sc.gmask;
  }
  *pos_out = 0xFFFFFFFFu;
  return 0;
}

// One tile of phase A: ops base + j*32 + lane for j < P.  kGroup: mutations
// join groups (false for read-only batches).  dedup: lanes of a warp that
// carry the same key share one lookup (warp-uniform flag).
// Which ops a probe pass handles: reads with read_lo <= i < read_hi, and the
// mutations when `muts` is set (the fused kernel splits a window's reads
// between the grouping pass and the sort pass to hide the latter).
struct ProbeSel {
  uint32_t read_lo, read_hi;
  bool muts;
};

// Probe (and, for mutations, group) the ops idx[j] whose type and key the
// caller loaded; lanes in ascending op-index order.  Every lane of the warp
// calls it.
template <class Tr, bool kGroup, int P>
__device__ __forceinline__ void probe_ops(const TableView& t, const Scratch& sc,
                                          const Window<Tr>& w, uint32_t lane, bool dedup,
                                          const uint32_t (&idx)[P], const uint8_t (&type)[P],
                                          const bool (&active)[P],
                                          const typename Tr::Key (&key)[P]) {
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  uint64_t h[P], value[P], loc[P];
  bool want[P], found[P];
  uint32_t src[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    h[j] = Tr::hash(key[j]);
    want[j] = active[j];
    src[j] = lane;
    if (dedup) {
      const uint32_t am = __ballot_sync(0xFFFFFFFFu, active[j]);
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key[j]) & am;
      if (active[j]) src[j] = __ffs(peers) - 1;
      want[j] = active[j] && src[j] == lane;
    }
  }
  if (t.lock_mode == kLockRW) {
#pragma unroll
    for (int j = 0; j < P; ++j) {
      found[j] = false;
      value[j] = 0;
      loc[j] = 0;
      if (!want[j]) continue;
      const uint32_t bucket = (uint32_t)h[j] & t.mask;
      if (lock_reader(t, bucket)) {
        found[j] = table_find<Tr>(t, key[j], h[j], &value[j], &loc[j]);
        unlock_reader(t, bucket);
      }
    }
  } else {
    table_find_n<Tr, P>(t, key, h, want, found, value, loc);
  }
#pragma unroll
  for (int j = 0; j < P; ++j) {
    if (dedup) {
      found[j] = __shfl_sync(0xFFFFFFFFu, found[j], src[j]);
      value[j] = __shfl_sync(0xFFFFFFFFu, value[j], src[j]);
      loc[j] = __shfl_sync(0xFFFFFFFFu, loc[j], src[j]);
    }
    const uint32_t i = idx[j];
    if (active[j]) write_result(w, i, type[j], found[j], value[j]);
    if (kGroup) {
      const bool is_mut = active[j] && type[j] != kOpRead;
      const uint32_t mm = __ballot_sync(0xFFFFFFFFu, is_mut);
      if (mm) {
        const uint32_t first = __reduce_min_sync(0xFFFFFFFFu, is_mut ? i : 0xFFFFFFFFu);
        uint32_t slot_base = 0;
        const uint32_t ldr = __ffs(mm) - 1;
        const uint32_t um = __ballot_sync(0xFFFFFFFFu, is_mut && type[j] == kOpUpdate);
        if (lane == ldr) {
          slot_base = atomicAdd(&w.cnt->mut_count, (uint32_t)__popc(mm));
          atomicMax(&w.cnt->inv_first_mut, ~first);
          if (um) atomicAdd(&w.cnt->upd_count, (uint32_t)__popc(um));
        }
        slot_base = __shfl_sync(0xFFFFFFFFu, slot_base, ldr);
        // same-key mutations of this warp join together: the lowest lane
        // (lowest op index) joins for all and hands out consecutive
        // positions in lane order, which is op-index order
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key[j]) & mm;
        const uint32_t lead = is_mut ? __ffs(peers) - 1 : lane;
        uint32_t gslot = 0, gpos = 0;
        if (is_mut && lead == lane)
          gslot = group_join<Tr>(sc, w, i, key[j], h[j], __popc(peers), &gpos);
        gslot = __shfl_sync(0xFFFFFFFFu, gslot, lead);
        gpos = __shfl_sync(0xFFFFFFFFu, gpos, lead);
        if (is_mut) {
          sc.mlist[slot_base + __popc(mm & lanemask_lt)] = i;
          group_store<Tr>(sc, w, gslot, gpos + __popc(peers & lanemask_lt), i, loc[j]);
        }
      }
    }
  }
}

// Ops base + j*32 + lane, j < P.  `perm` (optional): position -> op index
// (the binned order); positions are then mapped to ops, and sel's read range
// is in positions.
template <class Tr, bool kGroup, int P>
__device__ __forceinline__ void probe_tile(const TableView& t, const Scratch& sc,
                                           const Window<Tr>& w, uint32_t base, uint32_t lane,
                                           bool dedup, const ProbeSel& sel,
                                           const uint32_t* perm) {
  using Key = typename Tr::Key;
  Key key[P];
  uint8_t type[P];
  bool active[P];
  uint32_t idx[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const uint32_t pos = base + j * 32 + lane;
    uint32_t i = pos;
    if (perm != nullptr && pos < w.n) i = min(ld_cs_u32(perm + pos), w.n);
    idx[j] = i;
    type[j] = i < w.n ? (perm ? op_type(w, i) : op_type_stream(w, i)) : kOpRead;
    active[j] = i < w.n && (type[j] == kOpRead ? (pos >= sel.read_lo && pos < sel.read_hi) : sel.muts);
    key[j] = active[j] ? (perm ? key_of(w, i) : key_stream(w, i)) : (Key)0;
  }
  probe_ops<Tr, kGroup, P>(t, sc, w, lane, dedup, idx, type, active, key);
}

// Phase A for the mutations of a window (its reads are probed by blocks
// with no list tile left and in the ordering pass), in two grid steps with a
// grid barrier between them.
// Step 1 (phase_list_muts): a warp takes 512-op spans; each lane reads the
// types of 16 consecutive ops with one 16-byte load, and the span's mutations
// are appended in op-index order to a list, padded to whole 32-entry tiles
// (one atomic per span).  Step 2 (phase_probe_list): the tiles are probed and
// grouped by all warps.  A read-mostly window then costs two short passes
// instead of one dependent chain per 32 ops, and dense runs of mutations are
// spread over every warp of the grid.
constexpr uint32_t kListSpan = 512;

__host__ __device__ constexpr uint32_t clist_cap(uint32_t window) {
  return window + 32u * (window / kListSpan + 1u);  // each span pads < 32 entries
}

template <class Tr>
__device__ void phase_list_muts(const Scratch& sc, const Window<Tr>& w, uint32_t warp_id,
                                uint32_t num_warps) {
  constexpr uint32_t kPer = kListSpan / 32;
  static_assert(kPer == 16, "one 16-byte type load and a 16-bit mask per lane");
  if (w.types == nullptr && w.uniform == kOpRead) return;
  const uint32_t lane = lane_id();
  const uint32_t cap = clist_cap(sc.max_window);
  for (uint32_t base = warp_id * kListSpan; base < w.n; base += num_warps * kListSpan) {
    const uint32_t o = base + lane * kPer;
    uint32_t bits = 0;  // bit k: op o + k is a mutation
    if (w.types == nullptr) {
      if (o < w.n) bits = w.n - o >= kPer ? 0xFFFFu : (1u << (w.n - o)) - 1u;
    } else if (((uintptr_t)(w.types + base) & 15u) == 0 && base + kListSpan <= w.n) {
      // warp-uniform: the span is whole and its lanes' 16 bytes are aligned
      const uint4 v = ld_cg_v4(w.types + o);
      const uint32_t word[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int q = 0; q < 16; ++q)
        if (((word[q >> 2] >> (8 * (q & 3))) & 0xFFu) != kOpRead) bits |= 1u << q;
    } else {
      for (uint32_t q = 0; q < kPer && o + q < w.n; ++q)
        if (op_type(w, o + q) != kOpRead) bits |= 1u << q;
    }
    const uint32_t c = __popc(bits);
    uint32_t incl = c;  // inclusive prefix of the lanes' counts
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if (lane >= d) incl += y;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (total == 0) continue;  // warp-uniform
    const uint32_t padded = (total + 31u) & ~31u;
    uint32_t at = 0;
    if (lane == 0) at = atomicAdd(&w.cnt->clist_count, padded);
    at = __shfl_sync(0xFFFFFFFFu, at, 0);
    if (at > cap || padded > cap - at) {  // cannot happen: the list is sized for every span
      if (lane == 0) raise_status(sc.status, kStatusScratch);
      continue;
    }
    uint32_t* dst = sc.clist + at + (incl - c);
    for (uint32_t m = bits; m; m &= m - 1u) *dst++ = o + (uint32_t)(__ffs(m) - 1);
    if (lane < padded - total) sc.clist[at + total + lane] = 0xFFFFFFFFu;
  }
}

template <class Tr>
__device__ void phase_probe_list(const TableView& t, const Scratch& sc, const Window<Tr>& w,
                                 uint32_t warp_id, uint32_t num_warps, bool dedup) {
  using Key = typename Tr::Key;
  const uint32_t lane = lane_id();
  const uint32_t total = min(ld_cg_u32(&w.cnt->clist_count), clist_cap(sc.max_window));
  for (uint32_t tile = warp_id * 32; tile < total; tile += num_warps * 32) {
    const uint32_t i = tile + lane < total ? ld_cg_u32(sc.clist + tile + lane) : 0xFFFFFFFFu;
    uint32_t idx[1] = {0xFFFFFFFFu};
    uint8_t type[1] = {kOpRead};
    bool active[1] = {false};
    Key key[1] = {(Key)0};
    if (i < w.n) {
      idx[0] = i;
      type[0] = op_type(w, i);
      active[0] = type[0] != kOpRead;
      key[0] = key_of(w, i);
    }
    probe_ops<Tr, true, 1>(t, sc, w, lane, dedup, idx, type, active, key);
    if (lane == 0) atomicAdd(&w.cnt->tiles_done, 1u);
  }
}

// Phase A over the window from op `begin`.  cursor == null or chunk == 0:
// warp-uniform grid stride of 32*P ops.  Otherwise work is claimed in two
// levels: a block takes `chunk` consecutive ops with one atomic on *cursor,
// its warps take 32*P-op tiles of that chunk from a shared counter; blocks
// that finish early take more chunks (balance without a global atomic per
// tile).  With `stop_at`, a block takes no further chunk once *stop_at has
// reached stop_target (the rest is claimed by a later call on the same
// cursor).  Every thread of the block must call it.
template <class Tr, bool kGroup, int P>
__device__ void phase_probe(const TableView& t, const Scratch& sc, const Window<Tr>& w,
                            uint32_t warp_id, uint32_t num_warps, uint32_t* cursor,
                            uint32_t chunk, bool dedup,
                            ProbeSel sel = ProbeSel{0, 0xFFFFFFFFu, true}, uint32_t begin = 0,
                            const uint32_t* perm = nullptr, const uint32_t* stop_at = nullptr,
                            uint32_t stop_target = 0) {
  const uint32_t lane = lane_id();
  if (cursor == nullptr || chunk == 0) {
    for (uint32_t base = begin + warp_id * 32 * P; base < w.n; base += num_warps * 32 * P)
      probe_tile<Tr, kGroup, P>(t, sc, w, base, lane, dedup, sel, perm);
    return;
  }
  __shared__ uint32_t s_base, s_next;
  // whole tiles per claim: a tile crossing into the next claim would be
  // processed twice (and a mutation would join its group twice)
  chunk = max(32u * P, chunk - chunk % (32u * P));
  for (;;) {
    if (threadIdx.x == 0) {
      // checked before claiming, so no claimed chunk is ever dropped
      s_base = (stop_at != nullptr && ld_cg_u32(stop_at) >= stop_target)
                   ? 0xFFFFFFFFu
                   : begin + atomicAdd(cursor, chunk);
      s_next = 0;
    }
    __syncthreads();
    const uint32_t c0 = s_base;
    if (c0 >= w.n) break;  // block-uniform
    const uint32_t c1 = min(w.n, c0 + chunk);
    for (;;) {
      uint32_t off = 0;
      if (lane == 0) off = atomicAdd(&s_next, 32u * P);
      off = __shfl_sync(0xFFFFFFFFu, off, 0);
      if (c0 + off >= c1) break;
      probe_tile<Tr, kGroup, P>(t, sc, w, c0 + off, lane, dedup, sel, perm);
    }
    __syncthreads();  // s_base / s_next are rewritten next round
  }
}

// The reads of [lo, hi) (ops of other types are skipped) with the lean
// lookup, one op per thread: a block claims blockDim.x * 4 ops at a time
// from *cursor (relative to lo), so blocks that finish early take more.
// With stop_at, a block takes no further claim once *stop_at has reached
// stop_target (the rest is claimed by a later call on the same cursor).
// Every thread of the block calls it.
// kPair: each thread keeps two lookups in flight (both meta sectors, then
// both candidate slots; table_find_n), which recovers the memory
// parallelism that a 64-register kernel's half occupancy loses.
template <class Tr, bool kPair = false>
__device__ void phase_read_lean(const TableView& t, const Window<Tr>& w, uint32_t* cursor,
                                uint32_t lo, uint32_t hi, const uint32_t* stop_at = nullptr,
                                uint32_t stop_target = 0) {
  __shared__ uint32_t s_base;
  const uint32_t chunk = blockDim.x * 4;
  for (;;) {
    if (threadIdx.x == 0)
      s_base = (stop_at != nullptr && ld_cg_u32(stop_at) >= stop_target)
                   ? 0xFFFFFFFFu
                   : lo + atomicAdd(cursor, chunk);
    __syncthreads();
    const uint32_t c0 = s_base;
    __syncthreads();  // s_base is rewritten next round
    if (c0 >= hi || c0 < lo) break;  // block-uniform
    const uint32_t c1 = min(hi, c0 + chunk);
    if constexpr (kPair) {
      for (uint32_t i = c0 + threadIdx.x; i < c1; i += 2 * blockDim.x) {
        const uint32_t i2 = i + blockDim.x;
        typename Tr::Key key[2];
        uint64_t h[2], val[2], loc[2];
        bool want[2], found[2];
        want[0] = op_type(w, i) == kOpRead;
        want[1] = i2 < c1 && op_type(w, i2) == kOpRead;
        key[0] = want[0] ? key_stream(w, i) : (typename Tr::Key)0;
        key[1] = want[1] ? key_stream(w, i2) : (typename Tr::Key)0;
        h[0] = Tr::hash(key[0]);
        h[1] = Tr::hash(key[1]);
        table_find_n<Tr, 2>(t, key, h, want, found, val, loc);
        if (want[0]) write_result(w, i, kOpRead, found[0], val[0]);
        if (want[1]) write_result(w, i2, kOpRead, found[1], val[1]);
      }
    } else {
      for (uint32_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
        if (op_type(w, i) != kOpRead) continue;
        uint64_t val;
        const bool found = read_lookup<Tr>(t, key_stream(w, i), &val);
        write_result(w, i, kOpRead, found, val);
      }
    }
  }
}

// --------------------------------------------------------- region binning
// Random probes over a multi-GB table are limited by address translation:
// measured on B200, random 32-B reads over 4 GB run at ~19 G/s, but at ~48 G/s
// when each block stays inside a 32 MB region.  The fused path therefore
// probes a window in table-region order: ops are counted per region (the top
// kBinBits of the bucket index: consecutive slabs), then their indices are
// scattered into region order (perm), and the probe walks perm, so at any
// moment the grid works within one or two regions.  Each op still writes
// its own result; only the probing order changes.
constexpr uint32_t kBinBits = 6;
constexpr uint32_t kBins = 1u << kBinBits;
static_assert(kBins == 64, "the region scan gives each lane two regions");

struct BinCounters {
  uint32_t count[kBins];
  uint32_t cursor[kBins];
};

// Pass 1: per-op region (stored, one byte) and per-region counts.  Lanes of
// a warp that fall in the same region add together (hot keys would otherwise
// serialise on one shared-memory counter).  The keys are read with normal
// caching: the probe gathers them again in region order.
template <class Tr>
__device__ void phase_bin_count(const TableView& t, const Window<Tr>& w, uint8_t* obin,
                                BinCounters* bc, uint32_t shift) {
  __shared__ uint32_t hist[kBins];
  for (uint32_t b = threadIdx.x; b < kBins; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  const uint32_t nt = gridDim.x * blockDim.x, lane = threadIdx.x & 31u;
  // warp-uniform loop: every lane runs every round
  for (uint32_t i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); i0 < w.n; i0 += nt) {
    const uint32_t i = i0 + lane;
    uint32_t b = kBins;
    if (i < w.n) {
      b = ((uint32_t)Tr::hash(key_of(w, i)) & t.mask) >> shift;
      obin[i] = (uint8_t)b;
    }
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
    if (b < kBins && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&hist[b], __popc(peers));
  }
  __syncthreads();
  for (uint32_t b = threadIdx.x; b < kBins; b += blockDim.x)
    if (hist[b]) atomicAdd(&bc->count[b], hist[b]);
}

// Pass 2: each block reserves a range per region for the ops it counted in
// pass 1 (same grid-stride mapping, so the same ops) and writes their indices
// there.
template <class Tr>
__device__ void phase_bin_scatter(const Window<Tr>& w, const uint8_t* obin, uint32_t* perm,
                                  BinCounters* bc) {
  __shared__ uint32_t hist[kBins], base[kBins];
  for (uint32_t b = threadIdx.x; b < kBins; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  const uint32_t nt = gridDim.x * blockDim.x, lane = threadIdx.x & 31u;
  for (uint32_t i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); i0 < w.n; i0 += nt) {
    const uint32_t i = i0 + lane;
    const uint32_t b = i < w.n ? (obin[i] & (kBins - 1)) : kBins;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
    if (b < kBins && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&hist[b], __popc(peers));
  }
  __syncthreads();
  if (threadIdx.x < 32) {  // region starts: exclusive scan of the 64 counts
    const uint32_t c0 = ld_cg_u32(&bc->count[2 * lane]), c1 = ld_cg_u32(&bc->count[2 * lane + 1]);
    uint32_t x = c0 + c1;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
      if (lane >= (uint32_t)d) x += y;
    }
    const uint32_t start0 = x - c0 - c1;
    const uint32_t h0 = hist[2 * lane], h1 = hist[2 * lane + 1];
    base[2 * lane] = start0 + (h0 ? atomicAdd(&bc->cursor[2 * lane], h0) : 0u);
    base[2 * lane + 1] = start0 + c0 + (h1 ? atomicAdd(&bc->cursor[2 * lane + 1], h1) : 0u);
  }
  __syncthreads();
  for (uint32_t i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); i0 < w.n; i0 += nt) {
    const uint32_t i = i0 + lane;
    const uint32_t b = i < w.n ? (obin[i] & (kBins - 1)) : kBins;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t pos = 0;
    if (b < kBins && lane == leader) pos = atomicAdd(&base[b], __popc(peers));
    pos = __shfl_sync(0xFFFFFFFFu, pos, leader) + __popc(peers & ((1u << lane) - 1u));
    if (b < kBins && pos < w.n) perm[pos] = i;
  }
}

// ---------------------------------------------------------------- phase D
// Block-wide exclusive scan of one value per thread; `tmp` holds one word per
// warp.  Returns the prefix; *total receives the block sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* tmp,
                                                         uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t nwarps = (blockDim.x + 31) >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= (uint32_t)d) x += y;
  }
  if (lane == 31) tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nwarps ? tmp[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, d);
      if (lane >= (uint32_t)d) s += y;
    }
    if (lane < nwarps) tmp[lane] = s;
  }
  __syncthreads();
  uint32_t warp_base = warp ? tmp[warp - 1] : 0;
  *total = tmp[nwarps - 1];
  __syncthreads();
  return warp_base + x - v;
}

// Block-wide exclusive max-scan of one value per thread (thread order);
// `tmp` holds one word per warp.  Every thread of the block calls it.
__device__ __forceinline__ uint32_t block_exclusive_max_scan(uint32_t v, uint32_t* tmp) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t nwarps = (blockDim.x + 31) >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= (uint32_t)d) x = max(x, y);
  }
  const uint32_t excl_in_warp = __shfl_up_sync(0xFFFFFFFFu, x, 1);
  if (lane == 31) tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < nwarps ? tmp[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, d);
      if (lane >= (uint32_t)d) t = max(t, y);
    }
    if (lane < nwarps) tmp[lane] = t;
  }
  __syncthreads();
  uint32_t r = warp ? tmp[warp - 1] : 0;
  if (lane) r = max(r, excl_in_warp);
  __syncthreads();
  return r;
}

// For the members sorted[0..c) of one group, ascending op indices: each
// member's lnu = 1 + the last earlier member that is not an update, else
// `carry` (1 + such a member from before sorted[0], 0 = none).  Chunks of
// consecutive positions per thread and a block max-scan of the chunks' last
// non-update member (ascending, so the last is also the largest).  Whole
// block.
template <class Tr>
__device__ void block_lnu(const Scratch& sc, const Window<Tr>& w, const uint32_t* sorted,
                          uint32_t c, uint32_t carry) {
  __shared__ uint32_t s_mx[32];
  const uint32_t per = (c + blockDim.x - 1) / blockDim.x, j0 = threadIdx.x * per;
  uint32_t last = 0;
  for (uint32_t k = 0; k < per; ++k) {
    const uint32_t j = j0 + k;
    if (j < c) {
      const uint32_t x = sorted[j];
      if (x < w.n && op_type(w, x) != kOpUpdate) last = x + 1;
    }
  }
  uint32_t run = max(block_exclusive_max_scan(last, s_mx), carry);
  for (uint32_t k = 0; k < per; ++k) {
    const uint32_t j = j0 + k;
    if (j < c) {
      const uint32_t x = sorted[j];
      if (x < w.n) {
        sc.lnu[x] = run;
        if (op_type(w, x) != kOpUpdate) run = x + 1;
      }
    }
  }
  __syncthreads();
}

// Counting sort of op indices by a bitmap over their range [lo, hi], in
// passes of kSortChunkWords words; `get(j)` yields member j (< w.n) or an
// out-of-range value to skip.  Writes the sorted list to seg[off ..].
template <class Tr, class Get>
__device__ void bitmap_sort(const Scratch& sc, const Window<Tr>& w, uint32_t c, uint32_t off,
                            uint32_t* bits, uint32_t* pre, Get get, uint32_t* sorted) {
  __shared__ uint32_t s_lo, s_hi, s_tmp[32];
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  uint32_t lo = 0xFFFFFFFFu, hi = 0;
  for (uint32_t j = tid; j < c; j += nt) {
    const uint32_t x = get(j);
    if (x >= w.n) continue;  // never stored: skip rather than index with it
    lo = min(lo, x);
    hi = max(hi, x);
  }
  lo = __reduce_min_sync(0xFFFFFFFFu, lo);
  hi = __reduce_max_sync(0xFFFFFFFFu, hi);
  if (tid == 0) {
    s_lo = 0xFFFFFFFFu;
    s_hi = 0;
  }
  __syncthreads();
  if ((tid & 31) == 0) {
    atomicMin(&s_lo, lo);
    atomicMax(&s_hi, hi);
  }
  __syncthreads();
  lo = s_lo;
  hi = s_hi;
  __syncthreads();
  uint32_t rank_base = 0;
  const uint32_t span = kSortChunkWords * 32;
  for (uint32_t cl = lo; cl <= hi; cl += span) {
    const uint32_t words = min(kSortChunkWords, ((hi - cl) >> 5) + 1);
    for (uint32_t k = tid; k < words; k += nt) bits[k] = 0;
    __syncthreads();
    for (uint32_t j = tid; j < c; j += nt) {
      const uint32_t x = get(j);
      if (x <= hi && x >= cl && x - cl < span) atomicOr(&bits[(x - cl) >> 5], 1u << ((x - cl) & 31));
    }
    __syncthreads();
    const uint32_t per = (words + nt - 1) / nt;
    const uint32_t w0 = tid * per;
    uint32_t local = 0;
    for (uint32_t k = 0; k < per; ++k)
      if (w0 + k < words) local += __popc(bits[w0 + k]);
    uint32_t total;
    uint32_t run = block_exclusive_scan(local, s_tmp, &total);
    for (uint32_t k = 0; k < per; ++k) {
      if (w0 + k < words) {
        pre[w0 + k] = run;
        run += __popc(bits[w0 + k]);
      }
    }
    __syncthreads();
    for (uint32_t j = tid; j < c; j += nt) {
      const uint32_t x = get(j);
      if (x <= hi && x >= cl && x - cl < span) {
        const uint32_t d = x - cl, wd = d >> 5;
        const uint32_t r = rank_base + pre[wd] + __popc(bits[wd] & ((1u << (d & 31)) - 1u));
        sc.seg[off + r] = x;
        if (sorted) sorted[r] = x;
      }
    }
    rank_base += total;
    __syncthreads();
    if (hi - cl < span) break;
  }
}

// A group of kWarpSort+1 .. kHugeMin members, ordered by the whole block.
// The members are gathered into shared memory first (a warp per storage
// unit: the inline part, then each 32-member chunk with one chunk-table
// lookup), so the counting sort reads only shared memory.
template <class Tr>
__device__ void sort_group_block(const Scratch& sc, const Window<Tr>& w, uint32_t gslot,
                                 uint32_t c, uint32_t off, uint32_t* smem, bool upd) {
  uint32_t* sorted = smem + kSortSmall;
  uint32_t* bits = sorted + kSortSmall;
  uint32_t* pre = bits + kSortChunkWords;
  if (c > kSortSmall) return;  // block-uniform; larger groups take the huge_* phases
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const uint32_t nchunks = (c - kInline + kChunk - 1) / kChunk;  // <= kSortSmall / kChunk
  // all chunk-table lookups in flight at once (one per thread), parked in
  // the prefix area; then each warp copies its chunks, loads issued before
  // any store so they overlap
  for (uint32_t k = tid; k < nchunks; k += blockDim.x) pre[k] = chunk_find(sc, w.epoch, gslot, k);
  if (tid < kInline) smem[tid] = ld_cg_u32(&sc.ginl[(size_t)gslot * kInline + tid]);
  for (uint32_t j = tid; j < c; j += blockDim.x) sorted[j] = 0xFFFFFFFFu;  // holes stay invalid
  __syncthreads();
  for (uint32_t k0 = warp; k0 < nchunks; k0 += 4 * nwarps) {
    uint32_t v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t k = k0 + q * nwarps;
      const uint32_t j = kInline + k * kChunk + lane;
      const uint32_t cs = k < nchunks ? pre[k] : 0xFFFFFFFFu;
      v[q] = (j < c && cs != 0xFFFFFFFFu) ? ld_cg_u32(&sc.cdat[(size_t)cs * kChunk + lane])
                                          : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t j = kInline + (k0 + q * nwarps) * kChunk + lane;
      if (j < c) smem[j] = v[q];
    }
  }
  __syncthreads();
  bitmap_sort<Tr>(sc, w, c, off, bits, pre, [&](uint32_t j) { return smem[j]; }, sorted);
  // every member's predecessor from the sorted list in shared memory (the
  // bitmap pass ends with a __syncthreads)
  for (uint32_t j = tid; j < c; j += blockDim.x) {
    const uint32_t e = sorted[j];
    const uint32_t pe = j ? sorted[j - 1] : 0xFFFFFFFFu;
    const uint32_t p = pe < w.n ? pe + 1 : 0u;
    if (e < w.n) sc.pred[e] = p | (j + 1 == c ? kPredLast : 0u);
  }
  __syncthreads();
  if (upd) block_lnu<Tr>(sc, w, sorted, c, 0u);
}

// A group of kInline+1 .. kWarpSort members, ordered by one warp: each lane
// holds members lane + 32h (h < K) and ranks them against all others by
// shuffles, tracking each one's predecessor (the largest smaller index) on
// the way (32 K^2 compares a lane).
template <class Tr, int K>
__device__ void sort_group_warp_k(const Scratch& sc, const Window<Tr>& w, uint32_t gslot,
                                  uint32_t c, uint32_t off, bool upd) {
  const uint32_t lane = lane_id();
  uint32_t x[K];
#pragma unroll
  for (int h = 0; h < K; ++h) {
    const uint32_t j = lane + 32 * h;
    x[h] = j < c ? member_at(sc, w.epoch, gslot, j) : 0xFFFFFFFFu;
  }
  uint32_t rank[K], pred[K];
#pragma unroll
  for (int g = 0; g < K; ++g) {
    rank[g] = 0;
    pred[g] = 0xFFFFFFFFu;
  }
#pragma unroll
  for (int h = 0; h < K; ++h) {
    if (32u * h >= c) break;  // warp-uniform
    for (uint32_t q = 0; q < 32; ++q) {
      const uint32_t y = __shfl_sync(0xFFFFFFFFu, x[h], q);
#pragma unroll
      for (int g = 0; g < K; ++g) {
        if (32 * h + q < c && y < x[g]) {
          ++rank[g];
          if (pred[g] == 0xFFFFFFFFu || y > pred[g]) pred[g] = y;
        }
      }
    }
  }
#pragma unroll
  for (int g = 0; g < K; ++g) {
    const uint32_t j = lane + 32 * g;
    if (j < c && x[g] < w.n) {
      sc.seg[off + rank[g]] = x[g];
      sc.pred[x[g]] = (pred[g] < w.n ? pred[g] + 1 : 0u) | (rank[g] + 1 == c ? kPredLast : 0u);
    }
  }
  if (!upd) return;  // warp-uniform
  // lnu: the largest smaller member that is not an update
  uint32_t nu_of[K];
#pragma unroll
  for (int h = 0; h < K; ++h)
    nu_of[h] = (x[h] < w.n && op_type(w, x[h]) != kOpUpdate) ? x[h] : 0xFFFFFFFFu;
  uint32_t lnu[K];
#pragma unroll
  for (int g = 0; g < K; ++g) lnu[g] = 0;  // 1 + member, 0 = none
#pragma unroll
  for (int h = 0; h < K; ++h) {
    if (32u * h >= c) break;  // warp-uniform
    for (uint32_t q = 0; q < 32; ++q) {
      const uint32_t y = __shfl_sync(0xFFFFFFFFu, nu_of[h], q);
#pragma unroll
      for (int g = 0; g < K; ++g)
        if (y != 0xFFFFFFFFu && y < x[g] && y + 1 > lnu[g]) lnu[g] = y + 1;
    }
  }
#pragma unroll
  for (int g = 0; g < K; ++g)
    if (lane + 32 * g < c && x[g] < w.n) sc.lnu[x[g]] = lnu[g];
}

// Two members a lane: groups of up to 64.  (Four a lane, groups up to 128
// with the block sort taking only larger ones, measured slower: the fused
// kernel spilled more at its 64-register cap, 97 -> 103 us on the 2^20-op
// 95/5 batch, and the serving loop's latency did not change.)
template <class Tr>
__device__ void sort_group_warp(const Scratch& sc, const Window<Tr>& w, uint32_t gslot, uint32_t c,
                                uint32_t off, bool upd) {
  static_assert(kWarpSort == 64, "one warp holds at most 2 members a lane");
  sort_group_warp_k<Tr, 2>(sc, w, gslot, c, off, upd);
}

// Phase D: block b orders large groups b, b + gridDim.x, ... (the critical
// path); then warps take the groups of the big list by a static stride that
// starts at the warps of blocks without a large group.  No work is claimed
// through a shared counter, so no grid-wide atomic serializes the phase.
// `smem` holds kSortSmemBytes.
template <class Tr>
__device__ void phase_sort_big(const Scratch& sc, const Window<Tr>& w, uint32_t* smem) {
  __shared__ uint32_t s_off;
  const uint32_t tid = threadIdx.x;
  const bool upd = ld_cg_u32(&w.cnt->upd_count) != 0;  // settled: the probe has ended
  const uint32_t nlarge = ld_cg_u32(&w.cnt->large_count);
  for (uint32_t job = blockIdx.x; job < nlarge; job += gridDim.x) {
    const uint32_t gslot = ld_cg_u32(&sc.large[job]) & sc.gmask;
    const uint32_t c = min(g_count(ld_relaxed_u64(&sc.gtab[gslot])), w.n);
    if (c > kHugeMin) continue;  // the huge_* steps order it (c is block-uniform)
    if (tid == 0) {
      s_off = atomicAdd(&w.cnt->seg_cursor, c);
      sc.goff[gslot] = s_off;
    }
    __syncthreads();
    const uint32_t off = s_off;
    sort_group_block<Tr>(sc, w, gslot, c, off, smem, upd);  // ends with __syncthreads
  }
  const uint32_t nbig = ld_cg_u32(&w.cnt->big_count);
  const uint32_t lane = lane_id(), wpb = blockDim.x >> 5;
  const uint32_t nw = gridDim.x * wpb;
  const uint32_t busy = min(nlarge, gridDim.x) * wpb;  // warps of blocks with a large group
  const uint32_t gw = blockIdx.x * wpb + (threadIdx.x >> 5);
  for (uint32_t job = (gw + nw - busy % nw) % nw; job < nbig; job += nw) {
    const uint32_t gslot = ld_cg_u32(&sc.big[job]) & sc.gmask;
    const uint32_t c = g_count(ld_relaxed_u64(&sc.gtab[gslot]));
    if (c > kWarpSort) continue;  // a block (or the huge steps) took it
    uint32_t off = 0;
    if (lane == 0) {
      off = atomicAdd(&w.cnt->seg_cursor, c);
      sc.goff[gslot] = off;
    }
    off = __shfl_sync(0xFFFFFFFFu, off, 0);
    sort_group_warp<Tr>(sc, w, gslot, c, off, upd);
  }
}

// ------------------------------------------------------- huge groups (D')
// A group of more than kHugeMin members (a hot key) is ordered by the
// whole grid in four steps separated by grid barriers, so no block reads
// back global data that it wrote itself in the same step:
//   hist     every warp takes storage units (inline part / 32-member chunks)
//            of every huge group and counts members per index range
//            (kHugeBins equal ranges of [0, n); a range is at most kRunUnit
//            indices wide for windows up to 2^23 ops);
//   scan     a block per group: range offsets in seg, the group's runs (a run
//            starts at the first range beginning at or after each multiple of
//            kRunUnit; ranges hold at most kRunUnit members, so a run is
//            never empty and holds fewer than 2 * kRunUnit = kSortSmall) and
//            each range's run;
//   scatter  every warp again: members to their range's next free seg
//            position; each run's largest member by atomicMax;
//   runs     a block per run: counting sort in shared memory, written back
//            in place, then each member's predecessor (the previous run's
//            largest member for the first one).
constexpr uint32_t kHugeBins = 4096;
constexpr uint32_t kRunUnit = 2048;
static_assert(2 * kRunUnit == kSortSmall, "a run fits the shared-memory sort");
constexpr uint32_t kRunFirst = 1u << 30, kRunLast = 1u << 31;

__device__ __forceinline__ uint32_t huge_width(uint32_t n) {
  return (n + kHugeBins - 1) / kHugeBins;  // <= kRunUnit for n <= 2^23
}

__device__ __forceinline__ uint32_t huge_groups(const Scratch& sc, const WinCounters* c) {
  return min(ld_cg_u32(&c->huge_count), sc.hcap);
}

// Member `lane` of storage unit k of group gslot (unit 0: the inline part,
// unit k >= 1: chunk k-1), or 0xFFFFFFFF.  Whole warp.
template <class Tr>
__device__ __forceinline__ uint32_t huge_member(const Scratch& sc, const Window<Tr>& w,
                                                uint32_t gslot, uint32_t c, uint32_t k,
                                                uint32_t lane) {
  if (k == 0)
    return lane < kInline ? ld_cg_u32(&sc.ginl[(size_t)gslot * kInline + lane]) : 0xFFFFFFFFu;
  uint32_t cs = 0xFFFFFFFFu;
  if (lane == 0) cs = chunk_find(sc, w.epoch, gslot, k - 1);
  cs = __shfl_sync(0xFFFFFFFFu, cs, 0);
  const uint32_t j = kInline + (k - 1) * kChunk + lane;
  return (j < c && cs != 0xFFFFFFFFu) ? ld_cg_u32(&sc.cdat[(size_t)cs * kChunk + lane])
                                      : 0xFFFFFFFFu;
}

template <class Tr>
__device__ __forceinline__ uint32_t huge_size(const Scratch& sc, const Window<Tr>& w,
                                              uint32_t h, uint32_t* gslot) {
  *gslot = ld_cg_u32(&sc.hlist[h]) & sc.gmask;
  return min(g_count(ld_relaxed_u64(&sc.gtab[*gslot])), w.n);
}

// hist: every warp of the grid (gwarp of ngwarps).
template <class Tr>
__device__ void huge_hist(const Scratch& sc, const Window<Tr>& w, uint32_t gwarp,
                          uint32_t ngwarps) {
  const uint32_t H = huge_groups(sc, w.cnt), width = huge_width(w.n), lane = lane_id();
  for (uint32_t h = 0; h < H; ++h) {
    uint32_t gslot;
    const uint32_t c = huge_size(sc, w, h, &gslot);
    const uint32_t units = 1 + (c - kInline + kChunk - 1) / kChunk;
    uint32_t* bins = sc.hbins + (size_t)h * kHugeBins;
    for (uint32_t k = gwarp; k < units; k += ngwarps) {
      const uint32_t x = huge_member(sc, w, gslot, c, k, lane);
      const uint32_t b = x < w.n ? x / width : 0xFFFFFFFFu;
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
      if (b != 0xFFFFFFFFu && lane == (uint32_t)__ffs(peers) - 1)
        atomicAdd(&bins[b], (uint32_t)__popc(peers));
    }
  }
}

// scan: block b takes groups b, b + gridDim.x, ... (every thread derives the
// group itself: no claim is broadcast through shared memory).  `smem` holds
// kSortSmemBytes (kHugeBins words are used).
template <class Tr>
__device__ void huge_scan(const Scratch& sc, const Window<Tr>& w, uint32_t* smem) {
  __shared__ uint32_t s_off, s_base, s_last, s_tmp[32];
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  const uint32_t H = huge_groups(sc, w.cnt);
  const uint32_t per = (kHugeBins + nt - 1) / nt, b0 = tid * per;
  for (uint32_t h = blockIdx.x; h < H; h += gridDim.x) {
    if (tid == 0) s_last = 0;
    __syncthreads();
    uint32_t gslot;
    const uint32_t c = huge_size(sc, w, h, &gslot);
    uint32_t* bins = sc.hbins + (size_t)h * kHugeBins;
    uint32_t* hrun = sc.hrun + (size_t)h * kHugeBins;
    uint32_t local = 0;
    for (uint32_t k = 0; k < per; ++k)
      if (b0 + k < kHugeBins) {
        smem[b0 + k] = ld_cg_u32(&bins[b0 + k]);
        local += smem[b0 + k];
      }
    uint32_t total;
    uint32_t run = block_exclusive_scan(local, s_tmp, &total);
    total = min(total, c);
    uint32_t last = 0;  // offset of the last non-empty range
    for (uint32_t k = 0; k < per; ++k)
      if (b0 + k < kHugeBins) {
        const uint32_t n = smem[b0 + k];
        smem[b0 + k] = run;  // exclusive prefix
        if (n) last = run;
        run += n;
      }
    if (last) atomicMax(&s_last, last);
    __syncthreads();
    // run r exists when some non-empty range starts at or after r * kRunUnit,
    // so no run is empty (a range holds at most kRunUnit members)
    const uint32_t nrun = total ? min(s_last, total - 1) / kRunUnit + 1 : 0u;
    if (tid == 0) {
      s_off = atomicAdd(&w.cnt->seg_cursor, c);
      sc.goff[gslot] = s_off;
      s_base = atomicAdd(&w.cnt->run_count, nrun);
    }
    __syncthreads();
    const uint32_t off = s_off, base = s_base;
    if (tid == 0) {
      uint32_t* rec = sc.hrec + 4 * (size_t)h;
      rec[0] = off;
      rec[1] = total;
      rec[2] = base;
      rec[3] = nrun;
      if (nrun && base + nrun - 1 < sc.rcap) sc.runs[4 * (size_t)(base + nrun - 1) + 1] = off + total;
    }
    // cursors and runs of the ranges; run r begins at the first range whose
    // offset is >= r * kRunUnit (the virtual range kHugeBins sits at total)
    for (uint32_t b = tid; b <= kHugeBins; b += nt) {
      const uint32_t p = b < kHugeBins ? min(smem[b], total) : total;
      if (b < kHugeBins) {
        bins[b] = off + p;
        hrun[b] = base + min(p / kRunUnit, nrun ? nrun - 1 : 0u);
      }
      const uint32_t r0 = b ? min(smem[b - 1], total) / kRunUnit + 1 : 0u;
      for (uint32_t r = r0; r <= p / kRunUnit; ++r) {
        if (r < nrun && base + r < sc.rcap) {
          uint32_t* rr = sc.runs + 4 * (size_t)(base + r);
          rr[0] = off + p;
          rr[2] = h | (r == 0 ? kRunFirst : 0u) | (r + 1 == nrun ? kRunLast : 0u);
          rr[3] = 0;
          sc.rnu[base + r] = 0;
        }
        if (r >= 1 && r < nrun && base + r - 1 < sc.rcap)  // the last run ends at total
          sc.runs[4 * (size_t)(base + r - 1) + 1] = off + p;
      }
    }
    for (uint32_t j = total + tid; j < c; j += nt) sc.seg[off + j] = 0xFFFFFFFFu;
    __syncthreads();
  }
}

// scatter: every warp of the grid.
template <class Tr>
__device__ void huge_scatter(const Scratch& sc, const Window<Tr>& w, uint32_t gwarp,
                             uint32_t ngwarps) {
  const uint32_t H = huge_groups(sc, w.cnt), width = huge_width(w.n), lane = lane_id();
  const bool upd = ld_cg_u32(&w.cnt->upd_count) != 0;
  for (uint32_t h = 0; h < H; ++h) {
    uint32_t gslot;
    const uint32_t c = huge_size(sc, w, h, &gslot);
    const uint32_t units = 1 + (c - kInline + kChunk - 1) / kChunk;
    uint32_t* bins = sc.hbins + (size_t)h * kHugeBins;
    const uint32_t* hrun = sc.hrun + (size_t)h * kHugeBins;
    const uint32_t end =
        ld_cg_u32(&sc.hrec[4 * (size_t)h]) + ld_cg_u32(&sc.hrec[4 * (size_t)h + 1]);
    for (uint32_t k = gwarp; k < units; k += ngwarps) {
      const uint32_t x = huge_member(sc, w, gslot, c, k, lane);
      const uint32_t b = x < w.n ? x / width : 0xFFFFFFFFu;
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
      const uint32_t leader = (uint32_t)__ffs(peers) - 1;
      uint32_t p0 = 0;
      if (b != 0xFFFFFFFFu && lane == leader) p0 = atomicAdd(&bins[b], (uint32_t)__popc(peers));
      p0 = __shfl_sync(0xFFFFFFFFu, p0, leader);
      if (b == 0xFFFFFFFFu) continue;
      const uint32_t p = p0 + __popc(peers & ((1u << lane) - 1u));
      if (p < end && p < sc.max_window) {
        sc.seg[p] = x;
        const uint32_t r = ld_cg_u32(&hrun[b]);
        if (r < sc.rcap) {
          atomicMax(&sc.runs[4 * (size_t)r + 3], x + 1);
          if (upd && op_type(w, x) != kOpUpdate) atomicMax(&sc.rnu[r], x + 1);
        }
      } else {
        raise_status(sc.status, kStatusScratch);
      }
    }
  }
}

// runs: block b takes runs b, b + gridDim.x, ...; the range counters are
// cleared for the next window on the way (the scatter was their last user).
template <class Tr>
__device__ void huge_runs(const Scratch& sc, const Window<Tr>& w, uint32_t* smem, uint32_t gtid,
                          uint32_t gthreads) {
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  const uint32_t H = huge_groups(sc, w.cnt);
  for (size_t i = gtid; i < (size_t)H * kHugeBins; i += gthreads) sc.hbins[i] = 0;
  const uint32_t R = min(ld_cg_u32(&w.cnt->run_count), sc.rcap);
  const bool upd = ld_cg_u32(&w.cnt->upd_count) != 0;
  __shared__ uint32_t s_carry;
  uint32_t* sorted = smem + kSortSmall;
  uint32_t* bits = sorted + kSortSmall;
  uint32_t* pre = bits + kSortChunkWords;
  for (uint32_t r = blockIdx.x; r < R; r += gridDim.x) {
    const uint4 rec = ld_cg_v4(&sc.runs[4 * (size_t)r]);
    const uint32_t s = rec.x, e = rec.y, info = rec.z;
    uint32_t n = 0;
    if (s <= e && e - s <= kSortSmall && e <= sc.max_window)
      n = e - s;
    else if (tid == 0)
      raise_status(sc.status, kStatusScratch);
    for (uint32_t j = tid; j < n; j += nt) {
      smem[j] = ld_cg_u32(&sc.seg[s + j]);
      sorted[j] = 0xFFFFFFFFu;
    }
    __syncthreads();
    if (n) bitmap_sort<Tr>(sc, w, n, s, bits, pre, [&](uint32_t j) { return smem[j]; }, sorted);
    uint32_t first_pred = 0xFFFFFFFFu;
    if (!(info & kRunFirst) && r > 0) first_pred = ld_cg_u32(&sc.runs[4 * (size_t)(r - 1) + 3]) - 1u;
    for (uint32_t j = tid; j < n; j += nt) {
      const uint32_t x = sorted[j];
      const uint32_t pe = j ? sorted[j - 1] : first_pred;
      const bool last = (info & kRunLast) && j + 1 == n;
      if (x < w.n) sc.pred[x] = (pe < w.n ? pe + 1 : 0u) | (last ? kPredLast : 0u);
    }
    __syncthreads();
    if (upd) {  // block-uniform
      // carry: the largest non-update member of the nearest earlier run of
      // the same group that has one (each run's was recorded by the scatter)
      if (tid == 0) {
        uint32_t carry = 0, cur = r, cinfo = info;
        for (uint32_t hop = 0; hop < sc.rcap && !(cinfo & kRunFirst) && cur > 0; ++hop) {
          --cur;
          carry = ld_cg_u32(&sc.rnu[cur]);
          if (carry) break;
          cinfo = ld_cg_u32(&sc.runs[4 * (size_t)cur + 2]);
        }
        s_carry = carry;
      }
      __syncthreads();
      block_lnu<Tr>(sc, w, sorted, n, s_carry);  // ends with __syncthreads
    }
  }
}

// ------------------------------------------------------------ counters
// A table's counter block (two window-counter sets, the grid barrier and,
// for region binning, two bin-counter sets) is zero whenever none of the
// table's kernels runs.  The last block to leave a kernel that used it
// clears it for the next launch, so no memset launch precedes a batch.
// Every thread of every block calls this once, as the block's last action.
__device__ inline void release_counters(WinCounters* cnt, GridBarrier* bar, void* bins,
                                        uint32_t bin_words, uint32_t* epoch_out = nullptr,
                                        uint32_t epoch_next = 0) {
  __syncthreads();
  int last = 0;
  if (threadIdx.x == 0) {
    __threadfence();  // this block's counter updates before its exit is counted
    last = atomicAdd(&bar->exits, 1u) == gridDim.x - 1;
    if (last) __threadfence();
  }
  if (__syncthreads_or(last)) {
    uint32_t* words = reinterpret_cast<uint32_t*>(cnt);
    for (uint32_t i = threadIdx.x; i < 2 * sizeof(WinCounters) / 4; i += blockDim.x) words[i] = 0;
    uint32_t* b = static_cast<uint32_t*>(bins);
    for (uint32_t i = threadIdx.x; b && i < bin_words; i += blockDim.x) b[i] = 0;
    if (threadIdx.x == 0) bar->count = 0;
    if (threadIdx.x == 0 && epoch_out != nullptr) *epoch_out = epoch_next;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      bar->exits = 0;
    }
  }
}

// ---------------------------------------------------------------- phase E
// Last member of a small group (inline members only) before op x that is not
// an update, or 0xFFFFFFFF.
template <class Tr>
__device__ __noinline__ uint32_t inline_lnu(const Scratch& sc, const Window<Tr>& w, uint32_t gslot,
                                            uint32_t c, uint32_t x) {
  uint32_t best = 0xFFFFFFFFu;
  for (uint32_t q = 0; q < c && q < kInline; ++q) {
    const uint32_t m = ld_cg_u32(&sc.ginl[(size_t)gslot * kInline + q]);
    if (m < x && m < w.n && (best == 0xFFFFFFFFu || m > best) && op_type(w, m) != kOpUpdate)
      best = m;
  }
  return best;
}

// Whether the key of mutation x (group gslot of c members) is present just
// before x: decided by the last earlier member that is not an update (a put
// makes it present, a remove absent), else by the window's starting state,
// which the probe recorded for every member.  Only asked for updates.
template <class Tr>
__device__ __forceinline__ bool present_before(const Scratch& sc, const Window<Tr>& w,
                                               uint32_t gslot, uint32_t c, uint32_t x) {
  uint32_t l;
  if (c <= kInline) {
    l = inline_lnu<Tr>(sc, w, gslot, c, x);
  } else {
    const uint32_t e = ld_cg_u32(&sc.lnu[x]);
    l = e ? e - 1 : 0xFFFFFFFFu;
  }
  if (l < w.n) return op_type(w, l) == kOpWrite;
  return (ld_cg_u64(&sc.mloc[x]) & kLocLive) != 0;
}

// Post-state of mutation p (group gslot of c members) as (present, value):
// a put leaves {present, its value}, a remove {absent}, an update its value
// if the key was present before it and {absent} otherwise.
template <class Tr>
__device__ __forceinline__ void post_state(const Scratch& sc, const Window<Tr>& w, uint32_t p,
                                           uint32_t gslot, uint32_t c, bool* present,
                                           uint64_t* value) {
  const uint8_t pt = op_type(w, p);
  bool pres = pt == kOpWrite;
  if (pt == kOpUpdate) pres = present_before<Tr>(sc, w, gslot, c, p);
  *present = pres;
  *value = (Tr::kHasValue && pres) ? val_of(w, p) : 0ull;
}

// Inline members of a small group: predecessor of op i (or 0xFFFFFFFF) and
// whether i is the group's last mutation.
__device__ __forceinline__ uint32_t inline_pred(const Scratch& sc, uint32_t gslot, uint32_t c,
                                                uint32_t i, uint32_t n, bool* last) {
  const uint4 a = ld_cg_v4(&sc.ginl[(size_t)gslot * kInline]);
  const uint4 b = ld_cg_v4(&sc.ginl[(size_t)gslot * kInline + 4]);
  const uint32_t m[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  uint32_t best = 0xFFFFFFFFu;
  bool later = false;
#pragma unroll
  for (uint32_t q = 0; q < kInline; ++q) {
    if (q < c && m[q] < n) {
      if (m[q] < i && (best == 0xFFFFFFFFu || m[q] > best)) best = m[q];
      later |= m[q] > i;
    }
  }
  *last = !later;
  return best;
}

template <class Tr>
__device__ void phase_resolve_mutations(const TableView& t, const Scratch& sc,
                                        const Window<Tr>& w, uint32_t tid, uint32_t nthreads) {
  const uint32_t mcount = ld_cg_u32(&w.cnt->mut_count);
  for (uint32_t j = tid; j < mcount; j += nthreads) {
    const uint32_t m = ld_cg_u32(&sc.mlist[j]);
    if (m >= w.n) continue;
    // everything that depends on m alone in one round trip: the group slot,
    // the op, the slot location its probe found and its ordering record
    // (only meaningful, and only used, in groups of more than kInline)
    const uint64_t mi = ld_cg_u64(&sc.minfo[m]);
    const uint64_t loc = ld_cg_u64(&sc.mloc[m]);
    const uint32_t prec = ld_cg_u32(&sc.pred[m]);
    const uint8_t type = op_type(w, m);
    const typename Tr::Key key = key_of(w, m);
    const uint32_t gslot = (uint32_t)(mi >> 32) & sc.gmask;
    const uint32_t c = g_count(ld_relaxed_u64(&sc.gtab[gslot]));
    uint32_t pred;
    bool last = true;
    if (c == 1) {
      pred = 0xFFFFFFFFu;
    } else if (c <= kInline) {
      pred = inline_pred(sc, gslot, c, m, w.n, &last);
    } else {
      pred = (prec & kPredMask) ? (prec & kPredMask) - 1 : 0xFFFFFFFFu;
      last = (prec & kPredLast) != 0;
    }
    if (pred < w.n) {
      bool present;
      uint64_t value;
      post_state<Tr>(sc, w, pred, gslot, c, &present, &value);
      write_result(w, m, type, present, value);
    }
    if (last) {
      bool present = type == kOpWrite;
      if (type == kOpUpdate) present = present_before<Tr>(sc, w, gslot, c, m);
      const uint64_t val = (Tr::kHasValue && present) ? val_of(w, m) : 0ull;
      table_apply_known<Tr>(t, key, Tr::hash(key), loc, present, val);
    }
  }
}

template <class Tr>
__device__ void phase_resolve_reads(const Scratch& sc, const Window<Tr>& w, uint32_t tid,
                                    uint32_t nthreads) {
  const uint32_t first = ~ld_cg_u32(&w.cnt->inv_first_mut);
  if (first >= w.n) return;
  for (uint32_t i = first + 1 + tid; i < w.n; i += nthreads) {
    const uint8_t type = op_type(w, i);
    if (type != kOpRead) continue;
    const typename Tr::Key key = key_of(w, i);
    const uint64_t h = Tr::hash(key);
    uint32_t slot = gslot_of(h, sc.gmask);
    uint64_t v = 0;
    bool hit = false;
    for (uint32_t probe = 0; probe <= sc.gmask; ++probe) {
      v = ld_relaxed_u64(&sc.gtab[slot]);
      if (g_epoch(v) != w.epoch) break;
      if (key_of(w, g_owner(v) - 1) == key) {
        hit = true;
        break;
      }
      slot = (slot + 1) & sc.gmask;
    }
    if (!hit) continue;
    const uint32_t c = g_count(v);
    uint32_t pred_op = 0xFFFFFFFFu;
    if (c <= kInline) {
      bool last;
      pred_op = inline_pred(sc, slot, c, i, w.n, &last);
    } else {
      const uint32_t off = ld_cg_u32(&sc.goff[slot]);
      if (off > sc.max_window || c > sc.max_window - off) continue;
      uint32_t lo = 0, hi = c;  // count of members < i
      while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (ld_cg_u32(&sc.seg[off + mid]) < i)
          lo = mid + 1;
        else
          hi = mid;
      }
      if (lo > 0) pred_op = ld_cg_u32(&sc.seg[off + lo - 1]);
    }
    if (pred_op < w.n) {
      bool present;
      uint64_t value;
      post_state<Tr>(sc, w, pred_op, slot, c, &present, &value);
      write_result(w, i, type, present, value);
    }
  }
}

}  // namespace lsb
