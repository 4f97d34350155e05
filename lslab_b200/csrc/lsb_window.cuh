// The batch engine: runs a window of ops (reads and mutations, any mix, any
// key repetition) with results equal to running them one at a time in index
// order.
//
// Phases of one window (each a grid-stride pass; a grid-wide barrier or a
// kernel boundary between them):
//   A probe     every op reads the table (pre-window state) and writes that
//               as its tentative result; mutations join a per-key group in a
//               scratch hash table (open addressing, epoch-tagged slots so
//               nothing is cleared between windows) and list themselves.
//   B segment   each group with more than one mutation reserves a segment.
//   C scatter   mutations write their op index into their group's segment.
//   D sort      segments are sorted by op index (one thread for <= 16
//               entries, a block-wide bitmap counting sort above), and each
//               mutation learns its predecessor in index order and whether
//               it is the group's last.
//   E resolve   a mutation with a predecessor takes its result from it (the
//               predecessor's post-state: put -> {1, value}, remove -> {0, 0});
//               each group's last mutation writes the final state to the
//               table; a read after the window's first mutation looks its key
//               up among the groups and, if some mutation of that key precedes
//               it, takes its result from the latest one (binary search of the
//               sorted segment).
// Only phase E writes the table, and only one thread per key does, so no
// read ever races a same-key write; reads of other keys in the same bucket
// stay correct because the apply publishes slots with a fence before the tag.
//
// The reference runs each op under a per-bucket warp lock in lane order within
// a warp and in lock-acquisition order across warps
// (include/lslab/detail/traverse.h:39-143); the engine replaces that with an
// order fixed by op index, computed without locks on the read path.
#pragma once

#include "lsb_core.cuh"

namespace lsb {

constexpr uint32_t kSmallGroup = 16;
constexpr uint32_t kPredLast = 0x80000000u;
constexpr uint32_t kPredMask = 0x7FFFFFFFu;  // predecessor op index + 1; 0 = none
constexpr uint32_t kSortChunkWords = 4096;  // bitmap words per counting-sort chunk
constexpr uint32_t kSortSmemBytes = 2 * kSortChunkWords * 4;

// Group-table slot: bits 0..23 owner (op index + 1), 24..47 count, 48..63 epoch.
__device__ __forceinline__ uint32_t g_owner(uint64_t v) { return (uint32_t)(v & 0xFFFFFFu); }
__device__ __forceinline__ uint32_t g_count(uint64_t v) { return (uint32_t)((v >> 24) & 0xFFFFFFu); }
__device__ __forceinline__ uint32_t g_epoch(uint64_t v) { return (uint32_t)(v >> 48); }

// All counters start at zero, so a set is reset with a plain memset.
struct WinCounters {
  uint32_t mut_count;
  uint32_t seg_cursor;
  uint32_t big_count;
  uint32_t big_work;
  uint32_t inv_first_mut;  // ~(lowest mutation index); 0 = no mutation
  uint32_t pad[3];
};

__device__ inline void win_counters_reset(WinCounters* c) {
  c->mut_count = 0;
  c->seg_cursor = 0;
  c->big_count = 0;
  c->big_work = 0;
  c->inv_first_mut = 0;
}

// Scratch owned by a table, sized for max_window ops.
struct Scratch {
  uint64_t* gtab;   // group table, gmask + 1 slots
  uint32_t gmask;
  uint32_t max_window;
  uint64_t* minfo;  // per op: group slot << 32 | position in group
  uint32_t* pred;   // per op: predecessor + 1 | kPredLast
  uint32_t* goff;   // per group slot: segment offset
  uint32_t* seg;    // unsorted segments
  uint32_t* sseg;   // sorted segments
  uint32_t* mlist;  // mutation op indices
  uint32_t* big;    // group slots with more than kSmallGroup mutations
  WinCounters* cnt; // two sets, used by alternate windows
};

enum : uint32_t { kOutNone = 0, kOutResult = 1, kOutOld = 2, kOutBool = 3 };

template <class Tr>
struct Window {
  const uint8_t* types;  // null: every op has type `uniform`
  const typename Tr::Key* keys;
  const uint64_t* vals;  // map puts
  void* out;
  uint32_t kstride;      // elements between consecutive keys (2 for AoS pairs)
  uint32_t vstride;      // elements between consecutive values
  uint32_t n;
  uint32_t epoch;  // 1..65535
  uint8_t uniform;
  uint8_t out_kind;
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
  return w.vals[(size_t)i * w.vstride];
}

// Result of op i given the key's state just before it.
template <class Tr>
__device__ __forceinline__ void write_result(const Window<Tr>& w, uint32_t i, uint8_t type,
                                             bool found, uint64_t value) {
  switch (w.out_kind) {
    case kOutResult: {
      // two 8-byte stores: lsb_result arrays are only 8-byte aligned in C
      uint64_t* p = (uint64_t*)w.out + 2 * (size_t)i;
      st_cg_u64(p, found ? 1ull : 0ull);
      st_cg_u64(p + 1, found ? value : 0ull);
      break;
    }
    case kOutOld:
      ((uint64_t*)w.out)[i] = found ? value : 0ull;
      break;
    case kOutBool:
      ((uint8_t*)w.out)[i] = (type == kOpWrite) ? 1 : (found ? 1 : 0);
      break;
    default:
      break;
  }
}

__device__ __forceinline__ uint32_t lane_id() {
  uint32_t l;
  asm("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}

// ---------------------------------------------------------------- phase A
// Returns the op's group slot and position through minfo; mutation indices
// are appended to mlist (warp-aggregated).
template <class Tr>
__device__ __forceinline__ void group_join(const Scratch& sc, const Window<Tr>& w, uint32_t i,
                                           typename Tr::Key key, uint64_t h) {
  uint32_t slot = (uint32_t)(h >> 20) & sc.gmask;
  const uint64_t mine = ((uint64_t)w.epoch << 48) | (1ull << 24) | (uint64_t)(i + 1);
  for (uint32_t probe = 0; probe <= sc.gmask; ++probe) {
    uint64_t v = ld_relaxed_u64(&sc.gtab[slot]);
    if (g_epoch(v) != w.epoch) {
      uint64_t prev = atomicCAS((unsigned long long*)&sc.gtab[slot], v, mine);
      if (prev == v) {
        sc.minfo[i] = ((uint64_t)slot << 32);
        return;
      }
      v = prev;
      if (g_epoch(v) != w.epoch) {  // changed but still stale: retry this slot
        --probe;
        continue;
      }
    }
    if (key_of(w, g_owner(v) - 1) == key) {
      uint64_t old = atomicAdd((unsigned long long*)&sc.gtab[slot], 1ull << 24);
      sc.minfo[i] = ((uint64_t)slot << 32) | g_count(old);
      return;
    }
    slot = (slot + 1) & sc.gmask;
  }
}

// Phase A over ops [begin, end) with a warp-uniform grid stride.  kGroup:
// mutations join groups (false for read-only batches).  kDedup: lanes of a
// warp that carry the same key share one probe.
template <class Tr, bool kGroup, bool kDedup>
__device__ void phase_probe(const TableView& t, const Scratch& sc, const Window<Tr>& w,
                            uint32_t warp_id, uint32_t num_warps) {
  const uint32_t lane = lane_id();
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  for (uint32_t base = warp_id * 32; base < w.n; base += num_warps * 32) {
    const uint32_t i = base + lane;
    const bool active = i < w.n;
    const uint8_t type = active ? op_type(w, i) : kOpRead;
    const typename Tr::Key key = active ? key_of(w, i) : (typename Tr::Key)0;
    const uint64_t h = Tr::hash(key);
    bool found = false;
    uint64_t value = 0;
    bool leader = active;
    uint32_t src = lane;
    if (kDedup) {
      const uint32_t am = __ballot_sync(0xFFFFFFFFu, active);
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key) & am;
      src = active ? (uint32_t)(__ffs(peers) - 1) : lane;
      leader = active && src == lane;
    }
    if (leader) {
      const uint32_t bucket = (uint32_t)h & t.mask;
      if (t.lock_mode == kLockRW) {
        if (lock_reader(t, bucket)) {
          found = table_find<Tr>(t, key, h, &value);
          unlock_reader(t, bucket);
        }
      } else {
        found = table_find<Tr>(t, key, h, &value);
      }
    }
    if (kDedup) {
      found = __shfl_sync(0xFFFFFFFFu, found, src);
      value = __shfl_sync(0xFFFFFFFFu, value, src);
    }
    if (active) write_result(w, i, type, found, value);
    if (kGroup) {
      const bool is_mut = active && type != kOpRead;
      const uint32_t mm = __ballot_sync(0xFFFFFFFFu, is_mut);
      if (mm) {
        uint32_t first = __reduce_min_sync(0xFFFFFFFFu, is_mut ? i : 0xFFFFFFFFu);
        uint32_t slot_base = 0;
        const uint32_t ldr = __ffs(mm) - 1;
        if (lane == ldr) {
          slot_base = atomicAdd(&w.cnt->mut_count, (uint32_t)__popc(mm));
          atomicMax(&w.cnt->inv_first_mut, ~first);
        }
        slot_base = __shfl_sync(0xFFFFFFFFu, slot_base, ldr);
        if (is_mut) {
          sc.mlist[slot_base + __popc(mm & lanemask_lt)] = i;
          group_join<Tr>(sc, w, i, key, h);
        }
      }
    }
  }
}

// ---------------------------------------------------------------- phase B
template <class Tr>
__device__ void phase_segments(const Scratch& sc, const Window<Tr>& w, uint32_t tid,
                               uint32_t nthreads) {
  const uint32_t mcount = ld_cg_u32(&w.cnt->mut_count);
  for (uint32_t j = tid; j < mcount; j += nthreads) {
    const uint32_t m = ld_cg_u32(&sc.mlist[j]);
    const uint64_t mi = ld_cg_u64(&sc.minfo[m]);
    const uint32_t slot = (uint32_t)(mi >> 32), pos = (uint32_t)mi;
    const uint32_t c = g_count(ld_relaxed_u64(&sc.gtab[slot]));
    if (c == 1) {
      sc.pred[m] = kPredLast;
    } else if (pos == 0) {
      sc.goff[slot] = atomicAdd(&w.cnt->seg_cursor, c);
      if (c > kSmallGroup) sc.big[atomicAdd(&w.cnt->big_count, 1u)] = slot;
    }
  }
}

// ---------------------------------------------------------------- phase C
template <class Tr>
__device__ void phase_scatter(const Scratch& sc, const Window<Tr>& w, uint32_t tid,
                              uint32_t nthreads) {
  const uint32_t mcount = ld_cg_u32(&w.cnt->mut_count);
  for (uint32_t j = tid; j < mcount; j += nthreads) {
    const uint32_t m = ld_cg_u32(&sc.mlist[j]);
    const uint64_t mi = ld_cg_u64(&sc.minfo[m]);
    const uint32_t slot = (uint32_t)(mi >> 32), pos = (uint32_t)mi;
    const uint32_t c = g_count(ld_relaxed_u64(&sc.gtab[slot]));
    if (c > 1) sc.seg[ld_cg_u32(&sc.goff[slot]) + pos] = m;
  }
}

// ---------------------------------------------------------------- phase D
template <class Tr>
__device__ void phase_sort_small(const Scratch& sc, const Window<Tr>& w, uint32_t tid,
                                 uint32_t nthreads) {
  const uint32_t mcount = ld_cg_u32(&w.cnt->mut_count);
  for (uint32_t j = tid; j < mcount; j += nthreads) {
    const uint32_t m = ld_cg_u32(&sc.mlist[j]);
    const uint64_t mi = ld_cg_u64(&sc.minfo[m]);
    const uint32_t slot = (uint32_t)(mi >> 32), pos = (uint32_t)mi;
    if (pos != 0) continue;
    const uint32_t c = g_count(ld_relaxed_u64(&sc.gtab[slot]));
    if (c < 2 || c > kSmallGroup) continue;
    const uint32_t off = ld_cg_u32(&sc.goff[slot]);
    uint32_t e[kSmallGroup];
    for (uint32_t a = 0; a < c; ++a) {
      uint32_t x = ld_cg_u32(&sc.seg[off + a]);
      uint32_t b = a;
      while (b > 0 && e[b - 1] > x) {
        e[b] = e[b - 1];
        --b;
      }
      e[b] = x;
    }
    for (uint32_t a = 0; a < c; ++a) {
      sc.sseg[off + a] = e[a];
      sc.pred[e[a]] = (a ? e[a - 1] + 1 : 0u) | (a + 1 == c ? kPredLast : 0u);
    }
  }
}

// Block-wide exclusive scan of one value per thread; returns the prefix and
// the block total.  `tmp` holds one word per warp.
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
    if (lane < nwarps) tmp[lane] = s;  // inclusive warp prefix
  }
  __syncthreads();
  uint32_t warp_base = warp ? tmp[warp - 1] : 0;
  *total = tmp[nwarps - 1];
  __syncthreads();
  return warp_base + x - v;
}

// Sort the segments of big groups: each block takes groups from the list and
// orders their op indices by a bitmap counting sort in shared memory, chunk by
// chunk over the index range.  `smem` holds 2 * kSortChunkWords words.
template <class Tr>
__device__ void phase_sort_big(const Scratch& sc, const Window<Tr>& w, uint32_t* smem) {
  __shared__ uint32_t s_job, s_lo, s_hi, s_tmp[32];
  uint32_t* bits = smem;
  uint32_t* pre = smem + kSortChunkWords;
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  const uint32_t nbig = ld_cg_u32(&w.cnt->big_count);
  for (;;) {
    if (tid == 0) s_job = atomicAdd(&w.cnt->big_work, 1u);
    __syncthreads();
    const uint32_t job = s_job;
    if (job >= nbig) break;
    const uint32_t slot = ld_cg_u32(&sc.big[job]);
    const uint32_t c = g_count(ld_relaxed_u64(&sc.gtab[slot]));
    const uint32_t off = ld_cg_u32(&sc.goff[slot]);
    uint32_t lo = 0xFFFFFFFFu, hi = 0;
    for (uint32_t j = tid; j < c; j += nt) {
      uint32_t x = ld_cg_u32(&sc.seg[off + j]);
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
    uint32_t rank_base = 0;
    const uint32_t span = kSortChunkWords * 32;
    for (uint32_t cl = lo; cl <= hi; cl += span) {
      for (uint32_t k = tid; k < kSortChunkWords; k += nt) bits[k] = 0;
      __syncthreads();
      for (uint32_t j = tid; j < c; j += nt) {
        uint32_t x = ld_cg_u32(&sc.seg[off + j]);
        if (x >= cl && x - cl < span) atomicOr(&bits[(x - cl) >> 5], 1u << ((x - cl) & 31));
      }
      __syncthreads();
      // each thread owns a contiguous run of words
      const uint32_t per = (kSortChunkWords + nt - 1) / nt;
      const uint32_t w0 = tid * per;
      uint32_t local = 0;
      for (uint32_t k = 0; k < per; ++k)
        if (w0 + k < kSortChunkWords) local += __popc(bits[w0 + k]);
      uint32_t total;
      uint32_t run = block_exclusive_scan(local, s_tmp, &total);
      for (uint32_t k = 0; k < per; ++k) {
        if (w0 + k < kSortChunkWords) {
          pre[w0 + k] = run;
          run += __popc(bits[w0 + k]);
        }
      }
      __syncthreads();
      for (uint32_t j = tid; j < c; j += nt) {
        uint32_t x = ld_cg_u32(&sc.seg[off + j]);
        if (x >= cl && x - cl < span) {
          uint32_t d = x - cl, wd = d >> 5;
          uint32_t r = rank_base + pre[wd] + __popc(bits[wd] & ((1u << (d & 31)) - 1u));
          sc.sseg[off + r] = x;
        }
      }
      rank_base += total;
      __syncthreads();
      if (hi - cl < span) break;  // last chunk (also guards cl overflow)
    }
    __threadfence_block();
    __syncthreads();
    for (uint32_t j = tid; j < c; j += nt) {
      uint32_t e = ld_cg_u32(&sc.sseg[off + j]);
      uint32_t p = j ? ld_cg_u32(&sc.sseg[off + j - 1]) + 1 : 0u;
      sc.pred[e] = p | (j + 1 == c ? kPredLast : 0u);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- phase E
// Post-state of mutation p as (present, value).
template <class Tr>
__device__ __forceinline__ void post_state(const Window<Tr>& w, uint32_t p, bool* present,
                                           uint64_t* value) {
  const uint8_t pt = op_type(w, p);
  *present = pt == kOpWrite;
  *value = (Tr::kHasValue && pt == kOpWrite) ? val_of(w, p) : 0ull;
}

template <class Tr>
__device__ void phase_resolve_mutations(const TableView& t, const Scratch& sc,
                                        const Window<Tr>& w, uint32_t tid, uint32_t nthreads) {
  const uint32_t mcount = ld_cg_u32(&w.cnt->mut_count);
  for (uint32_t j = tid; j < mcount; j += nthreads) {
    const uint32_t m = ld_cg_u32(&sc.mlist[j]);
    const uint32_t p = ld_cg_u32(&sc.pred[m]);
    const uint8_t type = op_type(w, m);
    if (p & kPredMask) {
      bool present;
      uint64_t value;
      post_state(w, (p & kPredMask) - 1, &present, &value);
      write_result(w, m, type, present, value);
    }
    if (p & kPredLast) {
      const typename Tr::Key key = key_of(w, m);
      const bool present = type == kOpWrite;
      const uint64_t val = (Tr::kHasValue && present) ? val_of(w, m) : 0ull;
      table_apply<Tr>(t, key, Tr::hash(key), present, val);
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
    uint32_t slot = (uint32_t)(h >> 20) & sc.gmask;
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
    if (c == 1) {
      const uint32_t o = g_owner(v) - 1;
      if (o < i) pred_op = o;
    } else {
      const uint32_t off = ld_cg_u32(&sc.goff[slot]);
      uint32_t lo = 0, hi = c;  // count of entries < i
      while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (ld_cg_u32(&sc.sseg[off + mid]) < i)
          lo = mid + 1;
        else
          hi = mid;
      }
      if (lo > 0) pred_op = ld_cg_u32(&sc.sseg[off + lo - 1]);
    }
    if (pred_op != 0xFFFFFFFFu) {
      bool present;
      uint64_t value;
      post_state(w, pred_op, &present, &value);
      write_result(w, i, type, present, value);
    }
  }
}

}  // namespace lsb
