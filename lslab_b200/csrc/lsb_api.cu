// Host side of the library: table objects, kernel launches, the C-ABI of
// include/lsb.h.  Every batched entry point is asynchronous on the caller's
// stream; argument errors are returned, device errors land in the table's
// status word.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <map>
#include <mutex>
#include <cstring>
#include <new>
#include <vector>

#include "lsb.h"
#include "lsb_core.cuh"
#include "lsb_gather.cuh"
#include "lsb_internal.h"
#include "lsb_window.cuh"

using namespace lsb;

namespace {

constexpr uint32_t kDefaultWindow = 1u << 20;
constexpr uint32_t kMaxWindow = 1u << 23;  // owner field of a group slot is 24 bits
constexpr uint32_t kTraceCap = 1024;        // phase-trace entries per fused launch
constexpr uint32_t kFusedEpochs = 32767;    // odd epochs 1..65535 for fused windows
constexpr uint32_t kPlainEpochs = 32767;    // even epochs 2..65534 for per-phase windows
// One allocation for everything a fused launch zeroes first: two window
// counter sets, the grid barrier, two region-counter sets.
constexpr size_t kBinsOffset = 256;
constexpr size_t kCounterBytes = kBinsOffset + 2 * sizeof(BinCounters);
static_assert(2 * sizeof(WinCounters) + sizeof(GridBarrier) <= kBinsOffset, "counter block");

// Device arrays must be naturally aligned for their element type; a
// misaligned device access would fault the context, so it is refused here.
inline bool aligned(const void* p, size_t a) { return ((uintptr_t)p & (a - 1)) == 0; }

#define LSB_CK(call)                         \
  do {                                       \
    cudaError_t e_ = (call);                 \
    if (e_ != cudaSuccess) return LSB_ERR_CUDA; \
  } while (0)

// ------------------------------------------------------------- kernels
// Every kernel is bounded to 64 registers a thread (launch bound 1024), so any
// block size from 128 to 1024 threads can reach 2048 threads per SM.  The
// probe and fused kernels' bounds are build settings (blocks of 1024 threads
// resident per SM: 1 = up to 64 registers a thread, 2 = up to 32; or, for the
// fused kernel, LSB_FUSED_MAXNREG registers a thread at any block size).
#ifndef LSB_PROBE_MIN_BLOCKS
#define LSB_PROBE_MIN_BLOCKS 1
#endif
#ifndef LSB_FUSED_MIN_BLOCKS
#define LSB_FUSED_MIN_BLOCKS 1
#endif
#ifndef LSB_FUSED_LEAN_READS
#define LSB_FUSED_LEAN_READS 1
#endif
// Two-stream window form (tuning overlap): LSB_OVERLAP_SPLIT 1 = the mutation
// steps as three kernels (list, probe from the list, ordering), 0 = one
// cooperative kernel; LSB_OVERLAP_READ_BLOCKS = read-kernel blocks per SM
// (a grid-stride grid that leaves room on every SM for the mutation steps;
// 0 = one thread per op).  Measured on the 2^20-op 95/5 batch (per batch):
// 1/0 75.8 us, 1/4 78.6, 1/6 81.8, 1/7 79.6, 0/6 101.9; per-op-type calls
// 77.8 us.  With the resolve launch held to one wave of blocks: 1/0
// 69.6-70.7 us; the reads started after the listing 70.5-71.3; the
// mutations probed in op order by warps that skip tiles of reads (no list,
// an epoch-check kernel first) 73.8-74.4; per-op-type calls 77.1-77.3.
#ifndef LSB_OVERLAP_SPLIT
#define LSB_OVERLAP_SPLIT 1
#endif
#ifndef LSB_OVERLAP_READ_BLOCKS
#define LSB_OVERLAP_READ_BLOCKS 0
#endif
// threads per block of the ordering kernel k_sort (one block per SM; a
// block orders one big group at a time)
#ifndef LSB_SORT_THREADS
#define LSB_SORT_THREADS 256
#endif
// two read lookups in flight per thread in the fused kernel's lean read
// loop: measured slower at the 64-register cap (more spills), so off
#ifndef LSB_FUSED_READ_PAIR
#define LSB_FUSED_READ_PAIR 0
#endif
template <class Tr, bool kGroup, int P>
__global__ void __launch_bounds__(1024, LSB_PROBE_MIN_BLOCKS)
    k_probe(TableView t, Scratch sc, Window<Tr> w, uint32_t chunk, uint32_t dedup) {
  const uint32_t warp = spread_warp();
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  phase_probe<Tr, kGroup, P>(t, sc, w, warp, nwarps, &w.cnt->probe_cursor, chunk, dedup != 0);
}

// Windows run as launches on two streams (Table::run_plain, tuning overlap)
// take their epochs from the device counter of the fused path, so a CUDA
// graph of them can be replayed: every kernel of the window reads the
// counter f (written only by the window's last block, in k_resolve) and uses
// epoch 2f+1, or 1 after the tables were cleared when the epochs ran out.
__device__ __forceinline__ uint32_t dev_window_slot(const uint32_t* fused_epoch) {
  const uint32_t f = ld_cg_u32(fused_epoch);
  return f + 1 > kFusedEpochs ? 0u : f;
}

// A read's result in the caller's layout.
__device__ __forceinline__ void store_read(void* out, uint32_t out_kind, uint32_t i, bool found,
                                           uint64_t val) {
  if (out_kind == kOutResult) {
    uint64_t* p = (uint64_t*)out + 2 * (size_t)i;
    st_cs_u64(p, found ? 1ull : 0ull);
    st_cs_u64(p + 1, found ? val : 0ull);
  } else if (out_kind == kOutResult32) {
    st_cs_u64((uint64_t*)out + i, found ? (1ull | (val << 32)) : 0ull);
  } else if (out_kind == kOutBool) {
    st_cs_u8((uint8_t*)out + i, found ? 1 : 0);
  }
}

// Read-only batch (get / contains) in its lean form: one op per thread, no
// grouping, no work claims, the result written straight out; with `types`,
// the reads of a mixed window (other ops are left to the engine).  The code is
// kept within 32 registers a thread (launch bound 256 x 8), so 2048 threads
// fit an SM: a lookup is two dependent loads (meta sector, then the
// candidate slot), latency-bound, and twice the resident warps keep twice
// the lookups in flight.  The first candidate is tried inline; a second
// candidate or a longer chain continues in find_rest.
template <class Tr>
__global__ void __launch_bounds__(256, 8)
    k_read(TableView t, const uint8_t* types, const typename Tr::Key* keys, void* out,
           uint32_t out_kind, uint32_t n) {
  using Key = typename Tr::Key;
  // one op per thread with a grid of n threads; a smaller grid strides
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (types != nullptr && __ldcs(types + i) != kOpRead) continue;
    Key key;
    if constexpr (sizeof(Key) == 8)
      key = (Key)ld_cs_u64(keys + i);
    else
      key = (Key)ld_cs_u32(keys + i);
    uint64_t val;
    const bool found = read_lookup<Tr>(t, key, &val);
    store_read(out, out_kind, i, found, val);
  }
}

// A read's result written out of op order: one 16-byte store cached in L2
// (results land scattered over the output, so streaming half-sector stores
// would make L2 fetch the rest of each sector).
__device__ __forceinline__ void store_read_scattered(void* out, uint32_t out_kind, uint32_t i,
                                                     bool found, uint64_t val) {
  if (out_kind == kOutResult)
    st_cg_v2u64((uint64_t*)out + 2 * (size_t)i, found ? 1ull : 0ull, found ? val : 0ull);
  else if (out_kind == kOutResult32)
    st_cg_u64((uint64_t*)out + i, found ? (1ull | (val << 32)) : 0ull);
  else if (out_kind == kOutBool)
    st_cg_u8((uint8_t*)out + i, found ? 1 : 0);
}

// Reads in table-region order (tuning read_order 1).  Over a table larger
// than L2, a batch's reads taken in the order of their bucket's region (64
// equal ranges of the slab array) run ~1.9x faster on Zipf keys when the
// batch arrives ordered (40 -> 21 us for 2^20 gets over 2^22 buckets): the
// repeats of a hot key and the slabs of a region meet in the same SMs'
// caches and address-translation entries.  Built on the device the order
// does not pay (measured per kernel: count 15, offsets 19, scatter 20, reads
// through the order 29 us, against 38-40 us for the reads in op order, the
// ordered reads slowed by the key gather and the scattered result stores),
// so it is off by default.  Three steps order the reads: block b counts the
// reads of ops [b * kBinChunk, ...) per region, one block turns the counts
// into region-major offsets, block b writes its reads' op indices at those
// offsets; then k_read_ordered reads through the order.
constexpr uint32_t kReadRegions = 64;
constexpr uint32_t kBinChunk = 4096;

template <class Tr>
__device__ __forceinline__ uint32_t read_region(const TableView& t, typename Tr::Key key,
                                                uint32_t shift) {
  return ((uint32_t)Tr::hash(key) & t.mask) >> shift;
}

template <class Tr>
__global__ void __launch_bounds__(256)
    k_bin_count(TableView t, const uint8_t* types, const typename Tr::Key* keys, uint32_t n,
                uint32_t shift, uint32_t* hist) {
  __shared__ uint32_t h[kReadRegions];
  if (threadIdx.x < kReadRegions) h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t base = blockIdx.x * kBinChunk, end = min(n, base + kBinChunk);
  // warp-uniform loop: every lane takes part in the aggregation
  for (uint32_t i0 = base + (threadIdx.x & ~31u); i0 < end; i0 += blockDim.x) {
    const uint32_t i = i0 + lane;
    uint32_t r = kReadRegions;
    if (i < end && (types == nullptr || types[i] == kOpRead))
      r = read_region<Tr>(t, keys[i], shift);
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, r);
    if (r < kReadRegions && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&h[r], __popc(peers));
  }
  __syncthreads();
  if (threadIdx.x < kReadRegions) hist[threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// One block: hist (region-major, m entries) becomes exclusive offsets; the
// total (the read count) goes to hist[m].
__global__ void __launch_bounds__(1024) k_bin_scan(uint32_t* hist, uint32_t m) {
  __shared__ uint32_t tmp[32];
  const uint32_t per = (m + blockDim.x - 1) / blockDim.x, j0 = threadIdx.x * per;
  uint32_t local = 0;
  for (uint32_t k = 0; k < per; ++k)
    if (j0 + k < m) local += hist[j0 + k];
  uint32_t total;
  uint32_t run = block_exclusive_scan(local, tmp, &total);
  for (uint32_t k = 0; k < per; ++k)
    if (j0 + k < m) {
      const uint32_t c = hist[j0 + k];
      hist[j0 + k] = run;
      run += c;
    }
  if (threadIdx.x == 0) hist[m] = total;
}

template <class Tr>
__global__ void __launch_bounds__(256)
    k_bin_scatter(TableView t, const uint8_t* types, const typename Tr::Key* keys, uint32_t n,
                  uint32_t shift, const uint32_t* offs, uint32_t* order) {
  __shared__ uint32_t cur[kReadRegions];
  if (threadIdx.x < kReadRegions) cur[threadIdx.x] = offs[threadIdx.x * gridDim.x + blockIdx.x];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t base = blockIdx.x * kBinChunk, end = min(n, base + kBinChunk);
  for (uint32_t i0 = base + (threadIdx.x & ~31u); i0 < end; i0 += blockDim.x) {
    const uint32_t i = i0 + lane;
    uint32_t r = kReadRegions;
    if (i < end && (types == nullptr || types[i] == kOpRead))
      r = read_region<Tr>(t, keys[i], shift);
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, r);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t pos = 0;
    if (r < kReadRegions && lane == leader) pos = atomicAdd(&cur[r], __popc(peers));
    pos = __shfl_sync(0xFFFFFFFFu, pos, leader) + __popc(peers & ((1u << lane) - 1u));
    if (r < kReadRegions && pos < n) order[pos] = i;
  }
}

// The reads through the region order: thread t serves op order[t] for t
// below the read count (order[n] holds nothing; the count is hist's total).
template <class Tr>
__global__ void __launch_bounds__(256, 8)
    k_read_ordered(TableView t, const uint32_t* order, const uint32_t* count,
                   const typename Tr::Key* keys, void* out, uint32_t out_kind, uint32_t n) {
  const uint32_t c = min(ld_cg_u32(count), n);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < c; k += gridDim.x * blockDim.x) {
    const uint32_t i = ld_cs_u32(order + k);
    if (i >= n) continue;  // read back from scratch: checked before use
    uint64_t val;
    const bool found = read_lookup<Tr>(t, (typename Tr::Key)keys[i], &val);
    store_read_scattered(out, out_kind, i, found, val);
  }
}

// Read-only batch through the warp-cooperative probe of the reference's
// design (include/lslab/detail/traverse.h:39-96), kept as a measured
// alternative to k_read: each warp serves the distinct keys of its 32 lanes
// one at a time (lanes with the same key share one lookup, found with
// __match_any_sync); for every slab of the chain, lane l < kSlots reads
// slot l's tag and its key and value together (the warp reads the slab's
// whole key area, 14 sectors, plus the meta sector), and __ballot_sync finds
// the match.  k_read reads 2 sectors per hit instead.
template <class Tr>
__global__ void __launch_bounds__(256)
    k_read_coop(TableView t, const typename Tr::Key* keys, void* out, uint32_t out_kind,
                uint32_t n) {
  using Key = typename Tr::Key;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u;
  const bool active = i < n;
  const Key key = active ? keys[i] : (Key)0;
  const uint32_t act = __ballot_sync(0xFFFFFFFFu, active);
  const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key) & act;
  const uint32_t leader = active ? (uint32_t)__ffs(peers) - 1 : lane;
  uint32_t todo = __ballot_sync(0xFFFFFFFFu, active && leader == lane);
  bool my_found = false;
  uint64_t my_val = 0;
  while (todo) {  // warp-uniform
    const uint32_t src = __ffs(todo) - 1;
    todo &= todo - 1;
    const Key k = __shfl_sync(0xFFFFFFFFu, key, src);
    const uint64_t h = Tr::hash(k);
    const uint32_t live = 0x80u | fingerprint(h);
    uint32_t s = (uint32_t)h & t.mask;
    bool found = false;
    uint64_t val = 0;
    for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
      const uint8_t* slab = slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes);
      bool match = false;
      uint64_t v = 0;
      if (lane < (uint32_t)kSlots) {
        const uint32_t tw = ld_ca_u32(slab + 4 + 4 * (lane >> 2));
        const uint32_t tag = (tw >> (8 * (lane & 3))) & 0xFFu;
        if constexpr (Tr::kHasValue) {
          const ulonglong2 kv = ld_ca_v2u64(slab + kMetaBytes + lane * Tr::kSlotBytes);
          match = tag == live && kv.x == (uint64_t)k;
          v = kv.y;
        } else {
          match = tag == live && ld_ca_u32(slab + kMetaBytes + lane * Tr::kSlotBytes) == (uint32_t)k;
        }
      }
      const uint32_t next = ld_ca_u32(slab);
      const uint32_t hit = __ballot_sync(0xFFFFFFFFu, match);
      if (hit) {
        found = true;
        val = __shfl_sync(0xFFFFFFFFu, v, __ffs(hit) - 1);
        break;
      }
      if (next == 0) break;
      s = next;
    }
    if (lane == src) {
      my_found = found;
      my_val = val;
    }
  }
  const bool found = __shfl_sync(0xFFFFFFFFu, my_found, leader);
  const uint64_t val = __shfl_sync(0xFFFFFFFFu, my_val, leader);
  if (!active) return;
  if (out_kind == kOutResult) {
    uint64_t* p = (uint64_t*)out + 2 * (size_t)i;
    st_cs_u64(p, found ? 1ull : 0ull);
    st_cs_u64(p + 1, found ? val : 0ull);
  } else if (out_kind == kOutResult32) {
    st_cs_u64((uint64_t*)out + i, found ? (1ull | (val << 32)) : 0ull);
  } else if (out_kind == kOutBool) {
    st_cs_u8((uint8_t*)out + i, found ? 1 : 0);
  }
}

// Ordering of the window's big groups; when hot keys produced groups of
// more than kSortSmall members, the grid (a cooperative launch) continues
// with the huge_* steps between grid barriers.
// fused_epoch: the window's epoch is the device one (the two-stream form).
template <class Tr>
__global__ void __launch_bounds__(1024, 1)
    k_sort(Scratch sc, Window<Tr> w, GridBarrier* bar, const uint32_t* fused_epoch) {
  extern __shared__ uint32_t smem[];
  if (fused_epoch != nullptr) w.epoch = 2 * dev_window_slot(fused_epoch) + 1;
  phase_sort_big<Tr>(sc, w, smem);
  if (huge_groups(sc, w.cnt) == 0) return;  // grid-uniform: the probe kernel has ended
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gthreads = gridDim.x * blockDim.x;
  uint32_t seq = 0;
  huge_hist<Tr>(sc, w, gtid >> 5, gthreads >> 5);
  if (!grid_barrier(bar, gridDim.x, sc.status, seq)) return;
  huge_scan<Tr>(sc, w, smem);
  if (!grid_barrier(bar, gridDim.x, sc.status, seq)) return;
  huge_scatter<Tr>(sc, w, gtid >> 5, gthreads >> 5);
  if (!grid_barrier(bar, gridDim.x, sc.status, seq)) return;
  huge_runs<Tr>(sc, w, smem, gtid, gthreads);
}

// The mutation steps of the two-stream form as separate kernels of 256-thread
// blocks (LSB_OVERLAP_SPLIT 1): list, then probe and group from the list;
// the ordering is k_sort.  The window's epoch is the device one.
template <class Tr>
__global__ void __launch_bounds__(256) k_list_muts(Scratch sc, Window<Tr> w,
                                                   const uint32_t* fused_epoch) {
  if (ld_cg_u32(fused_epoch) + 1 > kFusedEpochs) {  // epochs ran out: clear the tables
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nt = (size_t)gridDim.x * blockDim.x;
    for (size_t i = tid; i <= sc.gmask; i += nt) sc.gtab[i] = 0;
    for (size_t i = tid; i <= sc.cmask; i += nt) sc.ctab[i] = 0;
  }
  phase_list_muts<Tr>(sc, w, spread_warp(), (gridDim.x * blockDim.x) >> 5);
}

template <class Tr>
__global__ void __launch_bounds__(256, 4)
    k_probe_list(TableView t, Scratch sc, Window<Tr> w, const uint32_t* fused_epoch) {
  w.epoch = 2 * dev_window_slot(fused_epoch) + 1;
  phase_probe_list<Tr>(t, sc, w, spread_warp(), (gridDim.x * blockDim.x) >> 5, false);
}

// The mutation steps of a window whose reads run beside it in k_read (the
// two-stream form, tuning overlap), in one cooperative launch of one
// 256-thread block per SM, launched first so its blocks are resident before
// the read kernel takes the rest of each SM: clear the group and chunk
// tables if the device epochs ran out, list the mutations in op-index order,
// probe and group them from the list, order the big groups (hot keys by the
// multi-step grid algorithm), with grid barriers between the steps.  Reads
// are neither probed nor resolved here.
template <class Tr>
__global__ void __launch_bounds__(256, 4)
    k_mutations(TableView t, Scratch sc, Window<Tr> w, GridBarrier* bar,
                const uint32_t* fused_epoch) {
  extern __shared__ uint32_t smem[];
  const uint32_t f = ld_cg_u32(fused_epoch);
  w.epoch = 2 * dev_window_slot(fused_epoch) + 1;
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gthreads = gridDim.x * blockDim.x;
  const uint32_t warp = spread_warp(), nwarps = gthreads >> 5;
  uint32_t seq = 0;
  if (f + 1 > kFusedEpochs) {  // grid-uniform: every block read the same counter
    for (size_t i = gtid; i <= sc.gmask; i += gthreads) sc.gtab[i] = 0;
    for (size_t i = gtid; i <= sc.cmask; i += gthreads) sc.ctab[i] = 0;
  }
  phase_list_muts<Tr>(sc, w, warp, nwarps);
  if (!grid_barrier(bar, gridDim.x, t.status, seq)) return;
  phase_probe_list<Tr>(t, sc, w, warp, nwarps, false);
  if (!grid_barrier(bar, gridDim.x, t.status, seq)) return;
  phase_sort_big<Tr>(sc, w, smem);
  if (huge_groups(sc, w.cnt) == 0) return;  // grid-uniform: the probe step has ended
  huge_hist<Tr>(sc, w, gtid >> 5, gthreads >> 5);
  if (!grid_barrier(bar, gridDim.x, t.status, seq)) return;
  huge_scan<Tr>(sc, w, smem);
  if (!grid_barrier(bar, gridDim.x, t.status, seq)) return;
  huge_scatter<Tr>(sc, w, gtid >> 5, gthreads >> 5);
  if (!grid_barrier(bar, gridDim.x, t.status, seq)) return;
  huge_runs<Tr>(sc, w, smem, gtid, gthreads);
}

// Last kernel of a per-phase window: it also leaves the counter block zeroed
// for the next launch.  With fused_epoch (a window on the device epoch), its
// last block also advances the epoch counter.
template <class Tr>
__global__ void __launch_bounds__(1024, 1)
    k_resolve(TableView t, Scratch sc, Window<Tr> w, GridBarrier* bar, uint32_t* fused_epoch) {
  const uint32_t tid = spread_tid(), nt = gridDim.x * blockDim.x;
  const uint32_t slot = fused_epoch != nullptr ? dev_window_slot(fused_epoch) : 0u;
  if (fused_epoch != nullptr) w.epoch = 2 * slot + 1;
  phase_resolve_mutations<Tr>(t, sc, w, tid, nt);
  phase_resolve_reads<Tr>(sc, w, tid, nt);
  release_counters(sc.cnt, bar, nullptr, 0, fused_epoch, slot + 1);
}

// One batch split into windows, all phases of all windows in one cooperative
// launch with bounded grid barriers between phases.
template <class Tr>
struct FusedJob {
  Window<Tr> base;  // whole batch; n = total ops
  uint32_t window;  // ops per window
  uint32_t* fused_epoch;  // device: fused windows run so far (epochs of the fused path)
  uint32_t chunk;   // probe work claim size (0 = static stride)
  uint32_t dedup;
  uint32_t split_q16;  // fraction of reads probed with the mutations (x 65536)
  uint64_t* trace;     // optional: phase-boundary timestamps (ns), block 0 records
  BinCounters* bins;   // two sets, by window parity
  uint32_t binned;     // probe in table-region order
  uint32_t bin_shift;  // bucket index >> bin_shift = region
};

// Phase trace: entry = globaltimer ns << 8 | window & 0x3F << 2 | phase (0 start,
// 1 after probe, 2 after sort, 3 after resolve).  Block 0, thread 0 only.
__device__ __forceinline__ void trace_mark(uint64_t* tr, uint32_t& at, uint32_t wi, uint32_t ph) {
  if (tr == nullptr || blockIdx.x != 0 || threadIdx.x != 0 || at >= kTraceCap) return;
  uint64_t ns;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ns));
  tr[at++] = (ns << 8) | ((uint64_t)(wi & 0x3F) << 2) | ph;
}

// Work for warp 0 of block 0 while the rest of the grid resolves the last
// window (the serving loop admits its next wave there).
struct NoHook {
  static constexpr bool kActive = false;
  __device__ void operator()() const {}
};

// All windows of one batch.  `seq` counts the grid barriers this launch has
// passed (shared with a caller that runs several batches in one launch).
// kList: compile the list-first probe order (fused_split 0); the serving
// loop, whose waves always probe in one pass, leaves it out.
template <class Tr, int P, bool kList = true, class Hook = NoHook>
__device__ void fused_windows(const TableView& t, const Scratch& sc, const FusedJob<Tr>& job,
                              GridBarrier* bar, uint32_t* smem, uint32_t& seq,
                              const Hook& hook = Hook{}) {
  const uint32_t nblocks = gridDim.x;
  // spread indices: small windows use many SMs; tid 0 is still thread 0 of block 0
  const uint32_t tid = spread_tid(), nt = gridDim.x * blockDim.x;
  const uint32_t warp = tid >> 5, nwarps = nt >> 5;
  const uint32_t nwin = (job.base.n + job.window - 1) / job.window;
  uint32_t tat = 0;
  // Window epochs live on the device so that a replayed CUDA graph of this
  // launch never reuses one: the fused path takes odd epochs 2f+1 (f = fused
  // windows so far), the per-phase path even ones from the host.  When the
  // 16-bit epoch would wrap, the grid clears the group and chunk tables first.
  uint32_t f = ld_cg_u32(job.fused_epoch);
  if (f + nwin > kFusedEpochs) {
    for (size_t i = tid; i <= sc.gmask; i += nt) sc.gtab[i] = 0;
    for (size_t i = tid; i <= sc.cmask; i += nt) sc.ctab[i] = 0;
    f = 0;
    if (!grid_barrier(bar, nblocks, t.status, seq)) return;
  }
  for (uint32_t wi = 0; wi < nwin; ++wi) {
    trace_mark(job.trace, tat, wi, 0);
    Window<Tr> w = job.base;
    const uint32_t start = wi * job.window;
    w.n = min(job.window, job.base.n - start);
    if (w.types) w.types += start;
    w.keys += (size_t)start * w.kstride;
    if (w.vals)
      w.vals = reinterpret_cast<const uint64_t*>(reinterpret_cast<const uint8_t*>(w.vals) +
                                                 (size_t)start * w.vstride * (w.v32 ? 4 : 8));
    if (w.out) w.out = (uint8_t*)w.out + (size_t)start * out_bytes(w.out_kind);
    w.epoch = 2 * (f + wi) + 1;
    w.cnt = &sc.cnt[wi & 1];
    // the other counter sets were last read in window wi-1, which has ended
    if (tid == 0) win_counters_reset(&sc.cnt[(wi + 1) & 1]);
    if (tid < 2 * kBins) (&job.bins[(wi + 1) & 1].count[0])[tid] = 0;
    const uint32_t* perm = nullptr;
    // Reads [0, split) are probed with the mutations; reads [split, n) in the
    // sort pass, where they fill the SMs that the (latency-bound, few-block)
    // ordering of big groups leaves idle.  Reads do not depend on the groups.
    const uint32_t split = (uint32_t)(((uint64_t)w.n * job.split_q16) >> 16);
    // ops a block claims at a time for the reads probed beside the mutation
    // list and the ordering pass: the tuned claim size (split 0 has no other
    // use for it), else one tile per warp
    const uint32_t late_chunk = (split == 0 && job.chunk) ? job.chunk : blockDim.x * P;
    // the list-first order's reads through the lean one-op-per-thread lookup
    // (no in-warp dedup, no reader locks, no region order)
    const bool lean_reads = LSB_FUSED_LEAN_READS && !job.dedup && t.lock_mode != kLockRW &&
                            !job.binned;
    if (kList && split == 0) {
      // Mutations listed, then probed from the list; while their (latency-
      // bound) chains run, blocks take reads from the same cursor as the sort
      // pass, until every list tile is done.  Region binning of the reads
      // rides along the two steps.
      phase_list_muts<Tr>(sc, w, warp, nwarps);
      if (job.binned) phase_bin_count<Tr>(t, w, sc.obin, &job.bins[wi & 1], job.bin_shift);
      if (!grid_barrier(bar, nblocks, t.status, seq)) return;
      const uint32_t listed = min(ld_cg_u32(&w.cnt->clist_count), clist_cap(sc.max_window));
      phase_probe_list<Tr>(t, sc, w, warp, nwarps, job.dedup != 0);
      if (job.binned) {
        phase_bin_scatter<Tr>(w, sc.obin, sc.perm, &job.bins[wi & 1]);
        perm = sc.perm;
      } else if (lean_reads) {
        phase_read_lean<Tr, LSB_FUSED_READ_PAIR != 0>(t, w, &w.cnt->late_cursor, 0, w.n,
                                                      &w.cnt->tiles_done, (listed + 31) / 32);
      } else {
        phase_probe<Tr, false, P>(t, sc, w, warp, nwarps, &w.cnt->late_cursor, late_chunk,
                                  job.dedup != 0, ProbeSel{0, w.n, false}, 0, nullptr,
                                  &w.cnt->tiles_done, (listed + 31) / 32);
      }
    } else {
      if (job.binned) {
        phase_bin_count<Tr>(t, w, sc.obin, &job.bins[wi & 1], job.bin_shift);
        if (!grid_barrier(bar, nblocks, t.status, seq)) return;
        phase_bin_scatter<Tr>(w, sc.obin, sc.perm, &job.bins[wi & 1]);
        if (!grid_barrier(bar, nblocks, t.status, seq)) return;
        perm = sc.perm;
      }
      phase_probe<Tr, true, P>(t, sc, w, warp, nwarps, &w.cnt->probe_cursor, job.chunk,
                               job.dedup != 0, ProbeSel{0, split, true}, 0, perm);
    }
    if (!grid_barrier(bar, nblocks, t.status, seq)) return;
    // every block has read the epoch counter (before its first barrier)
    if (wi == 0 && tid == 0) *job.fused_epoch = f + nwin;
    trace_mark(job.trace, tat, wi, 1);
    // counters read after the barrier: the same values in every block, so the
    // skips below are grid-uniform
    const bool has_big = ld_cg_u32(&w.cnt->big_count) != 0;
    const bool has_mut = ld_cg_u32(&w.cnt->mut_count) != 0;
    const bool has_huge = huge_groups(sc, w.cnt) != 0;
    if (has_big || split < w.n) {
      if (has_big) phase_sort_big<Tr>(sc, w, smem);
      if (has_huge) huge_hist<Tr>(sc, w, warp, nwarps);
      if (split < w.n && lean_reads && split == 0 && perm == nullptr)
        phase_read_lean<Tr, LSB_FUSED_READ_PAIR != 0>(t, w, &w.cnt->late_cursor, 0, w.n);
      else if (split < w.n)  // claimed, so blocks freed by the sort take more
        phase_probe<Tr, false, P>(t, sc, w, warp, nwarps, &w.cnt->late_cursor,
                                  late_chunk, job.dedup != 0, ProbeSel{split, w.n, false},
                                  split & ~31u, perm);
      if (!grid_barrier(bar, nblocks, t.status, seq)) return;
    }
    if (has_huge) {
      huge_scan<Tr>(sc, w, smem);
      if (!grid_barrier(bar, nblocks, t.status, seq)) return;
      huge_scatter<Tr>(sc, w, warp, nwarps);
      if (!grid_barrier(bar, nblocks, t.status, seq)) return;
      huge_runs<Tr>(sc, w, smem, tid, nt);
      if (!grid_barrier(bar, nblocks, t.status, seq)) return;
    }
    trace_mark(job.trace, tat, wi, 2);
    // with a hook, warp 0 (threads 0..31 of block 0) runs it during the last
    // window's resolve and takes no resolve work
    const uint32_t r0 = Hook::kActive ? 32u : 0u;
    if (Hook::kActive && wi + 1 == nwin && tid < 32) hook();
    if (has_mut && (!Hook::kActive || tid >= r0)) {
      // Mutations and the reads after the first mutation resolve
      // independently.  A small window (every thread holds at most one item
      // of each kind) runs them side by side on two shares of the grid, so
      // it pays one latency chain instead of two; a large one runs them one
      // after the other on the whole grid (mutations cost more per item).
      const uint32_t rt = tid - r0, rn = nt - r0;
      const uint64_t m = ld_cg_u32(&w.cnt->mut_count);
      const uint32_t first = ~ld_cg_u32(&w.cnt->inv_first_mut);
      const uint64_t r = first < w.n ? w.n - first - 1 : 0;
      const uint32_t ms = (uint32_t)((m + 31) / 32 * 32);
      if (m + r + 32 <= rn) {
        if (rt < ms)
          phase_resolve_mutations<Tr>(t, sc, w, rt, ms);
        else
          phase_resolve_reads<Tr>(sc, w, rt - ms, rn - ms);
      } else {
        phase_resolve_mutations<Tr>(t, sc, w, rt, rn);
        phase_resolve_reads<Tr>(sc, w, rt, rn);
      }
    }
    // Before the next window: its probes must see this window's writes, and
    // its first thread resets this window's counter set, which every block
    // must have finished reading.  The last window needs none (kernel end).
    if (wi + 1 < nwin && !grid_barrier(bar, nblocks, t.status, seq)) return;
    trace_mark(job.trace, tat, wi, 3);
  }
}

#ifdef LSB_FUSED_MAXNREG
#define LSB_FUSED_BOUNDS __maxnreg__(LSB_FUSED_MAXNREG)
#else
#define LSB_FUSED_BOUNDS __launch_bounds__(1024, LSB_FUSED_MIN_BLOCKS)
#endif
template <class Tr, int P>
__global__ void LSB_FUSED_BOUNDS
    k_fused(TableView t, Scratch sc, FusedJob<Tr> job, GridBarrier* bar) {
  extern __shared__ uint32_t smem[];
  uint32_t seq = 0;
  fused_windows<Tr, P>(t, sc, job, bar, smem, seq);
  release_counters(sc.cnt, bar, job.bins, 2 * sizeof(BinCounters) / 4);
}

// ------------------------------------------------------------------ serving
// A device-resident request loop over one map (lsb_serve_*): one persistent
// cooperative launch admits waves of queued requests (continuous batching:
// whatever arrived while the previous wave ran joins the next one), runs each
// wave through the batch engine as one window and publishes completions.
// Requests, their ops and their results sit in GPU-mapped pinned host memory,
// where a KV server's network layer would deliver them; the table, the pool
// and each wave's working copy stay in HBM.  Ops of a wave run in request
// order (FIFO admission), so a wave equals running its requests one after
// another.
struct ServeCtl {     // host-mapped
  uint64_t submitted;  // requests published by the host (monotonic)
  uint64_t completed;  // requests finished by the device (monotonic)
  uint64_t waves;      // waves run
  uint64_t ops;        // ops run
  uint32_t stop;       // host: end the loop once the queue is drained
  uint32_t state;      // device: see lsb_serve_stats.state
  // device: %globaltimer ns summed over waves by one timing thread (block 0,
  // thread 32, which takes part in every step but the admission), rewritten
  // after every wave: gather, engine (probe, ordering, its resolve share),
  // tail (the rest of the resolve, the admission, the last barrier), and the
  // waits for requests when the queue ran empty
  uint64_t t_gather, t_engine, t_tail, t_wait;
};

struct ServeReq {     // one request slot, host-mapped
  uint64_t op_off;     // first op in the arena (monotonic op count; slot = off % arena)
  uint32_t n;          // ops
  uint32_t puts;       // puts among them: the request's worst-case new slabs
  int32_t status;      // device: LSB_OK, or LSB_ERR_OOM when the pool cannot take it
  uint32_t pad;
};

struct WaveDesc {     // device: the wave that thread 0 admitted
  uint64_t first;      // first request of the wave
  uint64_t op_off;     // its first op in the arena
  uint32_t nreq;       // requests completed by this wave
  uint32_t nops;       // ops run (0 when the head request was refused)
  uint32_t stop;       // 1 drained after a stop request, 2 idle limit
  uint32_t puts;       // puts admitted (worst-case new slabs of the wave)
};

struct ServeJob {
  ServeCtl* ctl;
  ServeReq* ring;
  uint64_t ring_cap;
  const uint8_t* a_types;   // host-mapped op arena
  const uint64_t* a_keys;
  const uint64_t* a_vals;
  lsb_result* a_out;
  uint64_t arena_cap;
  uint8_t* d_types;         // HBM working copy of a wave's ops
  uint64_t* d_keys;
  uint64_t* d_vals;
  WaveDesc* wave;           // two descriptors, alternating by admission
  uint32_t max_wave_ops;
  uint32_t pad;
  uint64_t idle_ns;         // a blocking admission waits at most this long (%globaltimer)
  FusedJob<MapTraits> fj;   // engine parameters; base is set per wave
};

__device__ __forceinline__ uint64_t ld_acquire_sys_u64(const uint64_t* p) {
  uint64_t r;
  asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(r) : "l"(p) : "memory");
  return r;
}

__device__ __forceinline__ void st_release_sys_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid barrier behind a blocking admission: it waits until a %globaltimer
// deadline instead of for a number of polls, so its limit is stated in the
// same clock as the admission's wait (the caller passes the admission's
// deadline plus a margin).  Otherwise as grid_barrier.
__device__ bool grid_barrier_until(GridBarrier* b, uint32_t nblocks, uint32_t* status,
                                   uint32_t& seq, uint64_t deadline_ns) {
  __shared__ int ok;
  __syncthreads();
  ++seq;
  if (threadIdx.x == 0) {
    ok = 1;
    const uint32_t target = seq * nblocks;
    if (atom_add_acq_rel(&b->count, 1u) + 1 != target) {
      uint32_t it = 0;
      while ((int32_t)(ld_acquire_u32(&b->count) - target) < 0) {
        if ((*(volatile uint32_t*)status & kStatusBarrier) ||
            ((++it & 255u) == 0 && global_ns() > deadline_ns)) {
          raise_status(status, kStatusBarrier);
          ok = 0;
          break;
        }
        if (it > 256) __nanosleep(256);
      }
    }
  }
  __syncthreads();
  return ok != 0;
}

// Slabs the pool can still hand out: the free stack, what the global cursor
// has left, and what is left in the per-SM ranges (pool_alloc takes those
// before it reports OOM).  Whole warp; the result is warp-uniform.
__device__ uint64_t pool_free_slabs(const TableView& t) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t left = 0;
  for (int k = (int)lane; k < kPoolSlots; k += 32) {
    const uint64_t v = ld_cg_u64(&t.pool[2 + k]);
    const uint32_t cur = (uint32_t)v, end = (uint32_t)(v >> 32);
    left += cur < end ? end - cur : 0u;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) left += __shfl_xor_sync(0xFFFFFFFFu, left, d);
  const uint64_t limit = ld_cg_u64(&t.pool[1]), cursor = ld_cg_u64(&t.pool[0]);
  const long long top = (long long)ld_cg_u64(&t.pool[kPoolTop]);
  return left + (limit > cursor ? limit - cursor : 0) + (top > 0 ? (uint64_t)top : 0);
}

// Warp 0 of block 0: wait (bounded by idle_ns) for requests, then admit the
// longest FIFO prefix that fits the wave's op limit, whose ops are
// contiguous in one lap of the arena (the host never splits a request
// across the arena's end; a request that starts a new lap starts a new
// wave, so a wave's ops never wrap) and whose worst-case new slabs (one per
// put) fit the pool's free slabs.  Lanes read 32 descriptors at a time and
// admit by warp prefix sums.  `blocking`: wait for a request; otherwise an
// empty queue gives an empty wave.  `in_flight_puts`: puts of a wave still
// being applied, whose slabs the pool may not show as taken yet; the budget
// subtracts them in full, so it is a lower bound.  Only an exact budget (no
// wave in flight) refuses a head request that does not fit: it can never
// fit (slabs are not returned), so it completes alone with LSB_ERR_OOM;
// with a wave in flight the admission returns an empty wave instead and the
// loop retries once that wave is done.
__device__ void serve_admit(const TableView& t, const ServeJob& j, WaveDesc* out, uint64_t head,
                            bool blocking, uint64_t in_flight_puts) {
  const uint32_t lane = threadIdx.x & 31;
  WaveDesc wd{};
  wd.first = head;
  uint64_t sub = 0;
  uint32_t stop = 0;
  if (lane == 0) {
    const uint64_t t0 = blocking ? global_ns() : 0;
    for (uint32_t it = 0;; ++it) {
      sub = ld_acquire_sys_u64(&j.ctl->submitted);
      if (sub > head || !blocking) break;
      if (*(volatile uint32_t*)&j.ctl->stop) {
        stop = 1;
        break;
      }
      if (global_ns() - t0 > j.idle_ns) {
        stop = 2;
        break;
      }
      __nanosleep(it < 64 ? 128 : 2048);
    }
  }
  sub = __shfl_sync(0xFFFFFFFFu, sub, 0);
  stop = __shfl_sync(0xFFFFFFFFu, stop, 0);
  if (stop || sub <= head) {  // stop, or nothing queued (non-blocking)
    if (lane == 0) {
      wd.stop = stop;
      *out = wd;
    }
    return;
  }
  const uint64_t free_slabs = pool_free_slabs(t);
  uint64_t budget = free_slabs > in_flight_puts ? free_slabs - in_flight_puts : 0;
  const uint64_t budget0 = budget;
  const uint64_t end = min(sub, head + j.ring_cap);
  uint32_t nops = 0, nreq = 0;
  uint64_t next_off = 0;
  for (uint64_t base = head; base < end; base += 32) {
    const uint64_t r = base + lane;
    const bool valid = r < end;
    volatile ServeReq* q = &j.ring[r % j.ring_cap];
    const uint64_t off = valid ? q->op_off : 0;
    const uint32_t n = valid ? q->n : 0, puts = valid ? q->puts : 0;
    if (base == head) next_off = __shfl_sync(0xFFFFFFFFu, off, 0);
    // inclusive prefix sums of ops and puts over the lanes
    uint64_t cn = n, cp = puts;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t yn = __shfl_up_sync(0xFFFFFFFFu, cn, d);
      const uint64_t yp = __shfl_up_sync(0xFFFFFFFFu, cp, d);
      if (lane >= (uint32_t)d) {
        cn += yn;
        cp += yp;
      }
    }
    // contiguous: this request starts where the previous one ends, and not
    // at the start of a lap (the wave's ops would wrap the arena); the head
    // request of the wave (base == head, lane 0) is always taken as is
    const uint64_t prev_end = __shfl_up_sync(0xFFFFFFFFu, off + n, 1);
    const bool new_lap = off % j.arena_cap == 0 && !(base == head && lane == 0);
    const bool contiguous = (lane == 0 ? off == next_off : off == prev_end) && !new_lap;
    const bool fits = valid && contiguous && nops + cn <= j.max_wave_ops && cp <= budget;
    const uint32_t bad = __ballot_sync(0xFFFFFFFFu, !fits);
    const uint32_t take = bad ? (uint32_t)__ffs(bad) - 1 : 32u;
    if (lane < take) q->status = LSB_OK;
    if (take == 0) {
      // the head request alone does not fit the budget: refuse it only when
      // the budget is exact (no wave in flight); otherwise admit nothing now
      const bool refuse = nreq == 0 && in_flight_puts == 0 &&
                          __shfl_sync(0xFFFFFFFFu, valid && puts > budget, 0);
      if (refuse && lane == 0) {
        q->status = LSB_ERR_OOM;  // refused alone: no op of it runs
        wd.op_off = off;
        wd.nreq = 1;
        wd.nops = 0;
        *out = wd;
      }
      if (refuse) return;
      break;
    }
    if (nreq == 0) wd.op_off = __shfl_sync(0xFFFFFFFFu, off, 0);
    nops += (uint32_t)__shfl_sync(0xFFFFFFFFu, cn, take - 1);
    budget -= __shfl_sync(0xFFFFFFFFu, cp, take - 1);
    next_off = __shfl_sync(0xFFFFFFFFu, off + n, take - 1);
    nreq += take;
    if (take < 32) break;
  }
  if (lane == 0) {
    wd.nreq = nreq;
    wd.nops = nops;
    const uint64_t used = budget0 - budget;
    wd.puts = used > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)used;
    *out = wd;
  }
}

// The serving loop's hook: admit the next wave (non-blocking) while the grid
// resolves the current one.
struct AdmitNext {
  static constexpr bool kActive = true;
  const TableView* t;
  const ServeJob* j;
  WaveDesc* out;
  uint64_t head;
  uint64_t in_flight_puts;
  __device__ void operator()() const { serve_admit(*t, *j, out, head, false, in_flight_puts); }
};

template <int P>
__global__ void __launch_bounds__(1024, 1)
    k_serve(TableView t, Scratch sc, ServeJob j, GridBarrier* bar) {
  extern __shared__ uint32_t smem[];
  // spread indices (tid < 32 is still warp 0 of block 0)
  const uint32_t tid = spread_tid(), nt = gridDim.x * blockDim.x;
  uint32_t seq = 0;
  uint64_t head = 0;  // meaningful in warp 0 of block 0
  uint64_t waves = 0, ops = 0;  // meaningful in thread 0
  if (tid < 32) head = ld_acquire_sys_u64(&j.ctl->completed);
  if (tid == 0) {
    waves = *(volatile uint64_t*)&j.ctl->waves;
    ops = *(volatile uint64_t*)&j.ctl->ops;
  }
  if (tid == 0) *(volatile uint32_t*)&j.ctl->state = 1;
  const bool timer = blockIdx.x == 0 && threadIdx.x == 32;
  uint64_t tg = 0, te = 0, tt = 0, tw = 0;  // the timing thread's sums
  if (timer) {
    tg = *(volatile uint64_t*)&j.ctl->t_gather;
    te = *(volatile uint64_t*)&j.ctl->t_engine;
    tt = *(volatile uint64_t*)&j.ctl->t_tail;
    tw = *(volatile uint64_t*)&j.ctl->t_wait;
  }
  // Wave k+1 is admitted (without waiting) as wave k's last phase ends, so
  // one grid barrier both completes wave k and publishes wave k+1; only an
  // empty queue makes warp 0 wait for requests, after wave k is published.
  // Admission `a` writes descriptor a & 1, which every block finished
  // reading before the barrier of admission a - 1.
  uint32_t a = 0;
  // Barriers behind a blocking admission wait until the admission's own
  // deadline (idle_ns from about now) plus a margin, on the same clock.
  constexpr uint64_t kAdmitMarginNs = 2000000000ull;
  if (tid < 32) serve_admit(t, j, &j.wave[0], head, true, 0);
  if (!grid_barrier_until(bar, gridDim.x, t.status, seq, global_ns() + j.idle_ns + kAdmitMarginNs))
    goto out;
  for (;;) {
    const uint64_t t0 = timer ? global_ns() : 0;
    uint64_t t1 = t0, t2 = t0;
    const WaveDesc* cur = &j.wave[a & 1];
    const uint64_t first = ld_cg_u64(&cur->first), op_off = ld_cg_u64(&cur->op_off);
    const uint32_t nreq = ld_cg_u32(&cur->nreq), nops = ld_cg_u32(&cur->nops);
    const uint32_t stop = ld_cg_u32(&cur->stop), wave_puts = ld_cg_u32(&cur->puts);
    if (stop) {
      if (tid == 0) *(volatile uint32_t*)&j.ctl->state = stop == 1 ? 2 : 3;
      break;
    }
    if (nops && (op_off % j.arena_cap) + nops > j.arena_cap) {
      // cannot happen: admission never lets a wave wrap the arena
      if (tid == 0) raise_status(t.status, kStatusScratch);
      break;  // grid-uniform (every block read the same descriptor)
    }
    if (nops) {
      // the wave's ops (contiguous in one lap of the arena) into HBM; .cv
      // loads because the host rewrites arena slots between waves
      const uint64_t pos = op_off % j.arena_cap;
      // (Gathering the values during the probe instead, by the threads that
      // probe no op, measured no faster per op: the probe's barrier waited
      // for their PCIe loads.)
      gather_u64(j.a_keys + pos, j.d_keys, nops, tid, nt);
      gather_u64(j.a_vals + pos, j.d_vals, nops, tid, nt);
      gather_u8(j.a_types + pos, j.d_types, nops, tid, nt);
      if (!grid_barrier(bar, gridDim.x, t.status, seq)) break;
      if (timer) t1 = global_ns();
      FusedJob<MapTraits> fj = j.fj;
      fj.base.types = j.d_types;
      fj.base.keys = j.d_keys;
      fj.base.vals = j.d_vals;
      fj.base.out = j.a_out + pos;  // results go straight to the host-mapped arena
      fj.base.n = nops;
      // the next wave is admitted by warp 0 while the others resolve this one
      fused_windows<MapTraits, P, false>(
          t, sc, fj, bar, smem, seq,
          AdmitNext{&t, &j, &j.wave[(a + 1) & 1], first + nreq, wave_puts});
      if (timer) t2 = global_ns();
    }
    const uint64_t next = first + nreq;
    ++a;
    if (tid < 32 && nops == 0) serve_admit(t, j, &j.wave[a & 1], next, false, wave_puts);
    if (!grid_barrier(bar, gridDim.x, t.status, seq)) break;
    if (timer) {
      tg += t1 - t0;
      te += t2 - t1;
      tt += global_ns() - t2;
      *(volatile uint64_t*)&j.ctl->t_gather = tg;
      *(volatile uint64_t*)&j.ctl->t_engine = te;
      *(volatile uint64_t*)&j.ctl->t_tail = tt;
    }
    if (tid == 0) {
      win_counters_reset(&sc.cnt[0]);  // the next wave's counters (visible after its barrier)
      __threadfence_system();          // results before the completion count
      ++waves;  // kept in registers: a read of host memory costs a PCIe round trip
      ops += nops;
      *(volatile uint64_t*)&j.ctl->waves = waves;
      *(volatile uint64_t*)&j.ctl->ops = ops;
      st_release_sys_u64(&j.ctl->completed, next);
    }
    if (ld_cg_u32(&j.wave[a & 1].nreq) == 0 && ld_cg_u32(&j.wave[a & 1].stop) == 0) {
      // the queue was empty: wait for requests now that wave k is published
      ++a;
      const uint64_t t3 = timer ? global_ns() : 0;
      if (tid < 32) serve_admit(t, j, &j.wave[a & 1], next, true, 0);
      if (!grid_barrier_until(bar, gridDim.x, t.status, seq,
                              global_ns() + j.idle_ns + kAdmitMarginNs))
        break;
      if (timer) {
        tw += global_ns() - t3;
        *(volatile uint64_t*)&j.ctl->t_wait = tw;
      }
    }
  }
out:
  if (tid == 0 && (*(volatile uint32_t*)t.status & kStatusBarrier))
    *(volatile uint32_t*)&j.ctl->state = 4;
  release_counters(sc.cnt, bar, j.fj.bins, 2 * sizeof(BinCounters) / 4);
}

// Compaction (lsb_*_compact): one thread per bucket; the free-stack top was
// clamped to >= 0 by k_pool_clamp just before.
__global__ void k_pool_clamp(uint64_t* pool) {
  if ((long long)pool[kPoolTop] < 0) pool[kPoolTop] = 0;
}

template <class Tr>
__global__ void __launch_bounds__(256) k_compact(TableView t, uint32_t buckets) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < buckets) compact_bucket<Tr>(t, b);
}

// Live-entry count and dump: one thread per bucket walks the chain.
template <class Tr>
__global__ void k_count(TableView t, uint32_t buckets, unsigned long long* count) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long c = 0;
  if (b < buckets) {
    uint32_t s = b;
    for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
      Meta m = load_meta(slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes));
#pragma unroll
      for (int w = 0; w < 7; ++w) c += __popc(m.tag[w] & 0x80808080u) -
                                       __popc(__vcmpeq4(m.tag[w], 0x80808080u) & 0x80808080u);
      if (m.next == 0) break;
      s = m.next;
    }
  }
  c = __reduce_add_sync(0xFFFFFFFFu, (unsigned)c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

template <class Tr>
__global__ void k_dump(TableView t, uint32_t buckets, typename Tr::Key* keys, uint64_t* vals,
                       unsigned long long* cursor, unsigned long long cap) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= buckets) return;
  uint32_t s = b;
  for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
    const uint8_t* slab = slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes);
    Meta m = load_meta(slab);
    for (int slot = 0; slot < kSlots; ++slot) {
      uint32_t tag = (m.tag[slot >> 2] >> (8 * (slot & 3))) & 0xFFu;
      if (tag <= 0x80u) continue;  // empty, dead or busy
      unsigned long long at = atomicAdd(cursor, 1ull);
      if (at >= cap) continue;
      const uint8_t* sp = slab + kMetaBytes + slot * Tr::kSlotBytes;
      if constexpr (Tr::kHasValue) {
        keys[at] = (typename Tr::Key)ld_cg_u64(sp);
        vals[at] = ld_cg_u64(sp + 8);
      } else {
        keys[at] = (typename Tr::Key)ld_cg_u32(sp);
      }
    }
    if (m.next == 0) break;
    s = m.next;
  }
}

// ------------------------------------------------------------- tables
// Defaults: the best of a sweep on the 2^22-bucket, 95/5 Zipf(0.99) workload
// (block 512; lookahead and in-warp dedup both measured slower there).
struct Tuning {
  uint32_t block = 512;  // threads per block (128..1024)
  uint32_t chunk = 0;    // probe work claim (0 = static stride)
  uint32_t prefetch = 0; // extra lookups in flight per thread (0..2)
  uint32_t dedup = 0;
  uint32_t warp_probe = 0;  // read-only batches through k_read_coop
  uint32_t overlap = 0;     // mixed windows: reads in k_read beside the mutation steps
  uint32_t read_order = 0;  // 1: read calls in table-region order (slower; measured)
};

inline bool tuning_ok(const lsb_tuning& x) {
  return (x.block_threads == 128 || x.block_threads == 256 || x.block_threads == 512 ||
          x.block_threads == 1024) &&
         x.prefetch <= 2 && x.dedup <= 1 && x.chunk % 32 == 0 && x.chunk <= (1u << 20) &&
         x.fused_split <= 100 && x.region_order <= 1 && x.warp_probe <= 1 && x.overlap <= 1 &&
         x.read_order <= 1;
}

template <class Tr>
struct Table {
  int device = 0;
  unsigned log2 = 0;
  uint32_t buckets = 0;
  uint64_t pool_slabs = 0;
  uint32_t lock_mode = kLockWriter;
  uint8_t* slabs = nullptr;
  int32_t* locks = nullptr;
  uint32_t* status = nullptr;
  uint64_t* pool = nullptr;
  uint32_t* free_stack = nullptr;  // slabs returned by compaction (pool_slabs entries)
  GridBarrier* bar = nullptr;
  Scratch sc{};
  uint32_t epoch = 0;  // last epoch handed to a window
  uint32_t chunk = 1;  // per-SM pool refill size
  int num_sms = 0;
  Tuning tune;
  uint32_t split_q16 = 65536;  // every op in one probe pass (fused_split 100)
  uint64_t* trace = nullptr;   // device phase-trace buffer when tracing is on
  BinCounters* bins = nullptr; // inside the counter block (see kCounterBytes)
  uint32_t* fused_epoch = nullptr;  // device counter of fused windows (see k_fused)
  bool binned = false;         // fused path probes in table-region order (measured slower)
  int fused_per_sm[3][4] = {};  // occupancy by (prefetch, block size) once queried
  int resolve_per_sm = 0;       // resident 256-thread k_resolve blocks per SM once queried
  // tuning overlap: the mutation steps of a window run on `side` (highest
  // stream priority, so its blocks take SMs as k_read's blocks retire)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  uint32_t* rhist = nullptr;  // region counts of ordered reads (+ the read count)
  // Tracing of the two-stream form: per window, timing events at its start
  // and after each of its kernels (kSpanPoints points, kSpanWindows windows
  // of the last call), read back by read_trace.
  static constexpr int kSpanPoints = 6;  // start, list, probe, ordering, reads, resolve
  static constexpr int kSpanWindows = 16;
  cudaEvent_t span_ev[kSpanWindows][kSpanPoints] = {};
  int span_windows = 0;  // windows of the last traced two-stream call (0: none)

  TableView view() const {
    TableView v;
    v.slabs = slabs;
    v.locks = locks;
    v.status = status;
    v.pool = pool;
    v.free_stack = free_stack;
    v.mask = buckets - 1;
    v.lock_mode = lock_mode;
    v.chunk = chunk;
    return v;
  }

  void release() {
    void* ptrs[] = {slabs, locks, status, pool, free_stack, sc.gtab, sc.ginl, sc.ctab, sc.cdat,
                    sc.minfo, sc.mloc, sc.pred, sc.goff, sc.seg, sc.mlist, sc.big, sc.large,
                    sc.cnt, sc.obin, sc.perm, sc.clist, sc.hlist, sc.hrec, sc.hbins, sc.hrun, sc.runs,
                    sc.lnu, sc.rnu, trace, fused_epoch, rhist};
    for (void* p : ptrs) cudaFree(p);
    if (side) cudaStreamDestroy(side);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    destroy_spans();
  }

  void destroy_spans() {
    for (auto& w : span_ev)
      for (auto& e : w)
        if (e) {
          cudaEventDestroy(e);
          e = nullptr;
        }
    span_windows = 0;
  }

  // Timing event `point` of two-stream window `wi` on stream `st`, when
  // tracing is on and the stream is not being captured.
  int span_mark(int wi, int point, cudaStream_t st) {
    if (!trace || wi >= kSpanWindows) return LSB_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    LSB_CK(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return LSB_OK;
    cudaEvent_t& e = span_ev[wi][point];
    if (!e) LSB_CK(cudaEventCreate(&e));
    LSB_CK(cudaEventRecord(e, st));
    if (point == 0) span_windows = wi + 1;
    return LSB_OK;
  }

  int init(unsigned log2_buckets, const lsb_options* opt) {
    if (log2_buckets < 1 || log2_buckets > 30) return LSB_ERR_ARG;
    uint32_t window = opt && opt->max_window ? opt->max_window : kDefaultWindow;
    if (window > kMaxWindow || window < 32) return LSB_ERR_ARG;
    if (opt && opt->lock_mode > kLockRW) return LSB_ERR_ARG;
    if (opt && opt->device >= 0) LSB_CK(cudaSetDevice(opt->device));
    LSB_CK(cudaGetDevice(&device));
    LSB_CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    log2 = log2_buckets;
    buckets = 1u << log2_buckets;
    pool_slabs = opt && opt->pool_slabs ? opt->pool_slabs : (uint64_t)buckets / 4 + 4096;
    if ((uint64_t)buckets + pool_slabs >= 0xFFFFFFFFull) return LSB_ERR_ARG;
    lock_mode = opt ? opt->lock_mode : kLockWriter;
    chunk = (uint32_t)std::min<uint64_t>(kPoolChunkMax,
                                         std::max<uint64_t>(1, pool_slabs / (8ull * num_sms)));

    const size_t slab_bytes = ((size_t)buckets + pool_slabs) * Tr::kSlabBytes;
    uint32_t g = 64;
    while (g < 2 * window) g <<= 1;
    uint32_t cg = 64;  // chunk slots: at most window/kChunk full chunks + one per big group
    while (cg < 2 * (window / kChunk + window / (kInline + 1) + 1)) cg <<= 1;
    sc.gmask = g - 1;
    sc.cmask = cg - 1;
    sc.max_window = window;
    sc.hcap = window / (kHugeMin + 1) + 1;
    sc.rcap = window / kRunUnit + sc.hcap;
    bool ok =
        cudaMalloc(&slabs, slab_bytes) == cudaSuccess &&
        cudaMalloc(&locks, sizeof(int32_t) * buckets) == cudaSuccess &&
        cudaMalloc(&status, sizeof(uint32_t)) == cudaSuccess &&
        cudaMalloc(&pool, sizeof(uint64_t) * kPoolWords) == cudaSuccess &&
        cudaMalloc(&free_stack, sizeof(uint32_t) * std::max<uint64_t>(1, pool_slabs)) ==
            cudaSuccess &&
        cudaMalloc(&sc.gtab, sizeof(uint64_t) * g) == cudaSuccess &&
        cudaMalloc(&sc.ginl, sizeof(uint32_t) * kInline * (size_t)g) == cudaSuccess &&
        cudaMalloc(&sc.ctab, sizeof(uint64_t) * cg) == cudaSuccess &&
        cudaMalloc(&sc.cdat, sizeof(uint32_t) * kChunk * (size_t)cg) == cudaSuccess &&
        cudaMalloc(&sc.minfo, sizeof(uint64_t) * window) == cudaSuccess &&
        cudaMalloc(&sc.mloc, sizeof(uint64_t) * window) == cudaSuccess &&
        cudaMalloc(&sc.pred, sizeof(uint32_t) * window) == cudaSuccess &&
        cudaMalloc(&sc.goff, sizeof(uint32_t) * g) == cudaSuccess &&
        cudaMalloc(&sc.seg, sizeof(uint32_t) * window) == cudaSuccess &&
        cudaMalloc(&sc.mlist, sizeof(uint32_t) * window) == cudaSuccess &&
        cudaMalloc(&sc.big, sizeof(uint32_t) * (window / (kInline + 1) + 1)) == cudaSuccess &&
        cudaMalloc(&sc.large, sizeof(uint32_t) * (window / (kWarpSort + 1) + 1)) == cudaSuccess &&
        cudaMalloc(&sc.obin, window) == cudaSuccess &&
        cudaMalloc(&sc.perm, sizeof(uint32_t) * window) == cudaSuccess &&
        cudaMalloc(&sc.clist, sizeof(uint32_t) * clist_cap(window)) == cudaSuccess &&
        cudaMalloc(&sc.hlist, sizeof(uint32_t) * sc.hcap) == cudaSuccess &&
        cudaMalloc(&sc.hrec, sizeof(uint32_t) * 4 * sc.hcap) == cudaSuccess &&
        cudaMalloc(&sc.hbins, sizeof(uint32_t) * kHugeBins * (size_t)sc.hcap) == cudaSuccess &&
        cudaMalloc(&sc.hrun, sizeof(uint32_t) * kHugeBins * (size_t)sc.hcap) == cudaSuccess &&
        cudaMalloc(&sc.runs, sizeof(uint32_t) * 4 * (size_t)sc.rcap) == cudaSuccess &&
        cudaMalloc(&sc.lnu, sizeof(uint32_t) * window) == cudaSuccess &&
        cudaMalloc(&sc.rnu, sizeof(uint32_t) * (size_t)sc.rcap) == cudaSuccess &&
        cudaMalloc(&sc.cnt, kCounterBytes) == cudaSuccess &&
        cudaMalloc(&fused_epoch, sizeof(uint32_t)) == cudaSuccess &&
        cudaMalloc(&rhist, sizeof(uint32_t) * ((window / kBinChunk + 1) * (size_t)kReadRegions + 1)) ==
            cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      return LSB_ERR_OOM;
    }
    sc.status = status;
    LSB_CK(cudaMemset(slabs, 0, slab_bytes));
    LSB_CK(cudaMemset(locks, 0, sizeof(int32_t) * buckets));
    LSB_CK(cudaMemset(status, 0, sizeof(uint32_t)));
    std::vector<uint64_t> p(kPoolWords, 0);
    p[0] = buckets;
    p[1] = (uint64_t)buckets + pool_slabs;
    LSB_CK(cudaMemcpy(pool, p.data(), sizeof(uint64_t) * p.size(), cudaMemcpyHostToDevice));
    LSB_CK(cudaMemset(sc.gtab, 0, sizeof(uint64_t) * g));
    LSB_CK(cudaMemset(sc.ctab, 0, sizeof(uint64_t) * cg));
    LSB_CK(cudaMemset(sc.hbins, 0, sizeof(uint32_t) * kHugeBins * (size_t)sc.hcap));
    LSB_CK(cudaMemset(sc.cnt, 0, kCounterBytes));
    LSB_CK(cudaMemset(fused_epoch, 0, sizeof(uint32_t)));
    bar = reinterpret_cast<GridBarrier*>(sc.cnt + 2);
    bins = reinterpret_cast<BinCounters*>(reinterpret_cast<uint8_t*>(sc.cnt) + kBinsOffset);
    LSB_CK(cudaFuncSetAttribute(k_sort<Tr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSortSmemBytes));
    LSB_CK(cudaFuncSetAttribute(k_mutations<Tr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSortSmemBytes));
    LSB_CK(cudaFuncSetAttribute(k_fused<Tr, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSortSmemBytes));
    LSB_CK(cudaFuncSetAttribute(k_fused<Tr, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSortSmemBytes));
    LSB_CK(cudaFuncSetAttribute(k_fused<Tr, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSortSmemBytes));
    int least = 0, greatest = 0;
    LSB_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    LSB_CK(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, greatest));
    LSB_CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    LSB_CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    return LSB_OK;
  }

  int set_tuning(const lsb_tuning& x) {
    if (!tuning_ok(x)) return LSB_ERR_ARG;
    tune.block = x.block_threads;
    tune.chunk = x.chunk;
    tune.prefetch = x.prefetch;
    tune.dedup = x.dedup;
    tune.warp_probe = x.warp_probe;
    tune.overlap = x.overlap;
    tune.read_order = x.read_order;
    split_q16 = (uint32_t)(((uint64_t)x.fused_split << 16) / 100);
    binned = x.region_order != 0;
    return LSB_OK;
  }

  void get_tuning(lsb_tuning* x) const {
    x->block_threads = tune.block;
    x->chunk = tune.chunk;
    x->prefetch = tune.prefetch;
    x->dedup = tune.dedup;
    x->fused_split = (uint32_t)(((uint64_t)split_q16 * 100 + 32768) >> 16);
    x->region_order = binned ? 1u : 0u;
    x->warp_probe = tune.warp_probe;
    x->overlap = tune.overlap;
    x->read_order = tune.read_order;
  }

  // Epoch of the next per-phase window (even: 2, 4, ...; the fused path uses
  // odd ones on the device); clears the group and chunk tables when they wrap.
  int next_plain_epoch(cudaStream_t s, uint32_t* e) {
    if (epoch + 1 > kPlainEpochs) {
      LSB_CK(cudaMemsetAsync(sc.gtab, 0, sizeof(uint64_t) * (sc.gmask + 1ull), s));
      LSB_CK(cudaMemsetAsync(sc.ctab, 0, sizeof(uint64_t) * (sc.cmask + 1ull), s));
      epoch = 0;
    }
    epoch += 1;
    *e = 2 * epoch;
    return LSB_OK;
  }

  Window<Tr> window(const uint8_t* types, uint8_t uniform, const typename Tr::Key* keys,
                    uint32_t kstride, const uint64_t* vals, uint32_t vstride, void* out,
                    uint32_t out_kind, uint32_t n, bool v32 = false) const {
    Window<Tr> w;
    w.v32 = v32 ? 1 : 0;
    w.types = types;
    w.uniform = uniform;
    w.keys = keys;
    w.kstride = kstride;
    w.vals = vals;
    w.vstride = vstride;
    w.out = out;
    w.out_kind = out ? out_kind : kOutNone;
    w.n = n;
    w.epoch = 0;
    w.cnt = sc.cnt;
    return w;
  }

  static size_t out_elem(uint32_t kind) { return out_bytes(kind); }

  int grid_for(uint32_t n) const {
    const int per_sm = 2048 / (int)tune.block;
    const uint32_t need = (n + tune.block * (tune.prefetch + 1) - 1) / (tune.block * (tune.prefetch + 1));
    return std::max(1, std::min<int>(per_sm * num_sms, (int)need));
  }

  template <bool kGroup>
  void launch_probe(int grid, const Window<Tr>& w, cudaStream_t s) {
    const TableView tv = view();
    switch (tune.prefetch) {
      case 0: k_probe<Tr, kGroup, 1><<<grid, tune.block, 0, s>>>(tv, sc, w, tune.chunk, tune.dedup); break;
      case 1: k_probe<Tr, kGroup, 2><<<grid, tune.block, 0, s>>>(tv, sc, w, tune.chunk, tune.dedup); break;
      default: k_probe<Tr, kGroup, 3><<<grid, tune.block, 0, s>>>(tv, sc, w, tune.chunk, tune.dedup); break;
    }
  }

  // Read-only batch: the lean read kernel (k_read), or, with in-warp dedup
  // or reader locks, the tuned probe kernel (one launch per 2^23 ops, no
  // grouping).
  // Whether a read call takes its reads in table-region order.
  bool ordered_reads(size_t) const { return tune.read_order == 1; }

  // The reads among ops [0, m) (all of them without types) in table-region
  // order: count, offsets, order, then the lookups (m <= the window size).
  int launch_read_ordered(const uint8_t* types, const typename Tr::Key* keys, void* out,
                          uint32_t out_kind, uint32_t m, cudaStream_t s) {
    if (m == 0) return LSB_OK;
    if (m > sc.max_window) return LSB_ERR_ARG;
    const uint32_t shift = log2 > 6 ? log2 - 6 : 0u;
    const uint32_t nb = (m + kBinChunk - 1) / kBinChunk;
    k_bin_count<Tr><<<nb, 256, 0, s>>>(view(), types, keys, m, shift, rhist);
    k_bin_scan<<<1, 1024, 0, s>>>(rhist, nb * kReadRegions);
    k_bin_scatter<Tr><<<nb, 256, 0, s>>>(view(), types, keys, m, shift, rhist, sc.perm);
    k_read_ordered<Tr><<<(m + 255) / 256, 256, 0, s>>>(view(), sc.perm, rhist + nb * kReadRegions,
                                                       keys, out, out_kind, m);
    LSB_CK(cudaGetLastError());
    return LSB_OK;
  }

  int run_reads(const typename Tr::Key* keys, void* out, uint32_t out_kind, size_t n,
                cudaStream_t s) {
    if (!tune.dedup && lock_mode != kLockRW && !tune.warp_probe && ordered_reads(n)) {
      for (size_t off = 0; off < n; off += sc.max_window) {
        const uint32_t m = (uint32_t)std::min<size_t>(sc.max_window, n - off);
        void* o = out ? (uint8_t*)out + off * out_elem(out_kind) : nullptr;
        int e = launch_read_ordered(nullptr, keys + off, o, out ? out_kind : kOutNone, m, s);
        if (e) return e;
      }
      return LSB_OK;
    }
    if (!tune.dedup && lock_mode != kLockRW) {
      for (size_t off = 0; off < n; off += (size_t)1 << 30) {
        const uint32_t m = (uint32_t)std::min<size_t>((size_t)1 << 30, n - off);
        void* o = out ? (uint8_t*)out + off * out_elem(out_kind) : nullptr;
        if (tune.warp_probe)
          k_read_coop<Tr><<<(m + 255) / 256, 256, 0, s>>>(view(), keys + off, o,
                                                          out ? out_kind : kOutNone, m);
        else
          k_read<Tr><<<(m + 255) / 256, 256, 0, s>>>(view(), nullptr, keys + off, o,
                                                     out ? out_kind : kOutNone, m);
        LSB_CK(cudaGetLastError());
      }
      return LSB_OK;
    }
    for (size_t off = 0; off < n; off += (size_t)kMaxWindow) {
      uint32_t m = (uint32_t)std::min<size_t>(kMaxWindow, n - off);
      Window<Tr> w = window(nullptr, kOpRead, keys + off, 1, nullptr, 1,
                            out ? (uint8_t*)out + off * out_elem(out_kind) : nullptr, out_kind, m);
      w.cnt = &sc.cnt[0];
      launch_probe<false>(grid_for(m), w, s);
      // the probe's claim cursor is the only counter it uses: clear it again
      if (tune.chunk) LSB_CK(cudaMemsetAsync(w.cnt, 0, sizeof(WinCounters), s));
      LSB_CK(cudaGetLastError());
    }
    return LSB_OK;
  }

  // General batch as per-phase launches, window by window: probe, sort of
  // big groups, resolve.
  // vals: u64 values, or u32 ones when v32 (vstride counts elements of that width).
  int run_plain(const uint8_t* types, uint8_t uniform, const typename Tr::Key* keys,
                uint32_t kstride, const uint64_t* vals, uint32_t vstride, void* out,
                uint32_t out_kind, size_t n, cudaStream_t s, bool v32 = false) {
    const uint32_t W = sc.max_window;
    for (size_t off = 0; off < n; off += W) {
      uint32_t m = (uint32_t)std::min<size_t>(W, n - off);
      const uint64_t* v =
          !vals ? nullptr
          : v32 ? reinterpret_cast<const uint64_t*>(reinterpret_cast<const uint32_t*>(vals) +
                                                    off * vstride)
                : vals + off * vstride;
      Window<Tr> w = window(types ? types + off : nullptr, uniform, keys + off * kstride, kstride,
                            v, vstride, out ? (uint8_t*)out + off * out_elem(out_kind) : nullptr,
                            out_kind, m, v32);
      const bool overlap = types != nullptr && tune.overlap && !tune.dedup &&
                           lock_mode != kLockRW && kstride == 1 && out_kind != kOutOld &&
                           out_kind != kOutOld32;
      if (!overlap) {
        int e = next_plain_epoch(s, &w.epoch);
        if (e) return e;
      }
      w.cnt = &sc.cnt[0];
      // the counters and the sort launch's grid barrier are zero here: the
      // previous launch's last block cleared them (release_counters)
      uint32_t* dev_epoch = overlap ? fused_epoch : nullptr;
      const int wi = (int)(off / W);
      if (overlap && off == 0) span_windows = 0;
      if (overlap) {
        if (int e2 = span_mark(wi, 0, s)) return e2;
        // Reads write their results at probe time and never join a group;
        // only reads after a same-key mutation are rewritten by the resolve
        // step, which is also the only step that writes the table.  So the
        // window's reads go through k_read on `s` while the mutation steps
        // run in k_mutations on `side` (launched first: its one block per SM
        // is resident before k_read fills the SMs); the resolve step waits
        // for both.
        LSB_CK(cudaEventRecord(ev_fork, s));
        LSB_CK(cudaStreamWaitEvent(side, ev_fork, 0));
        if (LSB_OVERLAP_SPLIT) {
          const uint32_t spans = (m + kListSpan - 1) / kListSpan;  // a warp per 512-op span
          k_list_muts<Tr><<<std::max(1u, std::min<uint32_t>((spans + 7) / 8, num_sms * 8)), 256,
                            0, side>>>(sc, w, fused_epoch);
          if (int e2 = span_mark(wi, 1, side)) return e2;
          k_probe_list<Tr><<<num_sms * 2, 256, 0, side>>>(view(), sc, w, fused_epoch);
          if (int e2 = span_mark(wi, 2, side)) return e2;
          if (int e2 = launch_sort(w, side, fused_epoch)) return e2;
        } else {
          TableView tv = view();
          GridBarrier* b = bar;
          uint32_t* fe = fused_epoch;
          void* args[] = {&tv, &sc, &w, &b, &fe};
          cudaLaunchConfig_t cfg = {};
          cfg.gridDim = dim3(num_sms);
          cfg.blockDim = dim3(256);
          cfg.dynamicSmemBytes = kSortSmemBytes;
          cfg.stream = side;
          cudaLaunchAttribute attr[1];
          attr[0].id = cudaLaunchAttributeCooperative;
          attr[0].val.cooperative = 1;
          cfg.attrs = attr;
          cfg.numAttrs = 1;
          LSB_CK(cudaLaunchKernelExC(&cfg, (const void*)k_mutations<Tr>, args));
        }
        if (int e2 = span_mark(wi, 3, side)) return e2;
        LSB_CK(cudaEventRecord(ev_join, side));
        if (ordered_reads(m)) {
          if (int e2 = launch_read_ordered(w.types, w.keys, w.out, w.out_kind, m, s)) return e2;
        } else {
          const uint32_t rblocks = LSB_OVERLAP_READ_BLOCKS
                                       ? std::min<uint32_t>((m + 255) / 256,
                                                            num_sms * LSB_OVERLAP_READ_BLOCKS)
                                       : (m + 255) / 256;
          k_read<Tr><<<std::max(1u, rblocks), 256, 0, s>>>(view(), w.types, w.keys, w.out,
                                                            w.out_kind, m);
        }
        if (int e2 = span_mark(wi, 4, s)) return e2;
        LSB_CK(cudaStreamWaitEvent(s, ev_join, 0));
      } else {
        launch_probe<true>(grid_for(m), w, s);
        if (int e2 = launch_sort(w, s, nullptr)) return e2;
      }
      // One wave of blocks at most: the step's work is the window's
      // mutations (and the reads after its first one), walked by a grid
      // stride, and a second wave would run the same dependent chain again
      // after the first (20 against 10 us for the 52k puts of a 2^20-op
      // 95/5 window with a grid of one thread per op).
      if (resolve_per_sm == 0 &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resolve_per_sm, k_resolve<Tr>, 256, 0) !=
              cudaSuccess)
        resolve_per_sm = 4;
      const int rgrid =
          std::max(1, std::min<int>(num_sms * std::max(1, resolve_per_sm), (int)((m + 255) / 256)));
      k_resolve<Tr><<<rgrid, 256, 0, s>>>(view(), sc, w, bar, dev_epoch);
      LSB_CK(cudaGetLastError());
      if (overlap)
        if (int e2 = span_mark(wi, 5, s)) return e2;
    }
    return LSB_OK;
  }

  // Ordering of the window's big groups (k_sort, a cooperative launch: its
  // hot-key steps have grid barriers).
  int launch_sort(Window<Tr> w, cudaStream_t s, const uint32_t* dev_epoch) {
    GridBarrier* b = bar;
    void* args[] = {&sc, &w, &b, &dev_epoch};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(num_sms);
    cfg.blockDim = dim3(LSB_SORT_THREADS);
    cfg.dynamicSmemBytes = kSortSmemBytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    LSB_CK(cudaLaunchKernelExC(&cfg, (const void*)k_sort<Tr>, args));
    return LSB_OK;
  }

  int fused_grid() {
    const int pi = (int)tune.prefetch;
    const int bi = tune.block == 128 ? 0 : tune.block == 256 ? 1 : tune.block == 512 ? 2 : 3;
    int& per_sm = fused_per_sm[pi][bi];
    if (per_sm == 0) {
      const void* f = pi == 0 ? (const void*)k_fused<Tr, 1>
                    : pi == 1 ? (const void*)k_fused<Tr, 2> : (const void*)k_fused<Tr, 3>;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, (int)tune.block,
                                                        kSortSmemBytes) != cudaSuccess)
        per_sm = -1;
    }
    return per_sm > 0 ? per_sm * num_sms : 0;
  }

  int run_fused(const uint8_t* types, uint8_t uniform, const typename Tr::Key* keys,
                const uint64_t* vals, void* out, uint32_t out_kind, size_t n, cudaStream_t s) {
    if (n == 0) return LSB_OK;
    if (n > 0xFFFFFFFFull) return LSB_ERR_ARG;
    // windows as launches on two streams (reads beside the mutation steps)
    if (tune.overlap && types != nullptr && !tune.dedup && lock_mode != kLockRW)
      return run_plain(types, uniform, keys, 1, vals, 1, out, out_kind, n, s);
    span_windows = 0;  // read_trace reports this launch's phase stamps
    FusedJob<Tr> job;
    job.base = window(types, uniform, keys, 1, vals, 1, out, out_kind, (uint32_t)n);
    job.window = sc.max_window;
    job.chunk = tune.chunk;
    job.dedup = tune.dedup;
    job.split_q16 = split_q16;
    job.trace = trace;
    job.bins = bins;
    job.binned = binned ? 1u : 0u;
    job.bin_shift = log2 > kBinBits ? log2 - kBinBits : 0u;
    if (trace) LSB_CK(cudaMemsetAsync(trace, 0, sizeof(uint64_t) * kTraceCap, s));
    uint32_t nwin = (uint32_t)((n + job.window - 1) / job.window);
    if (nwin > kFusedEpochs / 2) return LSB_ERR_ARG;
    const int grid = fused_grid();
    if (grid <= 0) return LSB_ERR_STATE;
    job.fused_epoch = fused_epoch;
    // counters of both windows, the barrier and the region counters are zero
    // here: the previous launch's last block cleared them (release_counters)
    TableView tv = view();
    Scratch scv = sc;
    GridBarrier* b = bar;
    void* args[] = {&tv, &scv, &job, &b};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(tune.block);
    cfg.dynamicSmemBytes = kSortSmemBytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const void* f = tune.prefetch == 0 ? (const void*)k_fused<Tr, 1>
                  : tune.prefetch == 1 ? (const void*)k_fused<Tr, 2> : (const void*)k_fused<Tr, 3>;
    LSB_CK(cudaLaunchKernelExC(&cfg, f, args));
    return LSB_OK;
  }

  int set_trace(int on) {
    if (on && !trace) {
      if (cudaMalloc(&trace, sizeof(uint64_t) * kTraceCap) != cudaSuccess) return LSB_ERR_OOM;
      LSB_CK(cudaMemset(trace, 0, sizeof(uint64_t) * kTraceCap));
    } else if (!on && trace) {
      cudaFree(trace);
      trace = nullptr;
    }
    return LSB_OK;
  }

  int read_trace(uint64_t* out, size_t cap, size_t* count, cudaStream_t s) {
    if (!trace) return LSB_ERR_STATE;
    std::vector<uint64_t> h(kTraceCap);
    LSB_CK(cudaStreamSynchronize(s));
    if (span_windows > 0) {
      // the last call ran two-stream windows: entries from their events,
      // ns counted from the first window's start (+1 us, so none is zero)
      LSB_CK(cudaStreamSynchronize(side));
      static const uint32_t kPhase[kSpanPoints] = {0, 1, 2, 2, 1, 3};
      static const uint32_t kSub[kSpanPoints] = {0, 0x20, 0x20, 0, 0, 0};
      size_t n = 0;
      for (int wi = 0; wi < span_windows; ++wi)
        for (int p = 0; p < kSpanPoints; ++p) {
          if (!span_ev[wi][p]) continue;
          float ms = 0.f;
          LSB_CK(cudaEventElapsedTime(&ms, span_ev[0][0], span_ev[wi][p]));
          const uint64_t ns = 1000ull + (uint64_t)(ms * 1e6f);
          const uint64_t e =
              (ns << 8) | ((uint64_t)(((uint32_t)wi & 0x1Fu) | kSub[p]) << 2) | kPhase[p];
          if (n < cap) out[n] = e;
          ++n;
        }
      if (count) *count = n;
      return LSB_OK;
    }
    LSB_CK(cudaMemcpy(h.data(), trace, sizeof(uint64_t) * kTraceCap, cudaMemcpyDeviceToHost));
    size_t n = 0;
    while (n < kTraceCap && h[n] != 0) ++n;
    for (size_t i = 0; i < n && i < cap; ++i) out[i] = h[i];
    if (count) *count = n;
    return LSB_OK;
  }

  int read_status(uint32_t* flags, cudaStream_t s) {
    uint32_t v = 0;
    LSB_CK(cudaStreamSynchronize(s));
    LSB_CK(cudaMemcpy(&v, status, sizeof(v), cudaMemcpyDeviceToHost));
    LSB_CK(cudaMemset(status, 0, sizeof(uint32_t)));
    if (flags) *flags = v;
    return LSB_OK;
  }

  // Slabs out of the pool: handed out by the bump allocator (those parked in
  // per-SM ranges included) minus those back on the free stack.
  int pool_usage(uint64_t* used, uint64_t* cap, cudaStream_t s) {
    uint64_t p[2], top = 0;
    LSB_CK(cudaStreamSynchronize(s));
    LSB_CK(cudaMemcpy(p, pool, sizeof(p), cudaMemcpyDeviceToHost));
    LSB_CK(cudaMemcpy(&top, pool + kPoolTop, sizeof(top), cudaMemcpyDeviceToHost));
    const uint64_t on_stack = (long long)top > 0 ? top : 0;
    const uint64_t u = std::min(p[0], p[1]) - buckets - on_stack;
    if (used) *used = u;
    if (cap) *cap = pool_slabs;
    return LSB_OK;
  }

  // Compaction of every chain (see compact_bucket); *freed = slabs returned.
  int compact(uint64_t* freed, cudaStream_t s) {
    uint64_t before = 0, after = 0;
    k_pool_clamp<<<1, 1, 0, s>>>(pool);
    if (freed) LSB_CK(cudaMemcpyAsync(&before, pool + kPoolTop, 8, cudaMemcpyDeviceToHost, s));
    k_compact<Tr><<<(buckets + 255) / 256, 256, 0, s>>>(view(), buckets);
    LSB_CK(cudaGetLastError());
    if (freed) {
      LSB_CK(cudaMemcpyAsync(&after, pool + kPoolTop, 8, cudaMemcpyDeviceToHost, s));
      LSB_CK(cudaStreamSynchronize(s));
      *freed = after - before;
    }
    return LSB_OK;
  }

  int size(uint64_t* count, cudaStream_t s) {
    unsigned long long* d = nullptr;
    LSB_CK(cudaMalloc(&d, sizeof(*d)));
    cudaMemsetAsync(d, 0, sizeof(*d), s);
    k_count<Tr><<<(buckets + 255) / 256, 256, 0, s>>>(view(), buckets, d);
    unsigned long long h = 0;
    cudaError_t e1 = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e1 != cudaSuccess || e2 != cudaSuccess) return LSB_ERR_CUDA;
    *count = h;
    return LSB_OK;
  }

  // Live entries sorted by key, copied to host arrays.
  int dump(typename Tr::Key* keys_out, uint64_t* vals_out, size_t cap, uint64_t* count,
           cudaStream_t s) {
    uint64_t n = 0;
    int e = size(&n, s);
    if (e) return e;
    if (count) *count = n;
    if (n == 0 || cap == 0) return LSB_OK;
    typename Tr::Key* dk = nullptr;
    uint64_t* dv = nullptr;
    unsigned long long* cur = nullptr;
    if (cudaMalloc(&dk, sizeof(*dk) * n) != cudaSuccess ||
        (Tr::kHasValue && cudaMalloc(&dv, sizeof(uint64_t) * n) != cudaSuccess) ||
        cudaMalloc(&cur, sizeof(*cur)) != cudaSuccess) {
      cudaFree(dk);
      cudaFree(dv);
      cudaFree(cur);
      return LSB_ERR_OOM;
    }
    cudaMemsetAsync(cur, 0, sizeof(*cur), s);
    k_dump<Tr><<<(buckets + 255) / 256, 256, 0, s>>>(view(), buckets, dk, dv, cur, n);
    std::vector<typename Tr::Key> hk(n);
    std::vector<uint64_t> hv(Tr::kHasValue ? n : 0);
    cudaMemcpyAsync(hk.data(), dk, sizeof(*dk) * n, cudaMemcpyDeviceToHost, s);
    if (Tr::kHasValue) cudaMemcpyAsync(hv.data(), dv, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, s);
    cudaError_t err = cudaStreamSynchronize(s);
    cudaFree(dk);
    cudaFree(dv);
    cudaFree(cur);
    if (err != cudaSuccess) return LSB_ERR_CUDA;
    std::vector<size_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return hk[a] < hk[b]; });
    size_t w = std::min<size_t>(cap, n);
    for (size_t i = 0; i < w; ++i) {
      keys_out[i] = hk[idx[i]];
      if (Tr::kHasValue && vals_out) vals_out[i] = hv[idx[i]];
    }
    return LSB_OK;
  }
};

}  // namespace

// Tuned launch shapes by (container, log2 buckets), filled by the autotuner;
// a table created later with the same shape starts from them.
static std::mutex g_tune_mu;
static std::map<std::pair<int, unsigned>, lsb_tuning> g_tuned;

static bool tuned_lookup(int kind, unsigned log2, lsb_tuning* out) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tuned.find({kind, log2});
  if (it == g_tuned.end()) return false;
  *out = it->second;
  return true;
}

static void tuned_store(int kind, unsigned log2, const lsb_tuning& t) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tuned[{kind, log2}] = t;
}

// Sweep of the fused path's launch shape on a sample batch (see lsb.h).
template <class Tr>
int autotune(Table<Tr>& tb, int kind, const uint8_t* types, const typename Tr::Key* keys,
             const uint64_t* vals, void* out, uint32_t out_kind, size_t n, cudaStream_t s,
             lsb_tuning* best) {
  lsb_tuning cur;
  tb.get_tuning(&cur);
  cudaEvent_t e0, e1;
  LSB_CK(cudaEventCreate(&e0));
  LSB_CK(cudaEventCreate(&e1));
  float best_ms = 1e30f;
  lsb_tuning win = cur;
  int err = LSB_OK;
  // 4, 8, 16 and 32 warps a block; lookahead 0..2; the list-first order
  // (its reads claim whole blocks of ops; with in-warp dedup the claim size
  // is tuned below), or one pass with the probe's claim size static or
  // 32..4096 ops.  Each candidate: one warm-up run, then the median of three.
  static const uint32_t kChunks[] = {0u, 32u, 128u, 512u, 1024u, 2048u, 4096u};
  constexpr int kReps = 3;
  for (uint32_t block : {128u, 256u, 512u, 1024u}) {
    for (uint32_t prefetch : {0u, 1u, 2u}) {
      for (uint32_t cand = 0; cand < 1 + sizeof(kChunks) / sizeof(kChunks[0]); ++cand) {
        lsb_tuning c = cur;
        c.overlap = 0;
        c.block_threads = block;
        c.prefetch = prefetch;
        c.fused_split = cand == 0 ? 0u : 100u;
        c.chunk = cand == 0 ? (cur.dedup ? 2048u : 0u) : kChunks[cand - 1];
        if (tb.set_tuning(c) != LSB_OK) continue;
        if (tb.fused_grid() <= 0) continue;  // shape cannot be co-resident
        err = tb.run_fused(types, kOpRead, keys, vals, out, out_kind, n, s);  // warm-up
        if (err) break;
        float t[kReps];
        for (int r = 0; r < kReps && !err; ++r) {
          cudaEventRecord(e0, s);
          err = tb.run_fused(types, kOpRead, keys, vals, out, out_kind, n, s);
          cudaEventRecord(e1, s);
          if (!err && cudaEventSynchronize(e1) != cudaSuccess) err = LSB_ERR_CUDA;
          if (!err) cudaEventElapsedTime(&t[r], e0, e1);
        }
        if (err) break;
        std::sort(t, t + kReps);
        if (t[kReps / 2] < best_ms) {
          best_ms = t[kReps / 2];
          win = c;
        }
      }
      if (err) break;
    }
    if (err) break;
  }
  // the best shape with the two-stream window form (it uses the persistent
  // kernel's shape only where the form does not apply)
  if (!err && !cur.dedup && tb.lock_mode != kLockRW) {
    lsb_tuning c = win;
    c.overlap = 1;
    if (tb.set_tuning(c) == LSB_OK) {
      err = tb.run_fused(types, kOpRead, keys, vals, out, out_kind, n, s);  // warm-up
      float t[kReps];
      for (int r = 0; r < kReps && !err; ++r) {
        cudaEventRecord(e0, s);
        err = tb.run_fused(types, kOpRead, keys, vals, out, out_kind, n, s);
        cudaEventRecord(e1, s);
        if (!err && cudaEventSynchronize(e1) != cudaSuccess) err = LSB_ERR_CUDA;
        if (!err) cudaEventElapsedTime(&t[r], e0, e1);
      }
      if (!err) {
        std::sort(t, t + kReps);
        if (t[kReps / 2] < best_ms) {
          best_ms = t[kReps / 2];
          win = c;
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  tb.set_tuning(err ? cur : win);
  if (err) return err;
  tuned_store(kind, tb.log2, win);
  if (best) *best = win;
  return LSB_OK;
}

// A captured fused launch.
struct lsb_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

template <class Tr>
int capture_fused(Table<Tr>& tb, const uint8_t* types, const typename Tr::Key* keys,
                  const uint64_t* vals, void* out, uint32_t out_kind, size_t n,
                  lsb_graph** result) {
  cudaStream_t cs;
  LSB_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  lsb_graph* g = new (std::nothrow) lsb_graph();
  if (!g) {
    cudaStreamDestroy(cs);
    return LSB_ERR_OOM;
  }
  int err = LSB_OK;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    err = LSB_ERR_CUDA;
  } else {
    err = tb.run_fused(types, kOpRead, keys, vals, out, out_kind, n, cs);
    cudaGraph_t graph = nullptr;
    if (cudaStreamEndCapture(cs, &graph) != cudaSuccess || graph == nullptr) {
      if (!err) err = LSB_ERR_CUDA;
    } else {
      g->graph = graph;
      if (!err && cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) err = LSB_ERR_CUDA;
    }
  }
  cudaStreamDestroy(cs);
  if (err) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    cudaGetLastError();
    return err;
  }
  *result = g;
  return LSB_OK;
}

struct lsb_map {
  Table<MapTraits> t;
};
struct lsb_set {
  Table<SetTraits> t;
};

// Internal accessor for other translation units of the library (see
// lsb_internal.h): the device view and bucket count of a map.
void lsb_internal_map_view(const lsb_map* m, lsb::TableView* view, uint32_t* buckets) {
  *view = m->t.view();
  *buckets = m->t.buckets;
}

int lsb_internal_map_device(const lsb_map* m) { return m->t.device; }
uint32_t lsb_internal_lock_mode_map(const lsb_map* m) { return m->t.lock_mode; }
uint32_t lsb_internal_lock_mode_set(const lsb_set* s) { return s->t.lock_mode; }

// ------------------------------------------------------------------ serving
// Host side of the request loop (see k_serve).  One producer may submit while
// another thread takes results; both advance FIFO cursors.
struct lsb_server {
  lsb_map* map = nullptr;
  int device = 0;
  ServeCtl* ctl = nullptr;    // host pointers (pinned, mapped)
  ServeReq* ring = nullptr;
  uint8_t* a_types = nullptr;
  uint64_t* a_keys = nullptr;
  uint64_t* a_vals = nullptr;
  lsb_result* a_out = nullptr;
  uint64_t ring_cap = 0, arena_cap = 0;
  uint32_t max_wave_ops = 0;
  uint64_t idle_ns = 0;
  uint8_t* d_types = nullptr;  // HBM working copy of a wave
  uint64_t* d_keys = nullptr;
  uint64_t* d_vals = nullptr;
  WaveDesc* d_wave = nullptr;
  cudaStream_t stream = nullptr;
  bool running = false;
  std::mutex submit_mu;
  uint64_t next_req = 0, next_op = 0;         // producer cursors
  std::atomic<uint64_t> freed_req{0}, freed_op{0};  // taken (reclaimable) prefix
  std::vector<uint8_t> taken;                  // per ring slot: results taken
  std::mutex take_mu;

  void release() {
    cudaFreeHost(ctl);
    cudaFreeHost(ring);
    cudaFreeHost(a_types);
    cudaFreeHost(a_keys);
    cudaFreeHost(a_vals);
    cudaFreeHost(a_out);
    cudaFree(d_types);
    cudaFree(d_keys);
    cudaFree(d_vals);
    cudaFree(d_wave);
  }
};

namespace {
template <class T>
T* dev_ptr(T* host) {
  void* d = nullptr;
  return cudaHostGetDevicePointer(&d, host, 0) == cudaSuccess ? static_cast<T*>(d) : nullptr;
}
}  // namespace

// Device view of a table for the per-warp device API (lsb_*_device_view).
namespace {
template <class Tr>
void fill_view(const Table<Tr>& t, lsb_table_view* out) {
  const TableView v = t.view();
  out->slabs = v.slabs;
  out->locks = v.locks;
  out->status = v.status;
  out->pool = v.pool;
  out->free_stack = v.free_stack;
  out->mask = v.mask;
  out->lock_mode = v.lock_mode;
  out->chunk = v.chunk;
  out->pad = 0;
}
}  // namespace

extern "C" {

// ------------------------------------------------------------------ map
int lsb_map_create_ex(unsigned log2_buckets, const lsb_options* opt, lsb_map** out) {
  if (!out) return LSB_ERR_ARG;
  *out = nullptr;
  lsb_map* m = new (std::nothrow) lsb_map();
  if (!m) return LSB_ERR_OOM;
  int e = m->t.init(log2_buckets, opt);
  if (e) {
    m->t.release();
    delete m;
    return e;
  }
  lsb_tuning cached;
  if (tuned_lookup(0, log2_buckets, &cached)) m->t.set_tuning(cached);
  *out = m;
  return LSB_OK;
}

int lsb_map_create(unsigned log2_buckets, uint64_t pool_slabs, lsb_map** out) {
  lsb_options o{};
  o.pool_slabs = pool_slabs;
  o.device = -1;
  return lsb_map_create_ex(log2_buckets, &o, out);
}

int lsb_map_destroy(lsb_map* m) {
  if (!m) return LSB_ERR_ARG;
  m->t.release();
  delete m;
  return LSB_OK;
}

int lsb_map_get(lsb_map* m, const uint64_t* keys, lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_reads(keys, out, kOutResult, n, s);
}

int lsb_map_put(lsb_map* m, const uint64_t* keys, const uint64_t* vals, uint64_t* old_out,
                size_t n, cudaStream_t s) {
  if (!m || (n && (!keys || !vals))) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 8) || !aligned(old_out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_plain(nullptr, kOpWrite, keys, 1, vals, 1, old_out, kOutOld, n, s);
}

int lsb_map_put_pairs(lsb_map* m, const lsb_kv* ops, uint64_t* old_out, size_t n,
                      cudaStream_t s) {
  if (!m || (n && !ops)) return LSB_ERR_ARG;
  if (!aligned(ops, 8) || !aligned(old_out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  const uint64_t* base = reinterpret_cast<const uint64_t*>(ops);
  return m->t.run_plain(nullptr, kOpWrite, base, 2, base + 1, 2, old_out, kOutOld, n, s);
}

int lsb_map_update(lsb_map* m, const lsb_kv* ops, lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && !ops)) return LSB_ERR_ARG;
  if (!aligned(ops, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  const uint64_t* base = reinterpret_cast<const uint64_t*>(ops);
  return m->t.run_plain(nullptr, kOpUpdate, base, 2, base + 1, 2, out, kOutResult, n, s);
}

// ---- 32-bit values (lslab::map<K, unsigned>)
int lsb_map_get_v32(lsb_map* m, const uint64_t* keys, lsb_result32* out, size_t n,
                    cudaStream_t s) {
  if (!m || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_reads(keys, out, kOutResult32, n, s);
}

int lsb_map_put_v32(lsb_map* m, const uint64_t* keys, const uint32_t* vals, uint32_t* old_out,
                    size_t n, cudaStream_t s) {
  if (!m || (n && (!keys || !vals))) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 4) || !aligned(old_out, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_plain(nullptr, kOpWrite, keys, 1, reinterpret_cast<const uint64_t*>(vals), 1,
                        old_out, kOutOld32, n, s, true);
}

int lsb_map_put_pairs_v32(lsb_map* m, const lsb_kv32* ops, uint32_t* old_out, size_t n,
                          cudaStream_t s) {
  if (!m || (n && !ops)) return LSB_ERR_ARG;
  if (!aligned(ops, 8) || !aligned(old_out, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  const uint64_t* base = reinterpret_cast<const uint64_t*>(ops);
  return m->t.run_plain(nullptr, kOpWrite, base, 2, base + 1, 4, old_out, kOutOld32, n, s, true);
}

int lsb_map_update_v32(lsb_map* m, const lsb_kv32* ops, lsb_result32* out, size_t n,
                       cudaStream_t s) {
  if (!m || (n && !ops)) return LSB_ERR_ARG;
  if (!aligned(ops, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  const uint64_t* base = reinterpret_cast<const uint64_t*>(ops);
  return m->t.run_plain(nullptr, kOpUpdate, base, 2, base + 1, 4, out, kOutResult32, n, s, true);
}

int lsb_map_remove(lsb_map* m, const uint64_t* keys, lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_plain(nullptr, kOpRemove, keys, 1, nullptr, 1, out, kOutResult, n, s);
}

int lsb_map_execute(lsb_map* m, const uint8_t* types, const uint64_t* keys, const uint64_t* vals,
                    lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && (!types || !keys))) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_plain(types, kOpRead, keys, 1, vals, 1, out, kOutResult, n, s);
}

int lsb_map_execute_fused(lsb_map* m, const uint8_t* types, const uint64_t* keys,
                          const uint64_t* vals, lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && (!types || !keys))) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  return m->t.run_fused(types, kOpRead, keys, vals, out, kOutResult, n, s);
}

uint32_t lsb_map_buckets(const lsb_map* m) { return m ? m->t.buckets : 0; }

int lsb_map_get_tuning(const lsb_map* m, lsb_tuning* out) {
  if (!m || !out) return LSB_ERR_ARG;
  m->t.get_tuning(out);
  return LSB_OK;
}

int lsb_map_set_tuning(lsb_map* m, const lsb_tuning* t) {
  if (!m || !t) return LSB_ERR_ARG;
  return m->t.set_tuning(*t);
}

int lsb_map_set_trace(lsb_map* m, int on) {
  if (!m) return LSB_ERR_ARG;
  return m->t.set_trace(on);
}

int lsb_map_read_trace(lsb_map* m, uint64_t* out, size_t cap, size_t* count, cudaStream_t s) {
  if (!m || (cap && !out)) return LSB_ERR_ARG;
  return m->t.read_trace(out, cap, count, s);
}

int lsb_map_status(lsb_map* m, uint32_t* flags, cudaStream_t s) {
  if (!m) return LSB_ERR_ARG;
  return m->t.read_status(flags, s);
}

int lsb_map_pool_usage(lsb_map* m, uint64_t* used, uint64_t* capacity, cudaStream_t s) {
  if (!m) return LSB_ERR_ARG;
  return m->t.pool_usage(used, capacity, s);
}

int lsb_map_size(lsb_map* m, uint64_t* count, cudaStream_t s) {
  if (!m || !count) return LSB_ERR_ARG;
  return m->t.size(count, s);
}

int lsb_map_compact(lsb_map* m, uint64_t* freed, cudaStream_t s) {
  if (!m) return LSB_ERR_ARG;
  return m->t.compact(freed, s);
}

int lsb_set_compact(lsb_set* p, uint64_t* freed, cudaStream_t s) {
  if (!p) return LSB_ERR_ARG;
  return p->t.compact(freed, s);
}

int lsb_map_dump(lsb_map* m, uint64_t* keys_out, uint64_t* vals_out, size_t cap,
                 uint64_t* count, cudaStream_t s) {
  if (!m || (cap && (!keys_out || !vals_out))) return LSB_ERR_ARG;
  return m->t.dump(keys_out, vals_out, cap, count, s);
}

// ------------------------------------------------------------------ set
int lsb_set_create_ex(unsigned log2_buckets, const lsb_options* opt, lsb_set** out) {
  if (!out) return LSB_ERR_ARG;
  *out = nullptr;
  lsb_set* p = new (std::nothrow) lsb_set();
  if (!p) return LSB_ERR_OOM;
  int e = p->t.init(log2_buckets, opt);
  if (e) {
    p->t.release();
    delete p;
    return e;
  }
  lsb_tuning cached;
  if (tuned_lookup(1, log2_buckets, &cached)) p->t.set_tuning(cached);
  *out = p;
  return LSB_OK;
}

int lsb_set_create(unsigned log2_buckets, uint64_t pool_slabs, lsb_set** out) {
  lsb_options o{};
  o.pool_slabs = pool_slabs;
  o.device = -1;
  return lsb_set_create_ex(log2_buckets, &o, out);
}

int lsb_set_destroy(lsb_set* p) {
  if (!p) return LSB_ERR_ARG;
  p->t.release();
  delete p;
  return LSB_OK;
}

int lsb_set_insert(lsb_set* p, const uint32_t* keys, bool* out, size_t n, cudaStream_t s) {
  if (!p || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return p->t.run_plain(nullptr, kOpWrite, keys, 1, nullptr, 1, out, kOutBool, n, s);
}

int lsb_set_contains(lsb_set* p, const uint32_t* keys, bool* out, size_t n, cudaStream_t s) {
  if (!p || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return p->t.run_reads(keys, out, kOutBool, n, s);
}

int lsb_set_remove(lsb_set* p, const uint32_t* keys, bool* out, size_t n, cudaStream_t s) {
  if (!p || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return p->t.run_plain(nullptr, kOpRemove, keys, 1, nullptr, 1, out, kOutBool, n, s);
}

int lsb_set_execute(lsb_set* p, const uint8_t* types, const uint32_t* keys, bool* out, size_t n,
                    cudaStream_t s) {
  if (!p || (n && (!types || !keys))) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return p->t.run_plain(types, kOpRead, keys, 1, nullptr, 1, out, kOutBool, n, s);
}

int lsb_set_execute_fused(lsb_set* p, const uint8_t* types, const uint32_t* keys, bool* out,
                          size_t n, cudaStream_t s) {
  if (!p || (n && (!types || !keys))) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  return p->t.run_fused(types, kOpRead, keys, nullptr, out, kOutBool, n, s);
}

uint32_t lsb_set_buckets(const lsb_set* p) { return p ? p->t.buckets : 0; }

int lsb_set_get_tuning(const lsb_set* p, lsb_tuning* out) {
  if (!p || !out) return LSB_ERR_ARG;
  p->t.get_tuning(out);
  return LSB_OK;
}

int lsb_set_set_tuning(lsb_set* p, const lsb_tuning* t) {
  if (!p || !t) return LSB_ERR_ARG;
  return p->t.set_tuning(*t);
}

int lsb_set_set_trace(lsb_set* p, int on) {
  if (!p) return LSB_ERR_ARG;
  return p->t.set_trace(on);
}

int lsb_set_read_trace(lsb_set* p, uint64_t* out, size_t cap, size_t* count, cudaStream_t s) {
  if (!p || (cap && !out)) return LSB_ERR_ARG;
  return p->t.read_trace(out, cap, count, s);
}

int lsb_set_status(lsb_set* p, uint32_t* flags, cudaStream_t s) {
  if (!p) return LSB_ERR_ARG;
  return p->t.read_status(flags, s);
}

int lsb_set_pool_usage(lsb_set* p, uint64_t* used, uint64_t* capacity, cudaStream_t s) {
  if (!p) return LSB_ERR_ARG;
  return p->t.pool_usage(used, capacity, s);
}

int lsb_set_size(lsb_set* p, uint64_t* count, cudaStream_t s) {
  if (!p || !count) return LSB_ERR_ARG;
  return p->t.size(count, s);
}

int lsb_set_dump(lsb_set* p, uint32_t* keys_out, size_t cap, uint64_t* count, cudaStream_t s) {
  if (!p || (cap && !keys_out)) return LSB_ERR_ARG;
  return p->t.dump(keys_out, nullptr, cap, count, s);
}

// ------------------------------------------------------- graphs / autotune
int lsb_map_autotune(lsb_map* m, const uint8_t* types, const uint64_t* keys, const uint64_t* vals,
                     lsb_result* out, size_t n, cudaStream_t s, lsb_tuning* best) {
  if (!m || !n || !types || !keys) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  return autotune(m->t, 0, types, keys, vals, out, kOutResult, n, s, best);
}

int lsb_set_autotune(lsb_set* p, const uint8_t* types, const uint32_t* keys, bool* out, size_t n,
                     cudaStream_t s, lsb_tuning* best) {
  if (!p || !n || !types || !keys || !aligned(keys, 4)) return LSB_ERR_ARG;
  return autotune(p->t, 1, types, keys, nullptr, out, kOutBool, n, s, best);
}

int lsb_autotune_lookup(int container, unsigned log2_buckets, lsb_tuning* out) {
  if (!out || (container != 0 && container != 1)) return LSB_ERR_ARG;
  return tuned_lookup(container, log2_buckets, out) ? LSB_OK : LSB_ERR_STATE;
}

int lsb_map_capture_fused(lsb_map* m, const uint8_t* types, const uint64_t* keys,
                          const uint64_t* vals, lsb_result* out, size_t n, lsb_graph** graph) {
  if (!m || !graph || !n || !types || !keys) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  return capture_fused(m->t, types, keys, vals, out, kOutResult, n, graph);
}

int lsb_set_capture_fused(lsb_set* p, const uint8_t* types, const uint32_t* keys, bool* out,
                          size_t n, lsb_graph** graph) {
  if (!p || !graph || !n || !types || !keys || !aligned(keys, 4)) return LSB_ERR_ARG;
  return capture_fused(p->t, types, keys, nullptr, out, kOutBool, n, graph);
}

int lsb_graph_launch(lsb_graph* g, cudaStream_t s) {
  if (!g || !g->exec) return LSB_ERR_ARG;
  return cudaGraphLaunch(g->exec, s) == cudaSuccess ? LSB_OK : LSB_ERR_CUDA;
}

int lsb_graph_destroy(lsb_graph* g) {
  if (!g) return LSB_ERR_ARG;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return LSB_OK;
}

// ------------------------------------------------------ device per-warp API
int lsb_map_device_view(const lsb_map* m, lsb_table_view* out) {
  if (!m || !out) return LSB_ERR_ARG;
  fill_view(m->t, out);
  return LSB_OK;
}

int lsb_set_device_view(const lsb_set* s, lsb_table_view* out) {
  if (!s || !out) return LSB_ERR_ARG;
  fill_view(s->t, out);
  return LSB_OK;
}

// ------------------------------------------------------------------ misc
const char* lsb_error_string(int code) {
  switch (code) {
    case LSB_OK: return "ok";
    case LSB_ERR_ARG: return "invalid argument";
    case LSB_ERR_OOM: return "out of memory (slab pool or device memory)";
    case LSB_ERR_TIMEOUT: return "a bounded device wait gave up";
    case LSB_ERR_CUDA: return "CUDA runtime error";
    case LSB_ERR_STATE: return "invalid state";
    case LSB_ERR_IO: return "file could not be read or written, or is not a valid checkpoint";
    default: return "unknown error";
  }
}

int lsb_version(void) { return 100; }

/* ---------------------------------------------------------------- serving */
int lsb_serve_create(lsb_map* m, const lsb_serve_options* opt, lsb_server** out) {
  if (!m || !out) return LSB_ERR_ARG;
  *out = nullptr;
  lsb_serve_options o{};
  if (opt) o = *opt;
  const uint32_t wave = o.max_wave_ops ? o.max_wave_ops : (1u << 16);
  const uint64_t ring = o.ring_requests ? o.ring_requests : 16384;
  const uint64_t arena = o.arena_ops ? o.arena_ops : (1ull << 22);
  if (wave > m->t.sc.max_window || wave < 1 || arena < wave || ring > (1ull << 24) ||
      arena > (1ull << 32))
    return LSB_ERR_ARG;
  lsb_server* s = new (std::nothrow) lsb_server;
  if (!s) return LSB_ERR_OOM;
  s->map = m;
  s->device = m->t.device;
  s->ring_cap = ring;
  s->arena_cap = arena;
  s->max_wave_ops = wave;
  s->idle_ns = (uint64_t)(o.idle_ms ? o.idle_ms : 10000) * 1000000ull;
  s->taken.assign(ring, 0);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  const unsigned fl = cudaHostAllocMapped;
  bool ok =
      cudaHostAlloc((void**)&s->ctl, sizeof(ServeCtl), fl) == cudaSuccess &&
      cudaHostAlloc((void**)&s->ring, sizeof(ServeReq) * ring, fl) == cudaSuccess &&
      cudaHostAlloc((void**)&s->a_types, arena, fl) == cudaSuccess &&
      cudaHostAlloc((void**)&s->a_keys, 8 * arena, fl) == cudaSuccess &&
      cudaHostAlloc((void**)&s->a_vals, 8 * arena, fl) == cudaSuccess &&
      cudaHostAlloc((void**)&s->a_out, sizeof(lsb_result) * arena, fl) == cudaSuccess &&
      cudaMalloc(&s->d_types, wave) == cudaSuccess &&
      cudaMalloc(&s->d_keys, 8ull * wave) == cudaSuccess &&
      cudaMalloc(&s->d_vals, 8ull * wave) == cudaSuccess &&
      cudaMalloc(&s->d_wave, 2 * sizeof(WaveDesc)) == cudaSuccess &&
      cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess;
  cudaSetDevice(prev);
  if (!ok) {
    cudaGetLastError();
    s->release();
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return LSB_ERR_OOM;
  }
  std::memset(s->ctl, 0, sizeof(ServeCtl));
  std::memset(s->ring, 0, sizeof(ServeReq) * ring);
  *out = s;
  return LSB_OK;
}

int lsb_serve_start(lsb_server* s) {
  if (!s) return LSB_ERR_ARG;
  if (s->running) return LSB_ERR_STATE;
  auto& tb = s->map->t;
  int prev = 0;
  cudaGetDevice(&prev);
  LSB_CK(cudaSetDevice(s->device));
  s->ctl->stop = 0;
  s->ctl->state = 0;
  ServeJob j{};
  j.ctl = dev_ptr(s->ctl);
  j.ring = dev_ptr(s->ring);
  j.ring_cap = s->ring_cap;
  j.a_types = dev_ptr(s->a_types);
  j.a_keys = dev_ptr(s->a_keys);
  j.a_vals = dev_ptr(s->a_vals);
  j.a_out = dev_ptr(s->a_out);
  j.arena_cap = s->arena_cap;
  j.d_types = s->d_types;
  j.d_keys = s->d_keys;
  j.d_vals = s->d_vals;
  j.wave = s->d_wave;
  j.max_wave_ops = s->max_wave_ops;
  j.idle_ns = s->idle_ns;
  if (!j.ctl || !j.ring || !j.a_types || !j.a_keys || !j.a_vals || !j.a_out) {
    cudaSetDevice(prev);
    return LSB_ERR_CUDA;
  }
  FusedJob<MapTraits>& fj = j.fj;
  fj.base = tb.window(s->d_types, 0, s->d_keys, 1, s->d_vals, 1, j.a_out, kOutResult,
                      s->max_wave_ops);
  fj.window = tb.sc.max_window;
  fj.fused_epoch = tb.fused_epoch;
  fj.chunk = tb.tune.chunk;
  fj.dedup = tb.tune.dedup;
  fj.split_q16 = 65536;  // a wave: every op in one probe pass (one grid barrier fewer)
  fj.trace = nullptr;
  fj.bins = tb.bins;
  fj.binned = 0;
  fj.bin_shift = 0;
  const int per_sm_grid = tb.fused_grid();  // same occupancy as the fused kernel
  if (per_sm_grid <= 0) {
    cudaSetDevice(prev);
    return LSB_ERR_STATE;
  }
  int per_sm = 0;
  const void* f = tb.tune.prefetch == 0 ? (const void*)k_serve<1>
                : tb.tune.prefetch == 1 ? (const void*)k_serve<2> : (const void*)k_serve<3>;
  if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kSortSmemBytes) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, (int)tb.tune.block,
                                                    kSortSmemBytes) != cudaSuccess ||
      per_sm <= 0) {
    cudaGetLastError();
    cudaSetDevice(prev);
    return LSB_ERR_CUDA;
  }
  TableView tv = tb.view();
  Scratch scv = tb.sc;
  GridBarrier* b = tb.bar;
  void* args[] = {&tv, &scv, &j, &b};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(per_sm * tb.num_sms);
  cfg.blockDim = dim3(tb.tune.block);
  cfg.dynamicSmemBytes = kSortSmemBytes;
  cfg.stream = s->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelExC(&cfg, f, args);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return LSB_ERR_CUDA;
  }
  s->running = true;
  return LSB_OK;
}

int lsb_serve_submit(lsb_server* s, const uint8_t* types, const uint64_t* keys,
                     const uint64_t* vals, uint32_t n, uint64_t* ticket) {
  if (!s || !keys || !ticket || n == 0 || n > s->max_wave_ops) return LSB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->submit_mu);
  const uint64_t freed_req = s->freed_req.load(std::memory_order_acquire);
  const uint64_t freed_op = s->freed_op.load(std::memory_order_acquire);
  // a request never wraps the arena's end (a wave's ops stay contiguous):
  // skip to the next lap when it would
  uint64_t at = s->next_op;
  if (at % s->arena_cap + n > s->arena_cap) at += s->arena_cap - at % s->arena_cap;
  if (s->next_req - freed_req >= s->ring_cap || at + n - freed_op > s->arena_cap)
    return LSB_ERR_STATE;  // full: take results, then retry
  s->next_op = at;
  uint32_t puts = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const uint64_t pos = (s->next_op + i) % s->arena_cap;
    const uint8_t ty = types ? types[i] : (uint8_t)kOpRead;
    s->a_types[pos] = ty;
    s->a_keys[pos] = keys[i];
    s->a_vals[pos] = vals ? vals[i] : 0;
    puts += ty == kOpWrite;
  }
  ServeReq& q = s->ring[s->next_req % s->ring_cap];
  q.op_off = s->next_op;
  q.n = n;
  q.puts = puts;
  q.status = -1;
  *ticket = s->next_req;
  s->next_op += n;
  ++s->next_req;
  std::atomic_thread_fence(std::memory_order_release);
  __atomic_store_n(&s->ctl->submitted, s->next_req, __ATOMIC_RELEASE);
  return LSB_OK;
}

int lsb_serve_poll(lsb_server* s, uint64_t ticket, int* done) {
  if (!s || !done) return LSB_ERR_ARG;
  *done = __atomic_load_n(&s->ctl->completed, __ATOMIC_ACQUIRE) > ticket;
  return LSB_OK;
}

int lsb_serve_take(lsb_server* s, uint64_t ticket, lsb_result* out, int* status) {
  if (!s) return LSB_ERR_ARG;
  if (__atomic_load_n(&s->ctl->completed, __ATOMIC_ACQUIRE) <= ticket) return LSB_ERR_STATE;
  std::lock_guard<std::mutex> lk(s->take_mu);
  const uint64_t fr = s->freed_req.load(std::memory_order_relaxed);
  if (ticket < fr || ticket - fr >= s->ring_cap) return LSB_ERR_ARG;
  const ServeReq& q = s->ring[ticket % s->ring_cap];
  if (s->taken[ticket % s->ring_cap]) return LSB_ERR_STATE;
  if (status) *status = q.status;
  if (out) {
    for (uint32_t i = 0; i < q.n; ++i) out[i] = s->a_out[(q.op_off + i) % s->arena_cap];
  }
  s->taken[ticket % s->ring_cap] = 1;
  // reclaim the FIFO prefix of taken requests
  uint64_t r = fr, op = s->freed_op.load(std::memory_order_relaxed);
  const uint64_t done = __atomic_load_n(&s->ctl->completed, __ATOMIC_ACQUIRE);
  while (r < done && s->taken[r % s->ring_cap]) {
    const ServeReq& d = s->ring[r % s->ring_cap];
    s->taken[r % s->ring_cap] = 0;
    op = d.op_off + d.n;
    ++r;
  }
  s->freed_op.store(op, std::memory_order_release);
  s->freed_req.store(r, std::memory_order_release);
  return LSB_OK;
}

int lsb_serve_stop(lsb_server* s, lsb_serve_stats* stats) {
  if (!s) return LSB_ERR_ARG;
  int rc = LSB_OK;
  if (s->running) {
    __atomic_store_n(&s->ctl->stop, 1u, __ATOMIC_RELEASE);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) rc = LSB_ERR_CUDA;
    s->running = false;
  }
  if (stats) lsb_serve_query(s, stats);
  return rc;
}

int lsb_serve_query(lsb_server* s, lsb_serve_stats* stats) {
  if (!s || !stats) return LSB_ERR_ARG;
  volatile ServeCtl* c = s->ctl;
  stats->waves = c->waves;
  stats->ops = c->ops;
  stats->requests = c->completed;
  stats->state = c->state;
  stats->pad = 0;
  stats->gather_ns = c->t_gather;
  stats->engine_ns = c->t_engine;
  stats->tail_ns = c->t_tail;
  stats->wait_ns = c->t_wait;
  return LSB_OK;
}

int lsb_serve_destroy(lsb_server* s) {
  if (!s) return LSB_ERR_ARG;
  if (s->running) lsb_serve_stop(s, nullptr);
  s->release();
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return LSB_OK;
}

}  // extern "C"
