// CPU test driver for a whole map batch on the per-phase path (test
// infrastructure): the library's probe, ordering and resolve phases run
// window by window on an emulated grid with the launch shapes the library
// uses (blocks of one step run one after another; no step waits on another
// block).  Built with AddressSanitizer it checks every access of those
// phases against its buffer; the results are written for comparison with
// the oracle.
//
// usage: window_emu <ops file> <log2 buckets> <pool slabs> <block threads> <out file> [mode]
// mode muts_first: the probe runs as the fused kernel's split-0 form does:
// the mutation list, the probe of its tiles, then a pass over the reads.
// mode muts_first_binned: the same with the reads probed in table-region
// order (region counts beside the list, the scatter beside the list probe).
// mode compact: one-pass probe, and every bucket's chain compacted after each
// window (lsb_map_compact's step), so later windows run on packed chains and
// on slabs taken back from the free stack.
// mode lockfree: one-pass probe, writers without bucket locks (CAS on slab
// words, LSB_LOCK_FREE).
// ops file: u32 n, u32 max_window, n x u8 type, n x u64 key, n x u64 value
// out file: n x lsb_result (u8 found, 7 pad, u64 value), then u32 status,
// u64 pool cursor, u64 free-stack top
#include "simt_host.h"
#include "lsb_window.cuh"
#include "emu_phases.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

using namespace lsb;
using Tr = MapTraits;

int main(int argc, char** argv) {
  if (argc != 6 && argc != 7) {
    std::fprintf(stderr, "usage: window_emu <ops> <log2> <pool> <block> <out> [mode]\n");
    return 2;
  }
  const bool binned = argc == 7 && std::strcmp(argv[6], "muts_first_binned") == 0;
  const bool muts_first = binned || (argc == 7 && std::strcmp(argv[6], "muts_first") == 0);
  const bool compact = argc == 7 && std::strcmp(argv[6], "compact") == 0;
  const bool lockfree = argc == 7 && std::strcmp(argv[6], "lockfree") == 0;
  // mode v32put: every op a put (types ignored), 32-bit values (the low half
  // of each value), 32-bit old values out (lsb_map_put_v32's window)
  const bool v32put = argc == 7 && std::strcmp(argv[6], "v32put") == 0;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  uint32_t n = 0, window = 0;
  if (std::fread(&n, 4, 1, f) != 1 || std::fread(&window, 4, 1, f) != 1) return 2;
  std::vector<std::unique_ptr<uint8_t[]>> keep;
  auto alloc = [&](size_t bytes) {
    keep.emplace_back(new uint8_t[bytes]());
    return (void*)keep.back().get();
  };
  uint8_t* types = (uint8_t*)alloc(n);
  uint64_t* keys = (uint64_t*)alloc(8ull * n);
  uint64_t* vals = (uint64_t*)alloc(8ull * n);
  if (std::fread(types, 1, n, f) != n || std::fread(keys, 8, n, f) != n ||
      std::fread(vals, 8, n, f) != n)
    return 2;
  std::fclose(f);
  const unsigned log2 = (unsigned)std::atoi(argv[2]);
  const uint64_t pool_slabs = std::strtoull(argv[3], nullptr, 10);
  const unsigned block = (unsigned)std::atoi(argv[4]);
  const uint32_t buckets = 1u << log2;
  const unsigned num_sms = 148;

  TableView t{};
  t.slabs = (uint8_t*)alloc(((size_t)buckets + pool_slabs) * Tr::kSlabBytes);
  t.locks = (int32_t*)alloc(4ull * buckets);
  t.status = (uint32_t*)alloc(4);
  t.pool = (uint64_t*)alloc(8ull * kPoolWords);
  t.pool[0] = buckets;
  t.pool[1] = buckets + pool_slabs;
  t.free_stack = (uint32_t*)alloc(4ull * std::max<uint64_t>(1, pool_slabs));
  t.mask = buckets - 1;
  t.lock_mode = lockfree ? kLockFree : kLockWriter;
  t.chunk = (uint32_t)std::min<uint64_t>(kPoolChunkMax,
                                         std::max<uint64_t>(1, pool_slabs / (8ull * num_sms)));
  Scratch sc;
  emu::alloc_scratch(sc, window, t.status, keep);
  uint8_t* out = (uint8_t*)alloc(16ull * n);
  uint32_t* vals32 = (uint32_t*)alloc(4ull * n);
  for (uint32_t i = 0; i < n; ++i) vals32[i] = (uint32_t)vals[i];
  std::vector<uint32_t> smem(kSortSmemBytes / 4);
  BinCounters* bins = (BinCounters*)alloc(sizeof(BinCounters));
  const uint32_t bin_shift = log2 > kBinBits ? log2 - kBinBits : 0u;

  uint32_t epoch = 0;
  for (uint32_t off = 0; off < n; off += window) {
    const uint32_t m = std::min(window, n - off);
    Window<Tr> w{};
    w.types = types + off;
    w.keys = keys + off;
    w.vals = vals + off;
    w.out = out + (size_t)off * 16;
    w.kstride = 1;
    w.vstride = 1;
    w.n = m;
    epoch += 2;
    w.epoch = epoch;
    w.out_kind = kOutResult;
    if (v32put) {
      w.types = nullptr;
      w.uniform = kOpWrite;
      w.vals = reinterpret_cast<const uint64_t*>(vals32 + off);
      w.v32 = 1;
      w.out = out + (size_t)off * 4;
      w.out_kind = kOutOld32;
    }
    w.cnt = &sc.cnt[0];
    std::memset(sc.cnt, 0, 2 * sizeof(WinCounters));
    std::memset(bins, 0, sizeof(BinCounters));
    // probe: the library's grid for prefetch 0, static stride
    const unsigned per_sm = 2048 / block;
    const unsigned grid = std::max(1u, std::min(per_sm * num_sms, (m + block - 1) / block));
    for (unsigned b = 0; b < grid; ++b)
      emu::run_block(block, b, grid, [&] {
        const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
        if (muts_first) {
          phase_list_muts<Tr>(sc, w, warp, nwarps);
          if (binned) phase_bin_count<Tr>(t, w, sc.obin, bins, bin_shift);
        } else {
          phase_probe<Tr, true, 1>(t, sc, w, warp, nwarps, &w.cnt->probe_cursor, 0, false);
        }
      });
    if (muts_first) {
      for (unsigned b = 0; b < grid; ++b)
        emu::run_block(block, b, grid, [&] {
          const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
          const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
          const uint32_t listed = std::min(w.cnt->clist_count, clist_cap(sc.max_window));
          phase_probe_list<Tr>(t, sc, w, warp, nwarps, false);
          if (binned)
            phase_bin_scatter<Tr>(w, sc.obin, sc.perm, bins);
          else  // reads until every list tile is done, as the fused kernel does
            phase_read_lean<Tr>(t, w, &w.cnt->late_cursor, 0, m, &w.cnt->tiles_done,
                                (listed + 31) / 32);
        });
      for (unsigned b = 0; b < grid; ++b)
        emu::run_block(block, b, grid, [&] {
          const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
          const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
          if (binned)
            phase_probe<Tr, false, 1>(t, sc, w, warp, nwarps, &w.cnt->late_cursor, block, false,
                                      ProbeSel{0, m, false}, 0, sc.perm);
          else
            phase_read_lean<Tr>(t, w, &w.cnt->late_cursor, 0, m);
        });
    }
    emu::sort_window<Tr>(sc, w, num_sms, 256, smem);
    const unsigned rgrid = std::max(1u, std::min(num_sms * 8, (m + 255) / 256));
    for (unsigned b = 0; b < rgrid; ++b)
      emu::run_block(256, b, rgrid, [&] {
        const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
        const uint32_t nt = gridDim.x * blockDim.x;
        phase_resolve_mutations<Tr>(t, sc, w, tid, nt);
        phase_resolve_reads<Tr>(sc, w, tid, nt);
      });
    if (compact) {
      if ((long long)t.pool[kPoolTop] < 0) t.pool[kPoolTop] = 0;  // k_pool_clamp
      const unsigned cgrid = (buckets + 255) / 256;
      for (unsigned b = 0; b < cgrid; ++b)
        emu::run_block(256, b, cgrid, [&] {
          const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
          if (k < buckets) compact_bucket<Tr>(t, k);
        });
    }
  }
  FILE* o = std::fopen(argv[5], "wb");
  if (!o) return 2;
  std::fwrite(out, v32put ? 4 : 16, n, o);
  std::fwrite(t.status, 4, 1, o);
  std::fwrite(&t.pool[0], 8, 1, o);
  std::fwrite(&t.pool[kPoolTop], 8, 1, o);
  std::fclose(o);
  std::printf("done status=%#x\n", *t.status);
  return 0;
}
