// CPU test driver for the ordering phase of a window (test infrastructure).
//
// Reads one window of ops (types, keys), joins every mutation to its key's
// group with the library's own group_join/group_store in a shuffled order
// (as concurrent warps would), then runs the library's ordering step on an
// emulated grid and checks, for every group of more than kInline members,
// that its list in seg is the members in op-index order and that each
// member's predecessor word names the previous member (the last one
// flagged).  Prints "OK ..." or the first mismatch and exits non-zero.
//
// usage: order_emu <window file> <threads per block> <blocks> <seed>
// window file: u32 n, u32 max_window, n x u8 type, n x u64 key (little endian)
#include "simt_host.h"
#include "lsb_window.cuh"
#include "emu_phases.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <vector>

using namespace lsb;
using Tr = MapTraits;

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: order_emu <window file> <threads> <blocks> <seed>\n");
    return 2;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  uint32_t n = 0, window = 0;
  if (std::fread(&n, 4, 1, f) != 1 || std::fread(&window, 4, 1, f) != 1 || n > window) return 2;
  std::vector<uint8_t> types(n);
  std::vector<uint64_t> keys(n);
  if (std::fread(types.data(), 1, n, f) != n || std::fread(keys.data(), 8, n, f) != n) return 2;
  std::fclose(f);
  const unsigned nthreads = (unsigned)std::atoi(argv[2]);
  const unsigned nblocks = (unsigned)std::atoi(argv[3]);
  const unsigned seed = (unsigned)std::atoi(argv[4]);

  std::vector<std::unique_ptr<uint8_t[]>> keep;
  uint32_t status = 0;
  Scratch sc;
  emu::alloc_scratch(sc, window, &status, keep);
  // stale contents, as reused device memory would hold
  std::fill(sc.seg, sc.seg + window, 0x5A5A5A5Au);
  std::fill(sc.pred, sc.pred + window, 0x5A5A5A5Au);
  std::fill(sc.cdat, sc.cdat + (size_t)kChunk * (sc.cmask + 1ull), 0x5A5A5A5Au);

  Window<Tr> w{};
  w.types = types.data();
  w.keys = keys.data();
  w.kstride = 1;
  w.vstride = 1;
  w.n = n;
  w.epoch = 2;
  w.out_kind = kOutNone;
  w.cnt = &sc.cnt[0];

  // phase A joins, one mutation at a time in a shuffled order
  std::vector<uint32_t> muts;
  for (uint32_t i = 0; i < n; ++i)
    if (types[i] != kOpRead) muts.push_back(i);
  std::mt19937 rng(seed);
  std::shuffle(muts.begin(), muts.end(), rng);
  for (uint32_t m : muts) {
    uint32_t pos = 0;
    const uint32_t slot = group_join<Tr>(sc, w, m, keys[m], Tr::hash(keys[m]), 1, &pos);
    group_store<Tr>(sc, w, slot, pos, m, 0);
  }

  std::vector<uint32_t> smem(kSortSmemBytes / 4);
  emu::sort_window<Tr>(sc, w, nblocks, nthreads, smem);

  std::map<uint64_t, std::vector<uint32_t>> groups;
  for (uint32_t i = 0; i < n; ++i)
    if (types[i] != kOpRead) groups[keys[i]].push_back(i);
  size_t checked = 0, biggest = 0;
  for (auto& [key, mem] : groups) {
    const uint32_t c = (uint32_t)mem.size();
    if (c <= kInline) continue;
    const uint32_t slot = (uint32_t)(sc.minfo[mem[0]] >> 32) & sc.gmask;
    const uint32_t off = sc.goff[slot];
    if (off > window || c > window - off) {
      std::printf("FAIL group key %llu: offset %u out of range\n", (unsigned long long)key, off);
      return 1;
    }
    for (uint32_t j = 0; j < c; ++j) {
      if (sc.seg[off + j] != mem[j]) {
        std::printf("FAIL group key %llu (c=%u): seg[%u]=%u want %u\n", (unsigned long long)key, c,
                    j, sc.seg[off + j], mem[j]);
        return 1;
      }
      const uint32_t want = (j ? mem[j - 1] + 1 : 0u) | (j + 1 == c ? kPredLast : 0u);
      if (sc.pred[mem[j]] != want) {
        std::printf("FAIL group key %llu (c=%u): pred[%u]=%#x want %#x\n",
                    (unsigned long long)key, c, mem[j], sc.pred[mem[j]], want);
        return 1;
      }
    }
    ++checked;
    biggest = std::max<size_t>(biggest, c);
  }
  if (status != 0) {
    std::printf("FAIL status %#x\n", status);
    return 1;
  }
  std::printf("OK groups=%zu biggest=%zu\n", checked, biggest);
  return 0;
}
