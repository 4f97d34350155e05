// The library's ordering step (k_sort / the fused kernel's sort section) as
// a sequence of emulated grid steps: each step runs every block to
// completion before the next begins, which is what the grid barriers
// between the steps guarantee on the device (test infrastructure).
#pragma once

#include <vector>

#include "simt_host.h"
#include "lsb_window.cuh"

namespace emu {

template <class Tr>
void sort_window(const lsb::Scratch& sc, const lsb::Window<Tr>& w, unsigned nblocks,
                 unsigned nthreads, std::vector<uint32_t>& smem) {
  using namespace lsb;
  auto grid_step = [&](auto&& f) {
    for (unsigned b = 0; b < nblocks; ++b) run_block(nthreads, b, nblocks, f);
  };
  grid_step([&] { phase_sort_big<Tr>(sc, w, smem.data()); });
  if (huge_groups(sc, w.cnt) == 0) return;
  grid_step([&] {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    huge_hist<Tr>(sc, w, g >> 5, (gridDim.x * blockDim.x) >> 5);
  });
  grid_step([&] { huge_scan<Tr>(sc, w, smem.data()); });
  grid_step([&] {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    huge_scatter<Tr>(sc, w, g >> 5, (gridDim.x * blockDim.x) >> 5);
  });
  grid_step([&] {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    huge_runs<Tr>(sc, w, smem.data(), g, gridDim.x * blockDim.x);
  });
}

// Scratch for `window` ops sized as the library sizes it, in caller-owned
// host buffers (exact sizes, so a sanitizer's redzones sit after each array).
inline void alloc_scratch(lsb::Scratch& sc, uint32_t window, uint32_t* status,
                          std::vector<std::unique_ptr<uint8_t[]>>& keep) {
  using namespace lsb;
  auto alloc = [&](size_t bytes) {
    keep.emplace_back(new uint8_t[bytes]());
    return (void*)keep.back().get();
  };
  uint32_t g = 64;
  while (g < 2 * window) g <<= 1;
  uint32_t cg = 64;
  while (cg < 2 * (window / kChunk + window / (kInline + 1) + 1)) cg <<= 1;
  sc = Scratch{};
  sc.gtab = (uint64_t*)alloc(8ull * g);
  sc.ginl = (uint32_t*)alloc(4ull * kInline * g);
  sc.ctab = (uint64_t*)alloc(8ull * cg);
  sc.cdat = (uint32_t*)alloc(4ull * kChunk * cg);
  sc.gmask = g - 1;
  sc.cmask = cg - 1;
  sc.max_window = window;
  sc.minfo = (uint64_t*)alloc(8ull * window);
  sc.mloc = (uint64_t*)alloc(8ull * window);
  sc.pred = (uint32_t*)alloc(4ull * window);
  sc.goff = (uint32_t*)alloc(4ull * g);
  sc.seg = (uint32_t*)alloc(4ull * window);
  sc.mlist = (uint32_t*)alloc(4ull * window);
  sc.big = (uint32_t*)alloc(4ull * (window / (kInline + 1) + 1));
  sc.large = (uint32_t*)alloc(4ull * (window / (kWarpSort + 1) + 1));
  sc.cnt = (WinCounters*)alloc(2 * sizeof(WinCounters));
  sc.obin = (uint8_t*)alloc(window);
  sc.perm = (uint32_t*)alloc(4ull * window);
  sc.clist = (uint32_t*)alloc(4ull * clist_cap(window));
  sc.hcap = window / (kHugeMin + 1) + 1;
  sc.rcap = window / kRunUnit + sc.hcap;
  sc.hlist = (uint32_t*)alloc(4ull * sc.hcap);
  sc.hrec = (uint32_t*)alloc(16ull * sc.hcap);
  sc.hbins = (uint32_t*)alloc(4ull * kHugeBins * sc.hcap);
  sc.hrun = (uint32_t*)alloc(4ull * kHugeBins * sc.hcap);
  sc.runs = (uint32_t*)alloc(16ull * sc.rcap);
  sc.lnu = (uint32_t*)alloc(4ull * window);
  sc.rnu = (uint32_t*)alloc(4ull * sc.rcap);
  sc.status = status;
}

}  // namespace emu
