// Probe-rate calibration: the memory accesses of one get at a uniformly
// random key, and nothing else, so its rate is the ceiling that address
// translation and DRAM latency put on random lookups over a table of this
// size.  Thread i reads an 8-byte request word (coalesced), picks a slab
// uniformly, loads its 32-byte meta sector, then, dependent on that load, one
// 16-byte slot of the same slab (the candidate slot a tag match would give),
// and stores a 16-byte result (coalesced): the 88 bytes a get moves.  The
// loads use the same cache policy as the read kernel (k_read).  No
// counterpart in the reference; a measuring instrument for the bench.
#include <cuda_runtime.h>

#include <cstdint>

#include "lsb.h"
#include "lsb_core.cuh"

namespace {

__global__ void __launch_bounds__(256, 8)
    k_probe_calibrate(const uint8_t* slabs, uint64_t nslabs, uint32_t slab_bytes,
                      const uint64_t* req, uint64_t* out, uint32_t n, uint64_t seed) {
  using namespace lsb;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t r = ld_cs_u64(req + i);
  const uint64_t h = mix64(r ^ seed ^ ((uint64_t)i << 32));
  const uint64_t s = h % nslabs;
  const uint8_t* slab = slabs + s * slab_bytes;
  const Meta m = load_meta<true>(slab);
  const uint32_t slots = (slab_bytes - kMetaBytes) / 16u;
  const uint32_t slot = (m.tag[0] ^ m.next ^ (uint32_t)h) % slots;
  const ulonglong2 kv = ld_ca_v2u64(slab + kMetaBytes + slot * 16u);
  st_cs_u64(out + 2 * (size_t)i, kv.x ^ h);
  st_cs_u64(out + 2 * (size_t)i + 1, kv.y);
}

}  // namespace

extern "C" int lsb_probe_calibrate(const void* slabs, uint64_t nslabs, uint32_t slab_bytes,
                                   const uint64_t* req, uint64_t* out, size_t n, uint64_t seed,
                                   cudaStream_t s) {
  if (!slabs || !req || !out || nslabs == 0 || slab_bytes < lsb::kMetaBytes + 16 ||
      slab_bytes % 32 != 0 || n > 0xFFFFFFFFull)
    return LSB_ERR_ARG;
  if (((uintptr_t)slabs & 31) || ((uintptr_t)req & 7) || ((uintptr_t)out & 15)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  k_probe_calibrate<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      static_cast<const uint8_t*>(slabs), nslabs, slab_bytes, req, out, (uint32_t)n, seed);
  return cudaGetLastError() == cudaSuccess ? LSB_OK : LSB_ERR_CUDA;
}
