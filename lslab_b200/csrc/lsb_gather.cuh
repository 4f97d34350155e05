// The serving loop's gather: a wave's ops from the host-mapped request arena
// into device memory.  Included by lsb_api.cu; the CPU tests compile it for
// the host (LSB_HOST_EMU) and check its index arithmetic on every alignment.
#pragma once

#include <cstdint>

#include "lsb_core.cuh"

namespace lsb {

#ifndef LSB_HOST_EMU
// Volatile loads (.cv): the host rewrites arena slots between waves, so no
// cached copy may be reused.
__device__ __forceinline__ uint8_t ld_cv_u8(const uint8_t* p) { return __ldcv(p); }
__device__ __forceinline__ uint64_t ld_cv_u64(const uint64_t* p) {
  return __ldcv(reinterpret_cast<const unsigned long long*>(p));
}
__device__ __forceinline__ uint4 ld_cv_v4(const uint4* p) { return __ldcv(p); }
__device__ __forceinline__ ulonglong2 ld_cv_v2u64(const ulonglong2* p) { return __ldcv(p); }
#endif

// n ops' worth of one arena array into dst, thread t of nt.  Loads are 16
// bytes wide where the source is 16-byte aligned, so a warp's loads cross
// PCIe as 512-byte requests; the ragged ends take scalar loads, so nothing
// outside [src, src + n) is read.  (One 1-, 8- and 8-byte load per op per
// thread moved 10-14 GB/s: 40 us of a 25k-op wave.)
__device__ __forceinline__ void gather_u64(const uint64_t* src, uint64_t* dst, uint32_t n,
                                           uint32_t t, uint32_t nt) {
  const uint32_t h = (((uintptr_t)src & 15u) != 0 && n != 0) ? 1u : 0u;  // to 16-B alignment
  const uint32_t pairs = (n - h) / 2;
  const ulonglong2* s2 = reinterpret_cast<const ulonglong2*>(src + h);
  for (uint32_t p = t; p < pairs; p += nt) {
    const ulonglong2 v = ld_cv_v2u64(s2 + p);
    dst[h + 2 * p] = v.x;
    dst[h + 2 * p + 1] = v.y;
  }
  if (h && t == 0) dst[0] = ld_cv_u64(src);
  if (((n - h) & 1u) && t == nt - 1) dst[n - 1] = ld_cv_u64(src + n - 1);
}

__device__ __forceinline__ void gather_u8(const uint8_t* src, uint8_t* dst, uint32_t n, uint32_t t,
                                          uint32_t nt) {
  const uint32_t h = min(n, (uint32_t)((16u - ((uintptr_t)src & 15u)) & 15u));
  const uint32_t chunks = (n - h) / 16;
  const uint4* s4 = reinterpret_cast<const uint4*>(src + h);
  for (uint32_t c = t; c < chunks; c += nt) {
    const uint4 v = ld_cv_v4(s4 + c);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    uint8_t* d = dst + h + 16 * c;
#pragma unroll
    for (int q = 0; q < 16; ++q) d[q] = (uint8_t)(w[q >> 2] >> (8 * (q & 3)));
  }
  for (uint32_t i = t; i < h; i += nt) dst[i] = ld_cv_u8(src + i);
  for (uint32_t i = h + 16 * chunks + t; i < n; i += nt) dst[i] = ld_cv_u8(src + i);
}

}  // namespace lsb
