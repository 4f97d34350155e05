// CPU check of the serving loop's gather (lsb_gather.cuh), compiled for the
// host (test infrastructure).  For every source alignment, op count and
// number of threads, the threads of the gather together must copy
// [src, src + n) exactly once into dst, write nothing past dst[n - 1], read
// nothing outside [src, src + n), and issue their 16-byte loads only at
// 16-byte-aligned addresses.  Prints "ok" and returns 0, or names the case.
#include "simt_host.h"
#include "lsb_gather.cuh"

#include <cstdio>
#include <vector>

namespace {
const uint8_t* g_lo = nullptr;
const uint8_t* g_hi = nullptr;
bool g_bad = false;

void check_read(const void* p, size_t bytes) {
  const uint8_t* b = static_cast<const uint8_t*>(p);
  if (b < g_lo || b + bytes > g_hi) g_bad = true;
  if (bytes == 16 && (reinterpret_cast<uintptr_t>(b) & 15u) != 0) g_bad = true;
}
}  // namespace

int main() {
  lsb::emu_read_hook = check_read;
  alignas(64) static uint8_t buf8[512];
  alignas(64) static uint64_t buf64[256];
  for (size_t i = 0; i < sizeof(buf8); ++i) buf8[i] = (uint8_t)(i * 37 + 11);
  for (size_t i = 0; i < 256; ++i) buf64[i] = 0x9E3779B97F4A7C15ull * (i + 1);
  const uint32_t nts[] = {1, 2, 3, 5, 32, 151};
  for (uint32_t nt : nts) {
    for (uint32_t off = 0; off < 32; ++off) {
      for (uint32_t n = 0; n <= 200; ++n) {
        // bytes: src at any byte offset
        const uint8_t* src = buf8 + 64 + off;
        std::vector<uint8_t> dst(n + 1, 0xEE);
        g_lo = src;
        g_hi = src + n;
        g_bad = false;
        for (uint32_t t = 0; t < nt; ++t) lsb::gather_u8(src, dst.data(), n, t, nt);
        for (uint32_t i = 0; i < n; ++i)
          if (dst[i] != src[i]) g_bad = true;
        if (dst[n] != 0xEE || g_bad) {
          std::printf("gather_u8 nt=%u off=%u n=%u\n", nt, off, n);
          return 1;
        }
        // 8-byte elements: src 8-byte aligned, 16-byte aligned or not
        if (off >= 2) continue;
        const uint64_t* s64 = buf64 + 8 + off;
        std::vector<uint64_t> d64(n + 1, 0xEEEEEEEEEEEEEEEEull);
        g_lo = reinterpret_cast<const uint8_t*>(s64);
        g_hi = reinterpret_cast<const uint8_t*>(s64 + n);
        g_bad = false;
        for (uint32_t t = 0; t < nt; ++t) lsb::gather_u64(s64, d64.data(), n, t, nt);
        for (uint32_t i = 0; i < n; ++i)
          if (d64[i] != s64[i]) g_bad = true;
        if (d64[n] != 0xEEEEEEEEEEEEEEEEull || g_bad) {
          std::printf("gather_u64 nt=%u off=%u n=%u\n", nt, off, n);
          return 1;
        }
      }
    }
  }
  std::printf("ok\n");
  return 0;
}
