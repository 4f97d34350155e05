// Host versions of the library's load/store helpers for the block emulation
// in simt_host.h (test infrastructure).  Every access is an atomic, so
// concurrently running emulated threads have defined behaviour; cache hints
// have no host meaning.  Included inside the library's namespace.
#pragma once

namespace emu_detail {
template <class T>
inline T ld(const void* p) {
  return __atomic_load_n(reinterpret_cast<const T*>(p), __ATOMIC_RELAXED);
}
template <class T>
inline void st(void* p, T v) {
  __atomic_store_n(reinterpret_cast<T*>(p), v, __ATOMIC_RELAXED);
}
}  // namespace emu_detail

inline uint4 ld_cg_v4(const void* p) {
  const uint32_t* q = static_cast<const uint32_t*>(p);
  return uint4{emu_detail::ld<uint32_t>(q), emu_detail::ld<uint32_t>(q + 1),
               emu_detail::ld<uint32_t>(q + 2), emu_detail::ld<uint32_t>(q + 3)};
}
inline ulonglong2 ld_cg_v2u64(const void* p) {
  const unsigned long long* q = static_cast<const unsigned long long*>(p);
  return ulonglong2{emu_detail::ld<unsigned long long>(q), emu_detail::ld<unsigned long long>(q + 1)};
}
inline uint32_t ld_cg_u32(const void* p) { return emu_detail::ld<uint32_t>(p); }
inline uint64_t ld_cg_u64(const void* p) { return emu_detail::ld<uint64_t>(p); }
inline uint64_t l2_keep() { return 0; }
inline uint4 ld_ca_v4(const void* p) { return ld_cg_v4(p); }
inline ulonglong2 ld_ca_v2u64(const void* p) { return ld_cg_v2u64(p); }
inline uint32_t ld_ca_u32(const void* p) { return ld_cg_u32(p); }
// Volatile loads of the serving gather (lsb_gather.cuh).  A test may set
// emu_read_hook to see every address and width they read.
inline void (*emu_read_hook)(const void* p, size_t bytes) = nullptr;
inline uint8_t ld_cv_u8(const uint8_t* p) {
  if (emu_read_hook) emu_read_hook(p, 1);
  return emu_detail::ld<uint8_t>(p);
}
inline uint64_t ld_cv_u64(const uint64_t* p) {
  if (emu_read_hook) emu_read_hook(p, 8);
  return emu_detail::ld<uint64_t>(p);
}
inline uint4 ld_cv_v4(const uint4* p) {
  if (emu_read_hook) emu_read_hook(p, 16);
  return ld_cg_v4(p);
}
inline ulonglong2 ld_cv_v2u64(const ulonglong2* p) {
  if (emu_read_hook) emu_read_hook(p, 16);
  return ld_cg_v2u64(p);
}
inline uint64_t ld_cs_u64(const void* p) { return emu_detail::ld<uint64_t>(p); }
inline uint32_t ld_cs_u32(const void* p) { return emu_detail::ld<uint32_t>(p); }
inline uint8_t ld_cs_u8(const void* p) { return emu_detail::ld<uint8_t>(p); }
inline void st_cs_u64(void* p, uint64_t v) { emu_detail::st<uint64_t>(p, v); }
inline void st_cs_u32(void* p, uint32_t v) { emu_detail::st<uint32_t>(p, v); }
inline void st_cs_u8(void* p, uint8_t v) { emu_detail::st<uint8_t>(p, v); }
inline uint32_t ld_acquire_u32(const uint32_t* p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }
inline void st_release_u32(uint32_t* p, uint32_t v) { __atomic_store_n(p, v, __ATOMIC_RELEASE); }
inline uint64_t ld_relaxed_u64(const uint64_t* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline void st_cg_u8(void* p, uint8_t v) { emu_detail::st<uint8_t>(p, v); }
inline void st_cg_u32(void* p, uint32_t v) { emu_detail::st<uint32_t>(p, v); }
inline void st_cg_u64(void* p, uint64_t v) { emu_detail::st<uint64_t>(p, v); }
inline void st_cg_v2u64(void* p, uint64_t a, uint64_t b) {
  emu_detail::st<uint64_t>(p, a);
  emu_detail::st<uint64_t>(static_cast<uint64_t*>(p) + 1, b);
}
inline uint32_t atom_add_acq_rel(uint32_t* p, uint32_t v) {
  return __atomic_fetch_add(p, v, __ATOMIC_ACQ_REL);
}
inline uint32_t sm_id() { return blockIdx.x; }
