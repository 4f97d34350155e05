// Test kernels for the per-warp device API (include/lsb_device.cuh), built
// by tests/test_device_api_gpu.py into a shared library and called through
// ctypes.  Each thread carries one op; ops are grouped 32 to a warp in index
// order.  one_warp: a single warp walks all ops 32 at a time (the sequential
// case: lane order within a group, groups in order); otherwise every warp
// takes its own group at once.
#include <cuda_runtime.h>

#include "lsb_device.cuh"

namespace {

__global__ void k_map_ops(lsb_table_view v, const uint8_t* types, const uint64_t* keys,
                          const uint64_t* vals, lsb_result* out, uint32_t n, int one_warp) {
  const lsb_dev::map_ref m(v);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = one_warp ? 1u : (gridDim.x * blockDim.x) >> 5;
  if (one_warp && warp != 0) return;
  for (uint32_t base = warp * 32; base < n; base += nwarps * 32) {  // warp-uniform
    const uint32_t i = base + lane;
    const bool active = i < n;
    const uint8_t ty = active ? types[i] : 0;
    const uint64_t key = active ? keys[i] : 0;
    const uint64_t val = active ? vals[i] : 0;
    lsb_result r{};
    // every lane calls each method; thread_mask selects the op type
    uint64_t got = 0;
    const bool found = m.get(key, got, active && ty == LSB_OP_GET);
    const uint64_t old = m.put(key, val, active && ty == LSB_OP_PUT);
    const lsb_result up = m.update(key, val, active && ty == LSB_OP_UPDATE);
    const lsb_result rm = m.remove(key, active && ty == LSB_OP_REMOVE);
    if (!active) continue;
    if (ty == LSB_OP_GET) {
      r.found = found;
      r.value = found ? got : 0;
    } else if (ty == LSB_OP_PUT) {
      r.found = 0;  // put reports the old value only (map.h:136-152)
      r.value = old;
    } else if (ty == LSB_OP_UPDATE) {
      r = up;
    } else {
      r = rm;
    }
    out[i] = r;
  }
}

__global__ void k_set_ops(lsb_table_view v, const uint8_t* types, const uint32_t* keys,
                          uint8_t* out, uint32_t n, int one_warp) {
  const lsb_dev::set_ref s(v);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = one_warp ? 1u : (gridDim.x * blockDim.x) >> 5;
  if (one_warp && warp != 0) return;
  for (uint32_t base = warp * 32; base < n; base += nwarps * 32) {
    const uint32_t i = base + lane;
    const bool active = i < n;
    const uint8_t ty = active ? types[i] : 0;
    const uint32_t key = active ? keys[i] : 0;
    const bool c = s.contains(key, active && ty == LSB_OP_CONTAINS);
    const bool a = s.insert(key, active && ty == LSB_OP_INSERT);
    const bool d = s.remove(key, active && ty == LSB_OP_REMOVE);
    if (active) out[i] = ty == LSB_OP_CONTAINS ? c : ty == LSB_OP_INSERT ? a : d;
  }
}

}  // namespace

extern "C" int dev_map_ops(const lsb_map* m, const uint8_t* types, const uint64_t* keys,
                           const uint64_t* vals, lsb_result* out, uint32_t n, int one_warp,
                           cudaStream_t s) {
  lsb_table_view v;
  if (lsb_map_device_view(m, &v) != LSB_OK) return 1;
  const uint32_t blocks = one_warp ? 1u : (n + 255) / 256;
  k_map_ops<<<blocks, one_warp ? 32 : 256, 0, s>>>(v, types, keys, vals, out, n, one_warp);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" int dev_set_ops(const lsb_set* st, const uint8_t* types, const uint32_t* keys,
                           uint8_t* out, uint32_t n, int one_warp, cudaStream_t s) {
  lsb_table_view v;
  if (lsb_set_device_view(st, &v) != LSB_OK) return 1;
  const uint32_t blocks = one_warp ? 1u : (n + 255) / 256;
  k_set_ops<<<blocks, one_warp ? 32 : 256, 0, s>>>(v, types, keys, out, n, one_warp);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
