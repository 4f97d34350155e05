// KV store: variable-size byte values over the map, the way a key-value
// store uses a slab hash (the reference's KVCG tests keep pointers to values
// in the map, test/slabunified_test.cu:360-380).  Values live in one device
// byte heap; the map holds key -> handle, handle = heap offset << 24 | length
// (offsets below 2^40, values of at most 2^24 - 1 bytes).
//
//   put     the batch's values arrive packed in one device buffer with n + 1
//           offsets (op i's bytes are vals[off[i] .. off[i+1])); they are
//           copied to the heap in one piece, each op gets its handle, and the
//           map takes the handles as a put batch (ops in index order, so the
//           last put of a key wins).  Space of replaced values becomes
//           garbage until lsb_kvs_compact.
//   get     handles by a read batch; lengths out; then the bytes of the found
//           values are copied to the caller's buffer at offsets that are the
//           exclusive prefix sums of the lengths (computed on the device).
//   remove  a map remove; the value's space becomes garbage.
//
// No counterpart in the reference's library itself (lslab maps fixed-size
// values only).
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "lsb.h"
#include "lsb_core.cuh"

namespace {

constexpr uint64_t kLenBits = 24;
constexpr uint64_t kMaxLen = (1ull << kLenBits) - 1;
constexpr uint64_t kMaxHeap = 1ull << 40;

__device__ __forceinline__ uint32_t h_len(uint64_t h) { return (uint32_t)(h & kMaxLen); }
__device__ __forceinline__ uint64_t h_off(uint64_t h) { return h >> kLenBits; }

// handle[i] = (base + off[i] - off[0]) << 24 | (off[i+1] - off[i]); a length
// over the limit raises *bad.
__global__ void k_handles(const uint64_t* off, uint64_t base, uint64_t* handle, uint32_t n,
                          uint32_t* bad) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t a = off[i], b = off[i + 1];
  if (b < a || b - a > kMaxLen) {
    atomicOr(bad, 1u);
    handle[i] = 0;
    return;
  }
  handle[i] = ((base + a - off[0]) << kLenBits) | (b - a);
}

// Garbage accounting: bytes of the values that a put or remove replaced.
__global__ void k_dead_bytes(const lsb_result* res, const uint64_t* old, uint32_t n,
                             unsigned long long* dead) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t v = 0;
  if (i < n) {
    if (res) v = res[i].found ? h_len(res[i].value) : 0;
    else v = h_len(old[i]);  // a put's old handle (0 when the key was absent)
  }
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, d);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(dead, (unsigned long long)v);
}

// Lengths of the looked-up values (0 when absent) and their exclusive prefix
// sums: one block, chunks of the ops per thread.
__global__ void __launch_bounds__(1024) k_lengths_scan(const lsb_result* res, uint32_t n,
                                                       uint32_t* len, uint64_t* dst_off,
                                                       uint8_t* found, uint64_t* total) {
  __shared__ unsigned long long part[1024];
  const uint32_t per = (n + blockDim.x - 1) / blockDim.x, j0 = threadIdx.x * per;
  unsigned long long s = 0;
  for (uint32_t k = 0; k < per; ++k) {
    const uint32_t j = j0 + k;
    if (j < n) s += res[j].found ? h_len(res[j].value) : 0;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (uint32_t d = 1; d < blockDim.x; d <<= 1) {  // inclusive scan of the parts
    const unsigned long long y = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
    __syncthreads();
    part[threadIdx.x] += y;
    __syncthreads();
  }
  unsigned long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (uint32_t k = 0; k < per; ++k) {
    const uint32_t j = j0 + k;
    if (j < n) {
      const uint32_t l = res[j].found ? h_len(res[j].value) : 0;
      len[j] = l;
      dst_off[j] = run;
      if (found) found[j] = res[j].found;
      run += l;
    }
  }
  if (threadIdx.x == blockDim.x - 1) *total = part[blockDim.x - 1];
}

// Copy each found value's bytes from the heap to dst + dst_off[i] (one warp
// per op, bytes striped over the lanes); values that would end past cap are
// skipped.
__global__ void k_gather(const lsb_result* res, const uint64_t* dst_off, const uint8_t* heap,
                         uint8_t* dst, uint64_t cap, uint32_t n) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
  if (w >= n || !res[w].found) return;
  const uint64_t h = res[w].value, o = dst_off[w];
  const uint32_t l = h_len(h);
  if (o + l > cap) return;
  const uint8_t* src = heap + h_off(h);
  for (uint32_t b = lane; b < l; b += 32) dst[o + b] = src[b];
}

// Heap compaction's move: value i (handle h[i]) to stage + dst_off[i]; one
// warp per value.
__global__ void k_move(const uint64_t* h, const uint64_t* dst_off, const uint8_t* heap,
                       uint8_t* stage, uint32_t n) {
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
  if (w >= n) return;
  const uint8_t* src = heap + h_off(h[w]);
  uint8_t* dst = stage + dst_off[w];
  for (uint32_t b = lane; b < h_len(h[w]); b += 32) dst[b] = src[b];
}

}  // namespace

struct lsb_kvs {
  lsb_map* map = nullptr;
  uint8_t* heap = nullptr;
  uint64_t heap_cap = 0;
  uint64_t heap_used = 0;      // bump cursor (host-side: every allocation goes through put)
  unsigned long long* dead = nullptr;  // device: bytes of replaced values
  uint32_t* bad = nullptr;     // device: a length over the limit
  uint64_t* tmp = nullptr;     // device scratch: handles / old handles / offsets
  lsb_result* res = nullptr;   // device scratch: lookup results
  uint32_t tmp_cap = 0;
};

namespace {

int ensure_tmp(lsb_kvs* s, size_t n) {
  if (n <= s->tmp_cap) return LSB_OK;
  cudaFree(s->tmp);
  cudaFree(s->res);
  s->tmp = nullptr;
  s->res = nullptr;
  s->tmp_cap = 0;
  if (cudaMalloc(&s->tmp, sizeof(uint64_t) * 2 * (n + 1)) != cudaSuccess ||
      cudaMalloc(&s->res, sizeof(lsb_result) * n) != cudaSuccess) {
    cudaGetLastError();
    return LSB_ERR_OOM;
  }
  s->tmp_cap = (uint32_t)n;
  return LSB_OK;
}

}  // namespace

extern "C" {

int lsb_kvs_create(unsigned log2_buckets, uint64_t heap_bytes, const lsb_options* opt,
                   lsb_kvs** out) {
  if (!out || heap_bytes == 0 || heap_bytes > kMaxHeap) return LSB_ERR_ARG;
  *out = nullptr;
  lsb_kvs* s = new (std::nothrow) lsb_kvs();
  if (!s) return LSB_ERR_OOM;
  lsb_options o{};
  if (opt) {
    o = *opt;
  } else {
    o.device = -1;
  }
  int rc = lsb_map_create_ex(log2_buckets, &o, &s->map);
  if (rc == LSB_OK &&
      (cudaMalloc(&s->heap, heap_bytes) != cudaSuccess ||
       cudaMalloc(&s->dead, sizeof(unsigned long long)) != cudaSuccess ||
       cudaMalloc(&s->bad, sizeof(uint32_t)) != cudaSuccess ||
       cudaMemset(s->dead, 0, sizeof(unsigned long long)) != cudaSuccess ||
       cudaMemset(s->bad, 0, sizeof(uint32_t)) != cudaSuccess)) {
    cudaGetLastError();
    rc = LSB_ERR_OOM;
  }
  if (rc != LSB_OK) {
    lsb_kvs_destroy(s);
    return rc;
  }
  s->heap_cap = heap_bytes;
  *out = s;
  return LSB_OK;
}

int lsb_kvs_destroy(lsb_kvs* s) {
  if (!s) return LSB_ERR_ARG;
  if (s->map) lsb_map_destroy(s->map);
  cudaFree(s->heap);
  cudaFree(s->dead);
  cudaFree(s->bad);
  cudaFree(s->tmp);
  cudaFree(s->res);
  delete s;
  return LSB_OK;
}

lsb_map* lsb_kvs_map(lsb_kvs* s) { return s ? s->map : nullptr; }

int lsb_kvs_put(lsb_kvs* s, const uint64_t* keys, const uint8_t* vals, const uint64_t* val_off,
                size_t n, cudaStream_t stream) {
  if (!s || (n && (!keys || !val_off))) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  if (n > 0xFFFFFFFFull) return LSB_ERR_ARG;
  uint64_t ends[2];
  if (cudaMemcpyAsync(&ends[0], val_off, 8, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(&ends[1], val_off + n, 8, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return LSB_ERR_CUDA;
  if (ends[1] < ends[0]) return LSB_ERR_ARG;
  const uint64_t bytes = ends[1] - ends[0];
  if (bytes && !vals) return LSB_ERR_ARG;
  if (bytes > s->heap_cap - s->heap_used) return LSB_ERR_OOM;  // no effect
  int rc = ensure_tmp(s, n);
  if (rc) return rc;
  const uint64_t base = s->heap_used;
  if (bytes && cudaMemcpyAsync(s->heap + base, vals + ends[0], bytes, cudaMemcpyDeviceToDevice,
                               stream) != cudaSuccess)
    return LSB_ERR_CUDA;
  uint64_t* handle = s->tmp;
  uint64_t* old = s->tmp + (n + 1);
  k_handles<<<(uint32_t)((n + 255) / 256), 256, 0, stream>>>(val_off, base, handle, (uint32_t)n,
                                                             s->bad);
  uint32_t bad = 0;
  if (cudaMemcpyAsync(&bad, s->bad, 4, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return LSB_ERR_CUDA;
  if (bad) {
    cudaMemsetAsync(s->bad, 0, 4, stream);
    return LSB_ERR_ARG;  // a value longer than 2^24 - 1 bytes: nothing stored
  }
  rc = lsb_map_put(s->map, keys, handle, old, n, stream);
  if (rc) return rc;
  k_dead_bytes<<<(uint32_t)((n + 255) / 256), 256, 0, stream>>>(nullptr, old, (uint32_t)n,
                                                                s->dead);
  s->heap_used += bytes;
  return cudaGetLastError() == cudaSuccess ? LSB_OK : LSB_ERR_CUDA;
}

int lsb_kvs_get(lsb_kvs* s, const uint64_t* keys, uint8_t* found_out, uint32_t* len_out,
                uint64_t* dst_off_out, uint8_t* dst, uint64_t dst_cap, size_t n,
                uint64_t* total_out, cudaStream_t stream) {
  if (!s || (n && (!keys || !len_out || !dst_off_out))) return LSB_ERR_ARG;
  if (n == 0) {
    if (total_out) *total_out = 0;
    return LSB_OK;
  }
  if (n > 0xFFFFFFFFull) return LSB_ERR_ARG;
  int rc = ensure_tmp(s, n);
  if (rc) return rc;
  rc = lsb_map_get(s->map, keys, s->res, n, stream);
  if (rc) return rc;
  uint64_t* total_d = s->tmp;
  k_lengths_scan<<<1, 1024, 0, stream>>>(s->res, (uint32_t)n, len_out, dst_off_out, found_out,
                                         total_d);
  if (dst && dst_cap) {
    const uint64_t threads = 32ull * n;
    k_gather<<<(uint32_t)((threads + 255) / 256), 256, 0, stream>>>(s->res, dst_off_out, s->heap,
                                                                   dst, dst_cap, (uint32_t)n);
  }
  if (total_out) {
    if (cudaMemcpyAsync(total_out, total_d, 8, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return LSB_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? LSB_OK : LSB_ERR_CUDA;
}

int lsb_kvs_remove(lsb_kvs* s, const uint64_t* keys, uint8_t* found_out, size_t n,
                   cudaStream_t stream) {
  if (!s || (n && !keys)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  if (n > 0xFFFFFFFFull) return LSB_ERR_ARG;
  int rc = ensure_tmp(s, n);
  if (rc) return rc;
  rc = lsb_map_remove(s->map, keys, s->res, n, stream);
  if (rc) return rc;
  k_dead_bytes<<<(uint32_t)((n + 255) / 256), 256, 0, stream>>>(s->res, nullptr, (uint32_t)n,
                                                                s->dead);
  if (found_out) {
    // found bytes are the first byte of each 16-byte result
    if (cudaMemcpy2DAsync(found_out, 1, s->res, sizeof(lsb_result), 1, n,
                          cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return LSB_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? LSB_OK : LSB_ERR_CUDA;
}

int lsb_kvs_usage(lsb_kvs* s, uint64_t* heap_used, uint64_t* heap_dead, uint64_t* heap_cap,
                  cudaStream_t stream) {
  if (!s) return LSB_ERR_ARG;
  unsigned long long dead = 0;
  if (cudaMemcpyAsync(&dead, s->dead, 8, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return LSB_ERR_CUDA;
  if (heap_used) *heap_used = s->heap_used;
  if (heap_dead) *heap_dead = dead;
  if (heap_cap) *heap_cap = s->heap_cap;
  return LSB_OK;
}

// Heap compaction: the live values move, in key order, to the front of the
// heap (through a staging copy), the map takes their new handles, and the
// garbage count restarts at zero.  Synchronises the stream.
int lsb_kvs_compact(lsb_kvs* s, cudaStream_t stream) {
  if (!s) return LSB_ERR_ARG;
  uint64_t n = 0;
  int rc = lsb_map_size(s->map, &n, stream);
  if (rc) return rc;
  std::vector<uint64_t> k(n), h(n), newh(n), off(n + 1, 0);
  uint64_t got = 0;
  rc = lsb_map_dump(s->map, k.data(), h.data(), n, &got, stream);
  if (rc) return rc;
  if (got != n) return LSB_ERR_STATE;
  for (uint64_t i = 0; i < n; ++i) {
    off[i + 1] = off[i] + (h[i] & kMaxLen);
    newh[i] = (off[i] << kLenBits) | (h[i] & kMaxLen);
  }
  const uint64_t live = off[n];
  uint8_t* stage = nullptr;
  uint64_t *d_keys = nullptr, *d_handles = nullptr, *d_old = nullptr, *d_off = nullptr;
  if ((live && cudaMalloc(&stage, live) != cudaSuccess) ||
      (n && (cudaMalloc(&d_keys, 8 * n) != cudaSuccess ||
             cudaMalloc(&d_handles, 8 * n) != cudaSuccess ||
             cudaMalloc(&d_old, 8 * n) != cudaSuccess ||
             cudaMalloc(&d_off, 8 * n) != cudaSuccess))) {
    cudaGetLastError();
    cudaFree(stage);
    cudaFree(d_keys);
    cudaFree(d_handles);
    cudaFree(d_old);
    cudaFree(d_off);
    return LSB_ERR_OOM;
  }
  // live values into the staging buffer in key order, then back to the front
  if (n &&
      (cudaMemcpyAsync(d_old, h.data(), 8 * n, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
       cudaMemcpyAsync(d_off, off.data(), 8 * n, cudaMemcpyHostToDevice, stream) != cudaSuccess))
    rc = LSB_ERR_CUDA;
  if (rc == LSB_OK && n)
    k_move<<<(uint32_t)((32ull * n + 255) / 256), 256, 0, stream>>>(d_old, d_off, s->heap, stage,
                                                                    (uint32_t)n);
  if (rc == LSB_OK && live &&
      cudaMemcpyAsync(s->heap, stage, live, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
    rc = LSB_ERR_CUDA;
  if (rc == LSB_OK && n &&
      (cudaMemcpyAsync(d_keys, k.data(), 8 * n, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
       cudaMemcpyAsync(d_handles, newh.data(), 8 * n, cudaMemcpyHostToDevice, stream) !=
           cudaSuccess))
    rc = LSB_ERR_CUDA;
  if (rc == LSB_OK && n) rc = lsb_map_put(s->map, d_keys, d_handles, nullptr, n, stream);
  if (rc == LSB_OK && cudaMemsetAsync(s->dead, 0, 8, stream) != cudaSuccess) rc = LSB_ERR_CUDA;
  if (rc == LSB_OK && cudaStreamSynchronize(stream) != cudaSuccess) rc = LSB_ERR_CUDA;
  cudaFree(stage);
  cudaFree(d_keys);
  cudaFree(d_handles);
  cudaFree(d_old);
  cudaFree(d_off);
  if (rc == LSB_OK) s->heap_used = live;
  return rc;
}

}  // extern "C"
