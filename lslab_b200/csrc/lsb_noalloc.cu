// lsb_map_size_noalloc: count a map's live entries without allocating.
//
// lsb_map_size allocates an 8-byte device accumulator with cudaMalloc on every
// call and synchronises the stream.  Some callers cannot do either: code that
// is recording a CUDA stream capture (cudaMalloc is a potentially
// synchronising call and is refused in global capture mode), and services that
// hand the library a fixed, fully pre-reserved memory budget and forbid
// further device allocation.  This entry point serves them: its only scratch
// is the file-scope device array below, it writes the count into a device
// word the caller provides, and it enqueues work on the caller's stream
// without waiting for it.
//
// Limits and sharing:
//  * one partial sum per block of 256 buckets lives in the scratch, so the
//    map may have at most kNoAllocMaxBlocks * 256 = 2^20 buckets; larger maps
//    are refused with LSB_ERR_ARG before anything is enqueued;
//  * every GPU that loads the library holds the array (32 KB + 256 B) until
//    the process exits;
//  * all calls share the one array, and it keeps the last call's contents:
//    the completion counter is cleared on the stream at the start of every
//    call; calls that overlap on the GPU (different streams, no ordering)
//    race on the array and give wrong counts;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, that device current); make that
//    first call before starting any stream capture.  The address is cached
//    for the life of the process: after cudaDeviceReset (or anything else
//    that tears down the device's primary context) the library must not be
//    used again on that device;
//  * the call runs on the current device, which must be the map's own: a map
//    created on another device is refused with LSB_ERR_ARG (the call neither
//    switches devices nor reads another GPU's memory).
#include <cuda_runtime.h>

#include <mutex>

#include "lsb.h"
#include "lsb_internal.h"

using namespace lsb;

namespace {

constexpr uint32_t kNoAllocMaxBlocks = 4096;
constexpr uint32_t kNoAllocBlock = 256;
// [0, kNoAllocMaxBlocks): per-block partial counts; [kNoAllocMaxBlocks]: the
// count of blocks that have finished (must start at zero each call).
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocMaxBlocks + 32];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned long long* g_scratch_ptr[kMaxDevices] = {};

__global__ void __launch_bounds__(kNoAllocBlock)
    k_count_noalloc(TableView t, uint32_t buckets, unsigned long long* scratch,
                    unsigned long long* out) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long c = 0;
  if (b < buckets) {
    uint32_t s = b;
    for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
      const Meta m = load_meta(slab_ptr((const uint8_t*)t.slabs, s, MapTraits::kSlabBytes));
#pragma unroll
      for (int w = 0; w < 7; ++w)  // live tags: top bit set, not the busy marker 0x80
        c += __popc(m.tag[w] & 0x80808080u) -
             __popc(__vcmpeq4(m.tag[w], 0x80808080u) & 0x80808080u);
      if (m.next == 0) break;
      s = m.next;
    }
  }
  c = __reduce_add_sync(0xFFFFFFFFu, (unsigned)c);
  __shared__ unsigned long long warp_sum[kNoAllocBlock / 32];
  __shared__ bool last;
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long total = 0;
    for (uint32_t w = 0; w < kNoAllocBlock / 32; ++w) total += warp_sum[w];
    scratch[blockIdx.x] = total;
    __threadfence();
    const unsigned long long done = atomicAdd(&scratch[kNoAllocMaxBlocks], 1ull);
    last = done + 1 == gridDim.x;
  }
  __syncthreads();
  if (!last) return;
  // the last block to finish sums every partial
  __threadfence();
  unsigned long long sum = 0;
  for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) sum += ld_cg_u64(&scratch[i]);
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) sum += __shfl_down_sync(0xFFFFFFFFu, sum, d);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long total = 0;
    for (uint32_t w = 0; w < kNoAllocBlock / 32; ++w) total += warp_sum[w];
    *out = total;
  }
}

// Device address of the scratch array on the current device (looked up on the
// first call per device).
int scratch_for_current_device(unsigned long long** ptr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return LSB_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr)
      return LSB_ERR_CUDA;
    g_scratch_ptr[dev] = static_cast<unsigned long long*>(p);
  }
  *ptr = g_scratch_ptr[dev];
  return LSB_OK;
}

}  // namespace

extern "C" int lsb_map_size_noalloc(lsb_map* m, uint64_t* count_out, cudaStream_t stream) {
  if (!m || !count_out || ((uintptr_t)count_out & 7u)) return LSB_ERR_ARG;
  TableView view;
  uint32_t buckets = 0;
  lsb_internal_map_view(m, &view, &buckets);
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return LSB_ERR_CUDA;
  if (dev != lsb_internal_map_device(m)) return LSB_ERR_ARG;
  const uint32_t blocks = (buckets + kNoAllocBlock - 1) / kNoAllocBlock;
  if (blocks == 0 || blocks > kNoAllocMaxBlocks) return LSB_ERR_ARG;  // over 2^20 buckets
  unsigned long long* scratch = nullptr;
  int e = scratch_for_current_device(&scratch);
  if (e != LSB_OK) return e;
  if (cudaMemsetAsync(scratch + kNoAllocMaxBlocks, 0, sizeof(unsigned long long), stream) !=
      cudaSuccess)
    return LSB_ERR_CUDA;
  k_count_noalloc<<<blocks, kNoAllocBlock, 0, stream>>>(
      view, buckets, scratch, reinterpret_cast<unsigned long long*>(count_out));
  return cudaGetLastError() == cudaSuccess ? LSB_OK : LSB_ERR_CUDA;
}
