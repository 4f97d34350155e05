// Host side of the library: table objects, kernel launches, the C-ABI of
// include/lsb.h.  Every batched entry point is asynchronous on the caller's
// stream; argument errors are returned, device errors land in the table's
// status word.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "lsb.h"
#include "lsb_core.cuh"
#include "lsb_window.cuh"

using namespace lsb;

namespace {

constexpr uint32_t kDefaultWindow = 1u << 20;
constexpr uint32_t kMaxWindow = 1u << 23;  // owner field of a group slot is 24 bits
constexpr int kPlainBlock = 256;
constexpr int kFusedBlock = 512;

// Device arrays must be naturally aligned for their element type; a
// misaligned device access would fault the context, so it is refused here.
inline bool aligned(const void* p, size_t a) { return ((uintptr_t)p & (a - 1)) == 0; }

#define LSB_CK(call)                         \
  do {                                       \
    cudaError_t e_ = (call);                 \
    if (e_ != cudaSuccess) return LSB_ERR_CUDA; \
  } while (0)

// ------------------------------------------------------------- kernels
template <class Tr, bool kGroup, bool kDedup>
__global__ void __launch_bounds__(kPlainBlock) k_probe(TableView t, Scratch sc, Window<Tr> w) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  phase_probe<Tr, kGroup, kDedup>(t, sc, w, warp, nwarps);
}

template <class Tr>
__global__ void __launch_bounds__(kPlainBlock) k_segments(Scratch sc, Window<Tr> w) {
  phase_segments<Tr>(sc, w, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <class Tr>
__global__ void __launch_bounds__(kPlainBlock) k_scatter(Scratch sc, Window<Tr> w) {
  phase_scatter<Tr>(sc, w, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <class Tr>
__global__ void __launch_bounds__(kPlainBlock) k_sort(Scratch sc, Window<Tr> w) {
  extern __shared__ uint32_t smem[];
  phase_sort_small<Tr>(sc, w, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
  phase_sort_big<Tr>(sc, w, smem);
}

template <class Tr>
__global__ void __launch_bounds__(kPlainBlock) k_resolve(TableView t, Scratch sc, Window<Tr> w) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  phase_resolve_mutations<Tr>(t, sc, w, tid, nt);
  phase_resolve_reads<Tr>(sc, w, tid, nt);
}

// One batch split into windows, all phases of all windows in one cooperative
// launch with bounded grid barriers between phases.
template <class Tr>
struct FusedJob {
  Window<Tr> base;  // whole batch; n = total ops
  uint32_t window;  // ops per window
  uint32_t epoch0;  // epoch of the first window
};

template <class Tr>
__global__ void __launch_bounds__(kFusedBlock, 2)
    k_fused(TableView t, Scratch sc, FusedJob<Tr> job, GridBarrier* bar) {
  extern __shared__ uint32_t smem[];
  const uint32_t nblocks = gridDim.x;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  const uint32_t warp = tid >> 5, nwarps = nt >> 5;
  const uint32_t nwin = (job.base.n + job.window - 1) / job.window;
  for (uint32_t wi = 0; wi < nwin; ++wi) {
    Window<Tr> w = job.base;
    const uint32_t start = wi * job.window;
    w.n = min(job.window, job.base.n - start);
    if (w.types) w.types += start;
    w.keys += (size_t)start * w.kstride;
    if (w.vals) w.vals += (size_t)start * w.vstride;
    if (w.out) {
      size_t esz = w.out_kind == kOutResult ? 16 : (w.out_kind == kOutOld ? 8 : 1);
      w.out = (uint8_t*)w.out + (size_t)start * esz;
    }
    w.epoch = job.epoch0 + wi;
    w.cnt = &sc.cnt[wi & 1];
    if (tid == 0) win_counters_reset(&sc.cnt[(wi + 1) & 1]);
    phase_probe<Tr, true, true>(t, sc, w, warp, nwarps);
    if (!grid_barrier(bar, nblocks, t.status)) return;
    phase_segments<Tr>(sc, w, tid, nt);
    if (!grid_barrier(bar, nblocks, t.status)) return;
    phase_scatter<Tr>(sc, w, tid, nt);
    if (!grid_barrier(bar, nblocks, t.status)) return;
    phase_sort_small<Tr>(sc, w, tid, nt);
    phase_sort_big<Tr>(sc, w, smem);
    if (!grid_barrier(bar, nblocks, t.status)) return;
    phase_resolve_mutations<Tr>(t, sc, w, tid, nt);
    phase_resolve_reads<Tr>(sc, w, tid, nt);
    if (!grid_barrier(bar, nblocks, t.status)) return;
  }
}

// Live-entry count and dump: one thread per bucket walks the chain.
template <class Tr>
__global__ void k_count(TableView t, uint32_t buckets, unsigned long long* count) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long c = 0;
  if (b < buckets) {
    uint32_t s = b;
    for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
      Meta m = load_meta(slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes));
#pragma unroll
      for (int w = 0; w < 7; ++w) c += __popc(m.tag[w] & 0x80808080u) -
                                       __popc(__vcmpeq4(m.tag[w], 0x80808080u) & 0x80808080u);
      if (m.next == 0) break;
      s = m.next;
    }
  }
  c = __reduce_add_sync(0xFFFFFFFFu, (unsigned)c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

template <class Tr>
__global__ void k_dump(TableView t, uint32_t buckets, typename Tr::Key* keys, uint64_t* vals,
                       unsigned long long* cursor, unsigned long long cap) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= buckets) return;
  uint32_t s = b;
  for (uint32_t hop = 0; hop < kMaxHops; ++hop) {
    const uint8_t* slab = slab_ptr((const uint8_t*)t.slabs, s, Tr::kSlabBytes);
    Meta m = load_meta(slab);
    for (int slot = 0; slot < kSlots; ++slot) {
      uint32_t tag = (m.tag[slot >> 2] >> (8 * (slot & 3))) & 0xFFu;
      if (tag <= 0x80u) continue;  // empty, dead or busy
      unsigned long long at = atomicAdd(cursor, 1ull);
      if (at >= cap) continue;
      const uint8_t* sp = slab + kMetaBytes + slot * Tr::kSlotBytes;
      if constexpr (Tr::kHasValue) {
        keys[at] = (typename Tr::Key)ld_cg_u64(sp);
        vals[at] = ld_cg_u64(sp + 8);
      } else {
        keys[at] = (typename Tr::Key)ld_cg_u32(sp);
      }
    }
    if (m.next == 0) break;
    s = m.next;
  }
}

// ------------------------------------------------------------- tables
template <class Tr>
struct Table {
  int device = 0;
  unsigned log2 = 0;
  uint32_t buckets = 0;
  uint64_t pool_slabs = 0;
  uint32_t lock_mode = kLockWriter;
  uint8_t* slabs = nullptr;
  int32_t* locks = nullptr;
  uint32_t* status = nullptr;
  uint64_t* pool = nullptr;
  GridBarrier* bar = nullptr;
  Scratch sc{};
  uint32_t epoch = 0;  // last epoch handed to a window
  uint32_t chunk = 1;  // per-SM pool refill size
  int num_sms = 0;
  int plain_grid = 0;
  int fused_grid = 0;
  bool dedup = true;

  TableView view() const {
    TableView v;
    v.slabs = slabs;
    v.locks = locks;
    v.status = status;
    v.pool = pool;
    v.mask = buckets - 1;
    v.lock_mode = lock_mode;
    v.chunk = chunk;
    return v;
  }

  void release() {
    cudaFree(slabs);
    cudaFree(locks);
    cudaFree(status);
    cudaFree(pool);
    cudaFree(bar);
    cudaFree(sc.gtab);
    cudaFree(sc.minfo);
    cudaFree(sc.pred);
    cudaFree(sc.goff);
    cudaFree(sc.seg);
    cudaFree(sc.sseg);
    cudaFree(sc.mlist);
    cudaFree(sc.big);
    cudaFree(sc.cnt);
  }

  int init(unsigned log2_buckets, const lsb_options* opt) {
    if (log2_buckets < 1 || log2_buckets > 30) return LSB_ERR_ARG;
    uint32_t window = opt && opt->max_window ? opt->max_window : kDefaultWindow;
    if (window > kMaxWindow) return LSB_ERR_ARG;
    if (opt && opt->lock_mode > kLockRW) return LSB_ERR_ARG;
    if (opt && opt->device >= 0) LSB_CK(cudaSetDevice(opt->device));
    LSB_CK(cudaGetDevice(&device));
    LSB_CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    log2 = log2_buckets;
    buckets = 1u << log2_buckets;
    pool_slabs = opt && opt->pool_slabs ? opt->pool_slabs : (uint64_t)buckets / 4 + 4096;
    if ((uint64_t)buckets + pool_slabs >= 0xFFFFFFFFull) return LSB_ERR_ARG;
    lock_mode = opt ? opt->lock_mode : kLockWriter;
    chunk = (uint32_t)std::min<uint64_t>(kPoolChunkMax,
                                         std::max<uint64_t>(1, pool_slabs / (8ull * num_sms)));

    const size_t slab_bytes = ((size_t)buckets + pool_slabs) * Tr::kSlabBytes;
    uint32_t g = 2;
    while (g < 2 * window) g <<= 1;
    sc.gmask = g - 1;
    sc.max_window = window;
    if (cudaMalloc(&slabs, slab_bytes) != cudaSuccess ||
        cudaMalloc(&locks, sizeof(int32_t) * buckets) != cudaSuccess ||
        cudaMalloc(&status, sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&pool, sizeof(uint64_t) * (2 + kPoolSlots)) != cudaSuccess ||
        cudaMalloc(&bar, sizeof(GridBarrier)) != cudaSuccess ||
        cudaMalloc(&sc.gtab, sizeof(uint64_t) * g) != cudaSuccess ||
        cudaMalloc(&sc.minfo, sizeof(uint64_t) * window) != cudaSuccess ||
        cudaMalloc(&sc.pred, sizeof(uint32_t) * window) != cudaSuccess ||
        cudaMalloc(&sc.goff, sizeof(uint32_t) * g) != cudaSuccess ||
        cudaMalloc(&sc.seg, sizeof(uint32_t) * window) != cudaSuccess ||
        cudaMalloc(&sc.sseg, sizeof(uint32_t) * window) != cudaSuccess ||
        cudaMalloc(&sc.mlist, sizeof(uint32_t) * window) != cudaSuccess ||
        cudaMalloc(&sc.big, sizeof(uint32_t) * (window / kSmallGroup + 1)) != cudaSuccess ||
        cudaMalloc(&sc.cnt, sizeof(WinCounters) * 2) != cudaSuccess) {
      cudaGetLastError();
      release();
      return LSB_ERR_OOM;
    }
    LSB_CK(cudaMemset(slabs, 0, slab_bytes));
    LSB_CK(cudaMemset(locks, 0, sizeof(int32_t) * buckets));
    LSB_CK(cudaMemset(status, 0, sizeof(uint32_t)));
    std::vector<uint64_t> p(2 + kPoolSlots, 0);
    p[0] = buckets;
    p[1] = (uint64_t)buckets + pool_slabs;
    LSB_CK(cudaMemcpy(pool, p.data(), sizeof(uint64_t) * p.size(), cudaMemcpyHostToDevice));
    LSB_CK(cudaMemset(bar, 0, sizeof(GridBarrier)));
    LSB_CK(cudaMemset(sc.gtab, 0, sizeof(uint64_t) * g));
    LSB_CK(cudaMemset(sc.cnt, 0, sizeof(WinCounters) * 2));

    plain_grid = num_sms * (2048 / kPlainBlock);
    LSB_CK(cudaFuncSetAttribute(k_sort<Tr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSortSmemBytes));
    LSB_CK(cudaFuncSetAttribute(k_fused<Tr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kSortSmemBytes));
    int per_sm = 0;
    LSB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<Tr>, kFusedBlock,
                                                         kSortSmemBytes));
    if (per_sm < 1) return LSB_ERR_STATE;
    fused_grid = per_sm * num_sms;
    return LSB_OK;
  }

  // Next epoch for a window; clears the group table when the 16-bit epoch wraps.
  int next_epochs(uint32_t count, cudaStream_t s, uint32_t* first) {
    if (epoch + count > 0xFFFFu) {
      LSB_CK(cudaMemsetAsync(sc.gtab, 0, sizeof(uint64_t) * (sc.gmask + 1ull), s));
      epoch = 0;
    }
    *first = epoch + 1;
    epoch += count;
    return LSB_OK;
  }

  Window<Tr> window(const uint8_t* types, uint8_t uniform, const typename Tr::Key* keys,
                    uint32_t kstride, const uint64_t* vals, uint32_t vstride, void* out,
                    uint32_t out_kind, uint32_t n) const {
    Window<Tr> w;
    w.types = types;
    w.uniform = uniform;
    w.keys = keys;
    w.kstride = kstride;
    w.vals = vals;
    w.vstride = vstride;
    w.out = out;
    w.out_kind = out ? out_kind : kOutNone;
    w.n = n;
    w.epoch = 0;
    w.cnt = sc.cnt;
    return w;
  }

  static size_t out_elem(uint32_t kind) {
    return kind == kOutResult ? 16 : (kind == kOutOld ? 8 : 1);
  }

  // Read-only batch: one probe launch, no scratch.
  int run_reads(const typename Tr::Key* keys, void* out, uint32_t out_kind, size_t n,
                cudaStream_t s) {
    for (size_t off = 0; off < n; off += (size_t)kMaxWindow) {
      uint32_t m = (uint32_t)std::min<size_t>(kMaxWindow, n - off);
      Window<Tr> w = window(nullptr, kOpRead, keys + off, 1, nullptr, 1,
                            out ? (uint8_t*)out + off * out_elem(out_kind) : nullptr, out_kind, m);
      int grid = std::min<int>(plain_grid, (int)((m + kPlainBlock - 1) / kPlainBlock));
      if (dedup)
        k_probe<Tr, false, true><<<grid, kPlainBlock, 0, s>>>(view(), sc, w);
      else
        k_probe<Tr, false, false><<<grid, kPlainBlock, 0, s>>>(view(), sc, w);
      LSB_CK(cudaGetLastError());
    }
    return LSB_OK;
  }

  // General batch as per-phase launches, window by window.
  int run_plain(const uint8_t* types, uint8_t uniform, const typename Tr::Key* keys,
                uint32_t kstride, const uint64_t* vals, uint32_t vstride, void* out,
                uint32_t out_kind, size_t n, cudaStream_t s) {
    const uint32_t W = sc.max_window;
    for (size_t off = 0; off < n; off += W) {
      uint32_t m = (uint32_t)std::min<size_t>(W, n - off);
      Window<Tr> w = window(types ? types + off : nullptr, uniform, keys + off * kstride, kstride,
                            vals ? vals + off * vstride : nullptr, vstride,
                            out ? (uint8_t*)out + off * out_elem(out_kind) : nullptr, out_kind, m);
      int e = next_epochs(1, s, &w.epoch);
      if (e) return e;
      w.cnt = &sc.cnt[0];
      LSB_CK(cudaMemsetAsync(w.cnt, 0, sizeof(WinCounters), s));
      int grid = std::min<int>(plain_grid, (int)((m + kPlainBlock - 1) / kPlainBlock));
      grid = std::max(grid, 1);
      TableView tv = view();
      if (dedup)
        k_probe<Tr, true, true><<<grid, kPlainBlock, 0, s>>>(tv, sc, w);
      else
        k_probe<Tr, true, false><<<grid, kPlainBlock, 0, s>>>(tv, sc, w);
      k_segments<Tr><<<grid, kPlainBlock, 0, s>>>(sc, w);
      k_scatter<Tr><<<grid, kPlainBlock, 0, s>>>(sc, w);
      k_sort<Tr><<<std::max(grid, num_sms), kPlainBlock, kSortSmemBytes, s>>>(sc, w);
      k_resolve<Tr><<<grid, kPlainBlock, 0, s>>>(tv, sc, w);
      LSB_CK(cudaGetLastError());
    }
    return LSB_OK;
  }

  int run_fused(const uint8_t* types, uint8_t uniform, const typename Tr::Key* keys,
                const uint64_t* vals, void* out, uint32_t out_kind, size_t n, cudaStream_t s) {
    if (n == 0) return LSB_OK;
    if (n > 0xFFFFFFFFull) return LSB_ERR_ARG;
    FusedJob<Tr> job;
    job.base = window(types, uniform, keys, 1, vals, 1, out, out_kind, (uint32_t)n);
    job.window = sc.max_window;
    uint32_t nwin = (uint32_t)((n + job.window - 1) / job.window);
    if (nwin > 0xFFF0u) return LSB_ERR_ARG;
    int e = next_epochs(nwin, s, &job.epoch0);
    if (e) return e;
    LSB_CK(cudaMemsetAsync(sc.cnt, 0, sizeof(WinCounters) * 2, s));
    LSB_CK(cudaMemsetAsync(bar, 0, sizeof(GridBarrier), s));
    TableView tv = view();
    Scratch scv = sc;
    GridBarrier* b = bar;
    void* args[] = {&tv, &scv, &job, &b};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(fused_grid);
    cfg.blockDim = dim3(kFusedBlock);
    cfg.dynamicSmemBytes = kSortSmemBytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    LSB_CK(cudaLaunchKernelExC(&cfg, (const void*)k_fused<Tr>, args));
    return LSB_OK;
  }

  int read_status(uint32_t* flags, cudaStream_t s) {
    uint32_t v = 0;
    LSB_CK(cudaStreamSynchronize(s));
    LSB_CK(cudaMemcpy(&v, status, sizeof(v), cudaMemcpyDeviceToHost));
    LSB_CK(cudaMemset(status, 0, sizeof(uint32_t)));
    if (flags) *flags = v;
    return LSB_OK;
  }

  int pool_usage(uint64_t* used, uint64_t* cap, cudaStream_t s) {
    uint64_t p[2];
    LSB_CK(cudaStreamSynchronize(s));
    LSB_CK(cudaMemcpy(p, pool, sizeof(p), cudaMemcpyDeviceToHost));
    uint64_t u = std::min(p[0], p[1]) - buckets;
    if (used) *used = u;
    if (cap) *cap = pool_slabs;
    return LSB_OK;
  }

  int size(uint64_t* count, cudaStream_t s) {
    unsigned long long* d = nullptr;
    LSB_CK(cudaMalloc(&d, sizeof(*d)));
    cudaMemsetAsync(d, 0, sizeof(*d), s);
    k_count<Tr><<<(buckets + 255) / 256, 256, 0, s>>>(view(), buckets, d);
    unsigned long long h = 0;
    cudaError_t e1 = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e1 != cudaSuccess || e2 != cudaSuccess) return LSB_ERR_CUDA;
    *count = h;
    return LSB_OK;
  }

  // Live entries sorted by key, copied to host arrays.
  int dump(typename Tr::Key* keys_out, uint64_t* vals_out, size_t cap, uint64_t* count,
           cudaStream_t s) {
    uint64_t n = 0;
    int e = size(&n, s);
    if (e) return e;
    if (count) *count = n;
    if (n == 0 || cap == 0) return LSB_OK;
    typename Tr::Key* dk = nullptr;
    uint64_t* dv = nullptr;
    unsigned long long* cur = nullptr;
    if (cudaMalloc(&dk, sizeof(*dk) * n) != cudaSuccess ||
        (Tr::kHasValue && cudaMalloc(&dv, sizeof(uint64_t) * n) != cudaSuccess) ||
        cudaMalloc(&cur, sizeof(*cur)) != cudaSuccess) {
      cudaFree(dk);
      cudaFree(dv);
      cudaFree(cur);
      return LSB_ERR_OOM;
    }
    cudaMemsetAsync(cur, 0, sizeof(*cur), s);
    k_dump<Tr><<<(buckets + 255) / 256, 256, 0, s>>>(view(), buckets, dk, dv, cur, n);
    std::vector<typename Tr::Key> hk(n);
    std::vector<uint64_t> hv(Tr::kHasValue ? n : 0);
    cudaMemcpyAsync(hk.data(), dk, sizeof(*dk) * n, cudaMemcpyDeviceToHost, s);
    if (Tr::kHasValue) cudaMemcpyAsync(hv.data(), dv, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, s);
    cudaError_t err = cudaStreamSynchronize(s);
    cudaFree(dk);
    cudaFree(dv);
    cudaFree(cur);
    if (err != cudaSuccess) return LSB_ERR_CUDA;
    std::vector<size_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return hk[a] < hk[b]; });
    size_t w = std::min<size_t>(cap, n);
    for (size_t i = 0; i < w; ++i) {
      keys_out[i] = hk[idx[i]];
      if (Tr::kHasValue && vals_out) vals_out[i] = hv[idx[i]];
    }
    return LSB_OK;
  }
};

}  // namespace

struct lsb_map {
  Table<MapTraits> t;
};
struct lsb_set {
  Table<SetTraits> t;
};

extern "C" {

// ------------------------------------------------------------------ map
int lsb_map_create_ex(unsigned log2_buckets, const lsb_options* opt, lsb_map** out) {
  if (!out) return LSB_ERR_ARG;
  *out = nullptr;
  lsb_map* m = new (std::nothrow) lsb_map();
  if (!m) return LSB_ERR_OOM;
  int e = m->t.init(log2_buckets, opt);
  if (e) {
    m->t.release();
    delete m;
    return e;
  }
  *out = m;
  return LSB_OK;
}

int lsb_map_create(unsigned log2_buckets, uint64_t pool_slabs, lsb_map** out) {
  lsb_options o{};
  o.pool_slabs = pool_slabs;
  o.device = -1;
  return lsb_map_create_ex(log2_buckets, &o, out);
}

int lsb_map_destroy(lsb_map* m) {
  if (!m) return LSB_ERR_ARG;
  m->t.release();
  delete m;
  return LSB_OK;
}

int lsb_map_get(lsb_map* m, const uint64_t* keys, lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_reads(keys, out, kOutResult, n, s);
}

int lsb_map_put(lsb_map* m, const uint64_t* keys, const uint64_t* vals, uint64_t* old_out,
                size_t n, cudaStream_t s) {
  if (!m || (n && (!keys || !vals))) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 8) || !aligned(old_out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_plain(nullptr, kOpWrite, keys, 1, vals, 1, old_out, kOutOld, n, s);
}

int lsb_map_put_pairs(lsb_map* m, const lsb_kv* ops, uint64_t* old_out, size_t n,
                      cudaStream_t s) {
  if (!m || (n && !ops)) return LSB_ERR_ARG;
  if (!aligned(ops, 8) || !aligned(old_out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  const uint64_t* base = reinterpret_cast<const uint64_t*>(ops);
  return m->t.run_plain(nullptr, kOpWrite, base, 2, base + 1, 2, old_out, kOutOld, n, s);
}

int lsb_map_remove(lsb_map* m, const uint64_t* keys, lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_plain(nullptr, kOpRemove, keys, 1, nullptr, 1, out, kOutResult, n, s);
}

int lsb_map_execute(lsb_map* m, const uint8_t* types, const uint64_t* keys, const uint64_t* vals,
                    lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && (!types || !keys))) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return m->t.run_plain(types, kOpRead, keys, 1, vals, 1, out, kOutResult, n, s);
}

int lsb_map_execute_fused(lsb_map* m, const uint8_t* types, const uint64_t* keys,
                          const uint64_t* vals, lsb_result* out, size_t n, cudaStream_t s) {
  if (!m || (n && (!types || !keys))) return LSB_ERR_ARG;
  if (!aligned(keys, 8) || !aligned(vals, 8) || !aligned(out, 8)) return LSB_ERR_ARG;
  return m->t.run_fused(types, kOpRead, keys, vals, out, kOutResult, n, s);
}

uint32_t lsb_map_buckets(const lsb_map* m) { return m ? m->t.buckets : 0; }

int lsb_map_status(lsb_map* m, uint32_t* flags, cudaStream_t s) {
  if (!m) return LSB_ERR_ARG;
  return m->t.read_status(flags, s);
}

int lsb_map_pool_usage(lsb_map* m, uint64_t* used, uint64_t* capacity, cudaStream_t s) {
  if (!m) return LSB_ERR_ARG;
  return m->t.pool_usage(used, capacity, s);
}

int lsb_map_size(lsb_map* m, uint64_t* count, cudaStream_t s) {
  if (!m || !count) return LSB_ERR_ARG;
  return m->t.size(count, s);
}

int lsb_map_dump(lsb_map* m, uint64_t* keys_out, uint64_t* vals_out, size_t cap,
                 uint64_t* count, cudaStream_t s) {
  if (!m || (cap && (!keys_out || !vals_out))) return LSB_ERR_ARG;
  return m->t.dump(keys_out, vals_out, cap, count, s);
}

// ------------------------------------------------------------------ set
int lsb_set_create_ex(unsigned log2_buckets, const lsb_options* opt, lsb_set** out) {
  if (!out) return LSB_ERR_ARG;
  *out = nullptr;
  lsb_set* p = new (std::nothrow) lsb_set();
  if (!p) return LSB_ERR_OOM;
  int e = p->t.init(log2_buckets, opt);
  if (e) {
    p->t.release();
    delete p;
    return e;
  }
  *out = p;
  return LSB_OK;
}

int lsb_set_create(unsigned log2_buckets, uint64_t pool_slabs, lsb_set** out) {
  lsb_options o{};
  o.pool_slabs = pool_slabs;
  o.device = -1;
  return lsb_set_create_ex(log2_buckets, &o, out);
}

int lsb_set_destroy(lsb_set* p) {
  if (!p) return LSB_ERR_ARG;
  p->t.release();
  delete p;
  return LSB_OK;
}

int lsb_set_insert(lsb_set* p, const uint32_t* keys, bool* out, size_t n, cudaStream_t s) {
  if (!p || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return p->t.run_plain(nullptr, kOpWrite, keys, 1, nullptr, 1, out, kOutBool, n, s);
}

int lsb_set_contains(lsb_set* p, const uint32_t* keys, bool* out, size_t n, cudaStream_t s) {
  if (!p || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return p->t.run_reads(keys, out, kOutBool, n, s);
}

int lsb_set_remove(lsb_set* p, const uint32_t* keys, bool* out, size_t n, cudaStream_t s) {
  if (!p || (n && !keys)) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return p->t.run_plain(nullptr, kOpRemove, keys, 1, nullptr, 1, out, kOutBool, n, s);
}

int lsb_set_execute(lsb_set* p, const uint8_t* types, const uint32_t* keys, bool* out, size_t n,
                    cudaStream_t s) {
  if (!p || (n && (!types || !keys))) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  if (n == 0) return LSB_OK;
  return p->t.run_plain(types, kOpRead, keys, 1, nullptr, 1, out, kOutBool, n, s);
}

int lsb_set_execute_fused(lsb_set* p, const uint8_t* types, const uint32_t* keys, bool* out,
                          size_t n, cudaStream_t s) {
  if (!p || (n && (!types || !keys))) return LSB_ERR_ARG;
  if (!aligned(keys, 4)) return LSB_ERR_ARG;
  return p->t.run_fused(types, kOpRead, keys, nullptr, out, kOutBool, n, s);
}

uint32_t lsb_set_buckets(const lsb_set* p) { return p ? p->t.buckets : 0; }

int lsb_set_status(lsb_set* p, uint32_t* flags, cudaStream_t s) {
  if (!p) return LSB_ERR_ARG;
  return p->t.read_status(flags, s);
}

int lsb_set_pool_usage(lsb_set* p, uint64_t* used, uint64_t* capacity, cudaStream_t s) {
  if (!p) return LSB_ERR_ARG;
  return p->t.pool_usage(used, capacity, s);
}

int lsb_set_size(lsb_set* p, uint64_t* count, cudaStream_t s) {
  if (!p || !count) return LSB_ERR_ARG;
  return p->t.size(count, s);
}

int lsb_set_dump(lsb_set* p, uint32_t* keys_out, size_t cap, uint64_t* count, cudaStream_t s) {
  if (!p || (cap && !keys_out)) return LSB_ERR_ARG;
  return p->t.dump(keys_out, nullptr, cap, count, s);
}

// ------------------------------------------------------------------ misc
const char* lsb_error_string(int code) {
  switch (code) {
    case LSB_OK: return "ok";
    case LSB_ERR_ARG: return "invalid argument";
    case LSB_ERR_OOM: return "out of memory (slab pool or device memory)";
    case LSB_ERR_TIMEOUT: return "a bounded device wait gave up";
    case LSB_ERR_CUDA: return "CUDA runtime error";
    case LSB_ERR_STATE: return "invalid state";
    default: return "unknown error";
  }
}

int lsb_version(void) { return 100; }

}  // extern "C"
