// Checkpoints: a table's live contents saved to a file and loaded into a new
// table.  The file holds sorted (key, value) records, not slabs, so it does
// not depend on the slab layout, the hash or the table size: a checkpoint
// loads into a table of any bucket count, and any producer that writes the
// format (lslab_b200/checkpoint.py writes and reads it on the host) can
// seed a table.
//
// File layout (little-endian):
//   0   char[8]  magic "LSBCKPT1"
//   8   u32      format version (1)
//   12  u32      container: 0 map<u64,u64>, 1 set<u32>
//   16  u32      log2 buckets of the saved table
//   20  u32      key bytes (8 map, 4 set)
//   24  u32      value bytes (8 map, 0 set)
//   28  u32      lock mode of the saved table
//   32  u64      overflow pool slabs of the saved table
//   40  u64      record count
//   48  u64      checksum of the records (below)
//   56  records, ascending by key: map {u64 key, u64 value}, set {u32 key}
// Checksum: the records read as little-endian u64 words (the last one padded
// with zero bytes), sum over i of mix64(word_i + i * 0x9E3779B97F4A7C15)
// modulo 2^64, mix64 being MurmurHash3's 64-bit finaliser.
//
// No counterpart in the reference (lslab has no persistence); its tables can
// only be rebuilt by replaying puts.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "lsb.h"
#include "lsb_core.cuh"
#include "lsb_internal.h"

namespace {

constexpr char kMagic[8] = {'L', 'S', 'B', 'C', 'K', 'P', 'T', '1'};
constexpr uint32_t kVersion = 1;
constexpr size_t kHeaderBytes = 56;
constexpr size_t kLoadChunk = size_t(1) << 22;  // records per bulk insert on load

struct Header {
  uint32_t container, log2, key_bytes, value_bytes, lock_mode;
  uint64_t pool_slabs, count, checksum;
};

void put32(uint8_t* p, uint32_t v) { std::memcpy(p, &v, 4); }
void put64(uint8_t* p, uint64_t v) { std::memcpy(p, &v, 8); }
uint32_t get32(const uint8_t* p) {
  uint32_t v;
  std::memcpy(&v, p, 4);
  return v;
}
uint64_t get64(const uint8_t* p) {
  uint64_t v;
  std::memcpy(&v, p, 8);
  return v;
}

// Running checksum over a byte stream cut into u64 words at absolute word
// positions (so records may arrive in chunks of any size).
struct Checksum {
  uint64_t sum = 0, word = 0, index = 0;
  uint32_t fill = 0;  // bytes in `word`
  void add(const uint8_t* p, size_t n) {
    for (size_t i = 0; i < n; ++i) {
      word |= (uint64_t)p[i] << (8 * fill);
      if (++fill == 8) flush();
    }
  }
  void flush() {
    sum += lsb::mix64(word + index * 0x9E3779B97F4A7C15ull);
    ++index;
    word = 0;
    fill = 0;
  }
  uint64_t done() {
    if (fill) flush();
    return sum;
  }
};

void encode_header(uint8_t* h, const Header& x) {
  std::memcpy(h, kMagic, 8);
  put32(h + 8, kVersion);
  put32(h + 12, x.container);
  put32(h + 16, x.log2);
  put32(h + 20, x.key_bytes);
  put32(h + 24, x.value_bytes);
  put32(h + 28, x.lock_mode);
  put64(h + 32, x.pool_slabs);
  put64(h + 40, x.count);
  put64(h + 48, x.checksum);
}

int decode_header(const uint8_t* h, uint32_t container, Header* x) {
  if (std::memcmp(h, kMagic, 8) != 0 || get32(h + 8) != kVersion) return LSB_ERR_IO;
  x->container = get32(h + 12);
  x->log2 = get32(h + 16);
  x->key_bytes = get32(h + 20);
  x->value_bytes = get32(h + 24);
  x->lock_mode = get32(h + 28);
  x->pool_slabs = get64(h + 32);
  x->count = get64(h + 40);
  x->checksum = get64(h + 48);
  const bool map = container == 0;
  if (x->container != container || x->key_bytes != (map ? 8u : 4u) ||
      x->value_bytes != (map ? 8u : 0u) || x->log2 < 1 || x->log2 > 30)
    return LSB_ERR_IO;
  return LSB_OK;
}

size_t record_bytes(uint32_t container) { return container == 0 ? 16 : 4; }

// Writes header + records; `rec` holds count records already in file order.
int write_file(const char* path, const Header& x, const uint8_t* rec) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return LSB_ERR_IO;
  uint8_t h[kHeaderBytes];
  encode_header(h, x);
  const size_t bytes = x.count * record_bytes(x.container);
  const bool ok = std::fwrite(h, 1, kHeaderBytes, f) == kHeaderBytes &&
                  (bytes == 0 || std::fwrite(rec, 1, bytes, f) == bytes);
  return (std::fclose(f) == 0 && ok) ? LSB_OK : LSB_ERR_IO;
}

// Reads the header, then hands records to `sink(records, count)` in chunks of
// at most kLoadChunk; verifies the count (no trailing bytes) and the checksum.
template <class Sink>
int read_file(const char* path, uint32_t container, Header* x, Sink sink) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return LSB_ERR_IO;
  uint8_t h[kHeaderBytes];
  int rc = std::fread(h, 1, kHeaderBytes, f) == kHeaderBytes ? decode_header(h, container, x)
                                                             : LSB_ERR_IO;
  const size_t rb = record_bytes(container);
  std::vector<uint8_t> buf;
  Checksum ck;
  uint64_t left = rc == LSB_OK ? x->count : 0;
  while (rc == LSB_OK && left) {
    const size_t n = (size_t)std::min<uint64_t>(left, kLoadChunk);
    buf.resize(n * rb);
    if (std::fread(buf.data(), 1, n * rb, f) != n * rb) {
      rc = LSB_ERR_IO;
      break;
    }
    ck.add(buf.data(), n * rb);
    rc = sink(buf.data(), n);
    left -= n;
  }
  if (rc == LSB_OK && (std::fgetc(f) != EOF || ck.done() != x->checksum)) rc = LSB_ERR_IO;
  std::fclose(f);
  return rc;
}

// Options for the loaded table: the saved shape unless the caller's say
// otherwise (a zero pool size takes the saved one).
lsb_options load_options(const lsb_options* opt, const Header& x) {
  lsb_options o{};
  if (opt) {
    o = *opt;
  } else {
    o.device = -1;
    o.lock_mode = x.lock_mode;
  }
  if (!o.pool_slabs) o.pool_slabs = x.pool_slabs;
  return o;
}

template <class T>
int finish_load(T* t, int rc, cudaStream_t stream, int (*status)(T*, uint32_t*, cudaStream_t),
                int (*destroy)(T*), T** out) {
  uint32_t st = 0;
  if (rc == LSB_OK) rc = status(t, &st, stream);
  if (rc == LSB_OK && st) rc = (st & LSB_STATUS_OOM) ? LSB_ERR_OOM : LSB_ERR_TIMEOUT;
  if (rc != LSB_OK) {
    if (t) destroy(t);
    return rc;
  }
  *out = t;
  return LSB_OK;
}

}  // namespace

extern "C" {

int lsb_map_save(lsb_map* m, const char* path, cudaStream_t stream) {
  if (!m || !path) return LSB_ERR_ARG;
  uint64_t n = 0, got = 0, used = 0, cap = 0;
  int rc = lsb_map_size(m, &n, stream);
  if (rc) return rc;
  std::vector<uint64_t> k(n), v(n);
  rc = lsb_map_dump(m, k.data(), v.data(), n, &got, stream);  // ascending keys
  if (rc) return rc;
  if (got != n) return LSB_ERR_STATE;
  rc = lsb_map_pool_usage(m, &used, &cap, stream);
  if (rc) return rc;
  std::vector<uint8_t> rec(n * 16);
  for (uint64_t i = 0; i < n; ++i) {
    put64(&rec[16 * i], k[i]);
    put64(&rec[16 * i + 8], v[i]);
  }
  Checksum ck;
  ck.add(rec.data(), rec.size());
  Header x{0, 0, 8, 8, lsb_internal_lock_mode_map(m), cap, n, ck.done()};
  while ((1u << x.log2) < lsb_map_buckets(m)) ++x.log2;
  return write_file(path, x, rec.data());
}

int lsb_map_load(const char* path, const lsb_options* opt, lsb_map** out, cudaStream_t stream) {
  if (!path || !out) return LSB_ERR_ARG;
  *out = nullptr;
  lsb_map* m = nullptr;
  uint64_t* d_keys = nullptr;
  uint64_t* d_vals = nullptr;
  Header x{};
  int rc = read_file(path, 0, &x, [&](const uint8_t* rec, size_t n) -> int {
    if (!m) {
      const lsb_options o = load_options(opt, x);
      int e = lsb_map_create_ex(x.log2, &o, &m);
      if (e) return e;
      if (cudaMalloc(&d_keys, 8 * kLoadChunk) != cudaSuccess ||
          cudaMalloc(&d_vals, 8 * kLoadChunk) != cudaSuccess)
        return LSB_ERR_OOM;
    }
    std::vector<uint64_t> k(n), v(n);
    for (size_t i = 0; i < n; ++i) {
      k[i] = get64(rec + 16 * i);
      v[i] = get64(rec + 16 * i + 8);
    }
    if (cudaMemcpyAsync(d_keys, k.data(), 8 * n, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
        cudaMemcpyAsync(d_vals, v.data(), 8 * n, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return LSB_ERR_CUDA;
    int e = lsb_map_put(m, d_keys, d_vals, nullptr, n, stream);
    if (e) return e;
    return cudaStreamSynchronize(stream) == cudaSuccess ? LSB_OK : LSB_ERR_CUDA;
  });
  if (rc == LSB_OK && !m) {  // an empty checkpoint
    const lsb_options o = load_options(opt, x);
    rc = lsb_map_create_ex(x.log2, &o, &m);
  }
  cudaFree(d_keys);
  cudaFree(d_vals);
  return finish_load(m, rc, stream, lsb_map_status, lsb_map_destroy, out);
}

int lsb_set_save(lsb_set* s, const char* path, cudaStream_t stream) {
  if (!s || !path) return LSB_ERR_ARG;
  uint64_t n = 0, got = 0, used = 0, cap = 0;
  int rc = lsb_set_size(s, &n, stream);
  if (rc) return rc;
  std::vector<uint32_t> k(n);
  rc = lsb_set_dump(s, k.data(), n, &got, stream);
  if (rc) return rc;
  if (got != n) return LSB_ERR_STATE;
  rc = lsb_set_pool_usage(s, &used, &cap, stream);
  if (rc) return rc;
  std::vector<uint8_t> rec(n * 4);
  for (uint64_t i = 0; i < n; ++i) put32(&rec[4 * i], k[i]);
  Checksum ck;
  ck.add(rec.data(), rec.size());
  Header x{1, 0, 4, 0, lsb_internal_lock_mode_set(s), cap, n, ck.done()};
  while ((1u << x.log2) < lsb_set_buckets(s)) ++x.log2;
  return write_file(path, x, rec.data());
}

int lsb_set_load(const char* path, const lsb_options* opt, lsb_set** out, cudaStream_t stream) {
  if (!path || !out) return LSB_ERR_ARG;
  *out = nullptr;
  lsb_set* s = nullptr;
  uint32_t* d_keys = nullptr;
  Header x{};
  int rc = read_file(path, 1, &x, [&](const uint8_t* rec, size_t n) -> int {
    if (!s) {
      const lsb_options o = load_options(opt, x);
      int e = lsb_set_create_ex(x.log2, &o, &s);
      if (e) return e;
      if (cudaMalloc(&d_keys, 4 * kLoadChunk) != cudaSuccess) return LSB_ERR_OOM;
    }
    std::vector<uint32_t> k(n);
    for (size_t i = 0; i < n; ++i) k[i] = get32(rec + 4 * i);
    if (cudaMemcpyAsync(d_keys, k.data(), 4 * n, cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return LSB_ERR_CUDA;
    int e = lsb_set_insert(s, d_keys, nullptr, n, stream);
    if (e) return e;
    return cudaStreamSynchronize(stream) == cudaSuccess ? LSB_OK : LSB_ERR_CUDA;
  });
  if (rc == LSB_OK && !s) {
    const lsb_options o = load_options(opt, x);
    rc = lsb_set_create_ex(x.log2, &o, &s);
  }
  cudaFree(d_keys);
  return finish_load(s, rc, stream, lsb_set_status, lsb_set_destroy, out);
}

}  // extern "C"
