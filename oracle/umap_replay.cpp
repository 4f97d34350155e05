// Test infrastructure (a reported CPU baseline, never the product): the
// batch op stream replayed on std::unordered_map<uint64_t, uint64_t> in
// op-index order on the host.  Results use the library's conventions: a get
// gives {found, value or 0}, a put {existed, old value or 0} and then stores
// the new value, a remove {existed, value or 0} and then erases the key, an
// update {existed, old value or 0} and then stores the new value if it existed.
//
// Keys are spread over `shards` maps by a multiplicative hash.  Ops on
// different keys commute, so a replay in which every shard processes its own
// ops in index order (one thread per shard) gives the sequential results; a
// replay with one thread walks all ops in index order.
#include <chrono>
#include <cstdint>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

struct Umap {
  std::vector<std::unordered_map<uint64_t, uint64_t>> maps;
  uint32_t shard_of(uint64_t k) const {
    return (uint32_t)(((k * 0x9E3779B97F4A7C15ull) >> 32) % maps.size());
  }
};

struct Result {
  uint8_t found;
  uint8_t pad[7];
  uint64_t value;
};

template <class F>
void on_threads(uint32_t threads, F f) {
  if (threads <= 1) {
    f(0u);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(threads);
  for (uint32_t t = 0; t < threads; ++t) pool.emplace_back(f, t);
  for (auto& th : pool) th.join();
}

void apply(std::unordered_map<uint64_t, uint64_t>& m, uint8_t type, uint64_t key, uint64_t val,
           Result* out) {
  auto it = m.find(key);
  const bool had = it != m.end();
  if (out) {
    out->found = had ? 1 : 0;
    out->value = had ? it->second : 0;
  }
  if (type == 1) {
    if (had)
      it->second = val;
    else
      m.emplace(key, val);
  } else if (type == 2 && had) {
    m.erase(it);
  } else if (type == 3 && had) {  // update-if-present
    it->second = val;
  }
}

}  // namespace

extern "C" {

// Shard maps filled with n prefill keys (later duplicates overwrite), one
// thread per shard.  Returns null on allocation failure.
void* umap_create(uint32_t shards, const uint64_t* keys, const uint64_t* vals, uint64_t n) {
  if (shards == 0) shards = 1;
  Umap* u = new (std::nothrow) Umap();
  if (!u) return nullptr;
  try {
    u->maps.resize(shards);
    for (auto& m : u->maps) m.reserve((size_t)(n / shards + n / (4 * shards) + 16));
    on_threads(shards, [&](uint32_t t) {
      auto& m = u->maps[t];
      for (uint64_t i = 0; i < n; ++i)
        if (u->shard_of(keys[i]) == t) m[keys[i]] = vals[i];
    });
  } catch (...) {
    delete u;
    return nullptr;
  }
  return u;
}

// Replays n ops (types 0 get, 1 put, 2 remove) with `threads` = 1 (index
// order over all maps) or the shard count (one thread per shard).  Writes
// results to out (may be null) and returns the replay's wall time in
// seconds (steady_clock), or -1 for a bad thread count.
double umap_replay(void* h, const uint8_t* types, const uint64_t* keys, const uint64_t* vals,
                   uint64_t n, uint32_t threads, void* out) {
  Umap* u = static_cast<Umap*>(h);
  if (threads != 1 && threads != u->maps.size()) return -1.0;
  Result* res = static_cast<Result*>(out);
  const auto t0 = std::chrono::steady_clock::now();
  if (threads == 1) {
    for (uint64_t i = 0; i < n; ++i)
      apply(u->maps[u->shard_of(keys[i])], types[i], keys[i], vals ? vals[i] : 0,
            res ? res + i : nullptr);
  } else {
    on_threads(threads, [&](uint32_t t) {
      auto& m = u->maps[t];
      for (uint64_t i = 0; i < n; ++i)
        if (u->shard_of(keys[i]) == t)
          apply(m, types[i], keys[i], vals ? vals[i] : 0, res ? res + i : nullptr);
    });
  }
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

uint64_t umap_size(void* h) {
  uint64_t s = 0;
  for (auto& m : static_cast<Umap*>(h)->maps) s += m.size();
  return s;
}

void umap_destroy(void* h) { delete static_cast<Umap*>(h); }

}  // extern "C"
