/* Test infrastructure, not product code: the CPU oracle (see lsb_oracle.h).
 *
 * Restates the reference's slab list (depaulmillz/lslab) on the host:
 *   slab layout      include/lslab/detail/slab_node.h:13-35
 *                    (31 key lanes + valid bitmap + next link; the map slab
 *                    carries 32 value lanes, lane 31 unused)
 *   hash             include/lslab/hash.h:10-15 (identity), bucket = hash &
 *                    (2^n - 1) (include/lslab/map.h:96,129; set.h:66,77,86)
 *   FIND             include/lslab/detail/traverse.h:69-96,127-130
 *   INSERT (upsert)  include/lslab/detail/traverse.h:69-93 (hit: functor on
 *                    value[lowest matching lane]), :54-55,75-78,98-113 (miss:
 *                    lowest empty lane of the TAIL slab), :114-124 (tail full:
 *                    allocate a zeroed slab, link it, retry there)
 *   REMOVE           include/lslab/detail/traverse.h:88-91 (valid ^= bit, then
 *                    the functor on the value lane)
 *   map put functor  include/lslab/map.h:136-152 (returns the slot's prior value)
 *   map get          include/lslab/map.h:105-119, include/lslab/detail/map_kernels.h:53-70
 *   set insert       include/lslab/detail/traverse.h:204-212,226-232 (true for a
 *                    new AND an existing key)
 *   set remove       include/lslab/detail/traverse.h:204-212,246-250
 * The reference serves a warp's 32 ops one at a time in lane order
 * (traverse.h:45-48); running the whole batch one op at a time in index order
 * is that rule applied to the batch, which is the order the CUDA path commits.
 *
 * Map remove has no public entry point in the reference; the harness that
 * reaches traverse<REMOVE> (oracle/ref_harness.cu) reports the old value and
 * zeroes the value lane, so a later insert into that lane returns 0.  The
 * oracle does the same.
 */
#include "lsb_oracle.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#define LANES 31
#define NO_NEXT 0xFFFFFFFFu

typedef struct {
  uint32_t valid;
  uint32_t next; /* pool index, NO_NEXT = null */
  uint64_t key[LANES];
  uint64_t value[32];
} map_slab;

typedef struct {
  uint32_t valid;
  uint32_t next;
  uint32_t key[LANES];
} set_slab;

struct orc_map {
  unsigned log2;
  map_slab* heads;
  map_slab* pool;
  uint64_t pool_cap;
  _Atomic uint64_t pool_used;
  int error;
};

struct orc_set {
  unsigned log2;
  set_slab* heads;
  set_slab* pool;
  uint64_t pool_cap;
  _Atomic uint64_t pool_used;
  int error;
};

/* ------------------------------------------------------------------ map */

static inline uint64_t map_bucket(const orc_map* m, uint64_t key) {
  return key & ((1ull << m->log2) - 1); /* identity hash, hash.h:12-14 */
}

static inline map_slab* map_at(orc_map* m, uint32_t idx) { return &m->pool[idx]; }

static uint32_t map_alloc(orc_map* m) {
  uint64_t idx = atomic_fetch_add(&m->pool_used, 1);
  if (idx >= m->pool_cap) {
    m->error = 1; /* the reference traps here (detail/device_allocator.h:65-68) */
    return NO_NEXT;
  }
  memset(&m->pool[idx], 0, sizeof(map_slab));
  m->pool[idx].next = NO_NEXT;
  return (uint32_t)idx;
}

static int map_reserve(orc_map* m, uint64_t extra) {
  uint64_t need = atomic_load(&m->pool_used) + extra;
  if (need <= m->pool_cap) return 0;
  uint64_t cap = m->pool_cap ? m->pool_cap : 1024;
  while (cap < need) cap *= 2;
  map_slab* p = (map_slab*)realloc(m->pool, cap * sizeof(map_slab));
  if (!p) return -1;
  m->pool = p;
  m->pool_cap = cap;
  return 0;
}

orc_map* orc_map_create(unsigned log2_buckets, uint64_t pool_capacity) {
  orc_map* m = (orc_map*)calloc(1, sizeof(orc_map));
  if (!m) return NULL;
  size_t nb = (size_t)1 << log2_buckets;
  m->log2 = log2_buckets;
  m->heads = (map_slab*)calloc(nb, sizeof(map_slab));
  if (!m->heads) {
    free(m);
    return NULL;
  }
  for (size_t b = 0; b < nb; ++b) m->heads[b].next = NO_NEXT;
  atomic_init(&m->pool_used, 0);
  m->pool = NULL;
  m->pool_cap = 0;
  if (map_reserve(m, pool_capacity ? pool_capacity : 1024)) {
    free(m->heads);
    free(m);
    return NULL;
  }
  return m;
}

void orc_map_destroy(orc_map* m) {
  if (!m) return;
  free(m->heads);
  free(m->pool);
  free(m);
}

/* Lowest valid lane of slab s holding key, or -1 (traverse.h:69-86). */
static inline int map_match(const map_slab* s, uint64_t key) {
  for (int lane = 0; lane < LANES; ++lane)
    if (((s->valid >> lane) & 1u) && s->key[lane] == key) return lane;
  return -1;
}

/* FIND: returns 1 and the value when present. */
static int map_find(orc_map* m, uint64_t key, uint64_t* value) {
  map_slab* s = &m->heads[map_bucket(m, key)];
  for (;;) {
    int lane = map_match(s, key);
    if (lane >= 0) {
      *value = s->value[lane];
      return 1;
    }
    if (s->next == NO_NEXT) return 0;
    s = map_at(m, s->next);
  }
}

/* INSERT with the put functor (map.h:138-146): on a hit the value lane is
 * overwritten; on a miss the key goes into the lowest empty lane of the tail
 * slab.  Either way the slot's prior value is returned (0 for a zeroed lane),
 * and *existed reports the hit. */
static uint64_t map_upsert(orc_map* m, uint64_t key, uint64_t val, int* existed) {
  map_slab* s = &m->heads[map_bucket(m, key)];
  for (;;) {
    int lane = map_match(s, key);
    if (lane >= 0) {
      uint64_t old = s->value[lane];
      s->value[lane] = val;
      *existed = 1;
      return old;
    }
    if (s->next != NO_NEXT) {
      s = map_at(m, s->next);
      continue;
    }
    for (int e = 0; e < LANES; ++e) {
      if (!((s->valid >> e) & 1u)) {
        uint64_t old = s->value[e];
        s->key[e] = key;
        s->valid |= 1u << e;
        s->value[e] = val;
        *existed = 0;
        return old;
      }
    }
    uint32_t n = map_alloc(m);
    if (n == NO_NEXT) {
      *existed = 0;
      return 0;
    }
    s->next = n;
    s = map_at(m, n);
  }
}

/* UPDATE (the UPDATE branch of traverse.h:127-130 with the functor of
 * map.h:167-183, which overwrites the value lane of a hit and does nothing on
 * a miss), reporting the lane's prior value: the reference's functor meant to
 * (its `tmp` receives the new value instead, map.h:170) and its batched
 * update_ calls put instead (map_kernels.h:85). */
static int map_update(orc_map* m, uint64_t key, uint64_t val, uint64_t* old) {
  map_slab* s = &m->heads[map_bucket(m, key)];
  for (;;) {
    int lane = map_match(s, key);
    if (lane >= 0) {
      *old = s->value[lane];
      s->value[lane] = val;
      return 1;
    }
    if (s->next == NO_NEXT) return 0;
    s = map_at(m, s->next);
  }
}

/* REMOVE with the harness functor: report and zero the value lane. */
static int map_erase(orc_map* m, uint64_t key, uint64_t* old) {
  map_slab* s = &m->heads[map_bucket(m, key)];
  for (;;) {
    int lane = map_match(s, key);
    if (lane >= 0) {
      s->valid ^= 1u << lane;
      *old = s->value[lane];
      s->value[lane] = 0;
      return 1;
    }
    if (s->next == NO_NEXT) return 0;
    s = map_at(m, s->next);
  }
}

static inline void map_apply(orc_map* m, uint8_t type, uint64_t key, uint64_t val,
                             orc_result* r) {
  memset(r, 0, sizeof(*r));
  if (type == ORC_GET) {
    uint64_t v = 0;
    r->found = (uint8_t)map_find(m, key, &v);
    r->value = r->found ? v : 0;
  } else if (type == ORC_PUT) {
    int existed = 0;
    uint64_t old = map_upsert(m, key, val, &existed);
    r->found = (uint8_t)existed;
    r->value = old;
  } else if (type == ORC_UPDATE) {
    uint64_t old = 0;
    r->found = (uint8_t)map_update(m, key, val, &old);
    r->value = r->found ? old : 0;
  } else {
    uint64_t old = 0;
    r->found = (uint8_t)map_erase(m, key, &old);
    r->value = r->found ? old : 0;
  }
}

void orc_map_get(orc_map* m, const uint64_t* keys, orc_result* out, size_t n) {
  for (size_t i = 0; i < n; ++i) map_apply(m, ORC_GET, keys[i], 0, &out[i]);
}

void orc_map_put(orc_map* m, const uint64_t* keys, const uint64_t* vals, uint64_t* old_out,
                 size_t n) {
  map_reserve(m, n);
  for (size_t i = 0; i < n; ++i) {
    orc_result r;
    map_apply(m, ORC_PUT, keys[i], vals[i], &r);
    old_out[i] = r.value;
  }
}

void orc_map_update(orc_map* m, const uint64_t* keys, const uint64_t* vals, orc_result* out,
                    size_t n) {
  for (size_t i = 0; i < n; ++i) map_apply(m, ORC_UPDATE, keys[i], vals[i], &out[i]);
}

void orc_map_remove(orc_map* m, const uint64_t* keys, orc_result* out, size_t n) {
  for (size_t i = 0; i < n; ++i) map_apply(m, ORC_REMOVE, keys[i], 0, &out[i]);
}

void orc_map_mixed(orc_map* m, const uint8_t* types, const uint64_t* keys,
                   const uint64_t* vals, orc_result* out, size_t n) {
  map_reserve(m, n);
  for (size_t i = 0; i < n; ++i)
    map_apply(m, types[i], keys[i], vals ? vals[i] : 0, &out[i]);
}

typedef struct {
  orc_map* m;
  orc_set* s;
  const uint8_t* types;
  const uint64_t* keys64;
  const uint32_t* keys32;
  const uint64_t* vals;
  orc_result* out16;
  uint8_t* out8;
  size_t n;
  int tid, threads;
} shard_job;

static void* map_shard(void* arg) {
  shard_job* j = (shard_job*)arg;
  for (size_t i = 0; i < j->n; ++i) {
    uint64_t k = j->keys64[i];
    if ((int)(map_bucket(j->m, k) % (uint64_t)j->threads) != j->tid) continue;
    map_apply(j->m, j->types[i], k, j->vals ? j->vals[i] : 0, &j->out16[i]);
  }
  return NULL;
}

int orc_map_mixed_mt(orc_map* m, const uint8_t* types, const uint64_t* keys,
                     const uint64_t* vals, orc_result* out, size_t n, int threads) {
  if (threads <= 1) {
    orc_map_mixed(m, types, keys, vals, out, n);
    return 1;
  }
  if (map_reserve(m, n)) return -1; /* the pool cannot move while threads run */
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
  shard_job* jobs = (shard_job*)calloc(threads, sizeof(shard_job));
  int started = 0;
  for (int t = 0; t < threads; ++t) {
    jobs[t] = (shard_job){m, NULL, types, keys, NULL, vals, out, NULL, n, t, threads};
    if (pthread_create(&th[t], NULL, map_shard, &jobs[t]) != 0) break;
    ++started;
  }
  for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
  /* shards that never started run here, still in index order */
  for (int t = started; t < threads; ++t) map_shard(&jobs[t]);
  free(th);
  free(jobs);
  return started ? started : 1;
}

size_t orc_map_dump(const orc_map* m, uint64_t* keys_out, uint64_t* vals_out, size_t cap) {
  size_t nb = (size_t)1 << m->log2, w = 0;
  for (size_t b = 0; b < nb; ++b) {
    const map_slab* s = &m->heads[b];
    for (;;) {
      for (int lane = 0; lane < LANES; ++lane) {
        if ((s->valid >> lane) & 1u) {
          if (w < cap) {
            keys_out[w] = s->key[lane];
            vals_out[w] = s->value[lane];
          }
          ++w;
        }
      }
      if (s->next == NO_NEXT) break;
      s = &m->pool[s->next];
    }
  }
  return w;
}

size_t orc_map_size(const orc_map* m) { return orc_map_dump(m, NULL, NULL, 0); }
uint64_t orc_map_slabs_used(const orc_map* m) { return atomic_load(&((orc_map*)m)->pool_used); }
int orc_map_error(const orc_map* m) { return m->error; }

/* ------------------------------------------------------------------ set */

static inline uint64_t set_bucket(const orc_set* s, uint32_t key) {
  return (uint64_t)key & ((1ull << s->log2) - 1);
}

static uint32_t set_alloc(orc_set* s) {
  uint64_t idx = atomic_fetch_add(&s->pool_used, 1);
  if (idx >= s->pool_cap) {
    s->error = 1;
    return NO_NEXT;
  }
  memset(&s->pool[idx], 0, sizeof(set_slab));
  s->pool[idx].next = NO_NEXT;
  return (uint32_t)idx;
}

static int set_reserve(orc_set* s, uint64_t extra) {
  uint64_t need = atomic_load(&s->pool_used) + extra;
  if (need <= s->pool_cap) return 0;
  uint64_t cap = s->pool_cap ? s->pool_cap : 1024;
  while (cap < need) cap *= 2;
  set_slab* p = (set_slab*)realloc(s->pool, cap * sizeof(set_slab));
  if (!p) return -1;
  s->pool = p;
  s->pool_cap = cap;
  return 0;
}

orc_set* orc_set_create(unsigned log2_buckets, uint64_t pool_capacity) {
  orc_set* s = (orc_set*)calloc(1, sizeof(orc_set));
  if (!s) return NULL;
  size_t nb = (size_t)1 << log2_buckets;
  s->log2 = log2_buckets;
  s->heads = (set_slab*)calloc(nb, sizeof(set_slab));
  if (!s->heads) {
    free(s);
    return NULL;
  }
  for (size_t b = 0; b < nb; ++b) s->heads[b].next = NO_NEXT;
  atomic_init(&s->pool_used, 0);
  if (set_reserve(s, pool_capacity ? pool_capacity : 1024)) {
    free(s->heads);
    free(s);
    return NULL;
  }
  return s;
}

void orc_set_destroy(orc_set* s) {
  if (!s) return;
  free(s->heads);
  free(s->pool);
  free(s);
}

static inline int set_match(const set_slab* sl, uint32_t key) {
  for (int lane = 0; lane < LANES; ++lane)
    if (((sl->valid >> lane) & 1u) && sl->key[lane] == key) return lane;
  return -1;
}

/* One set op in the reference's semantics; returns the op's bool result. */
static uint8_t set_apply(orc_set* s, uint8_t type, uint32_t key) {
  set_slab* sl = &s->heads[set_bucket(s, key)];
  for (;;) {
    int lane = set_match(sl, key);
    if (lane >= 0) {
      if (type == ORC_SET_REMOVE) sl->valid ^= 1u << lane;
      return 1; /* contains / insert-existing / remove-hit */
    }
    if (sl->next != NO_NEXT) {
      sl = &s->pool[sl->next];
      continue;
    }
    if (type != ORC_INSERT) return 0;
    for (int e = 0; e < LANES; ++e) {
      if (!((sl->valid >> e) & 1u)) {
        sl->key[e] = key;
        sl->valid |= 1u << e;
        return 1;
      }
    }
    uint32_t n = set_alloc(s);
    if (n == NO_NEXT) return 0;
    sl->next = n;
    sl = &s->pool[n];
  }
}

void orc_set_insert(orc_set* s, const uint32_t* keys, uint8_t* out, size_t n) {
  set_reserve(s, n);
  for (size_t i = 0; i < n; ++i) out[i] = set_apply(s, ORC_INSERT, keys[i]);
}

void orc_set_contains(orc_set* s, const uint32_t* keys, uint8_t* out, size_t n) {
  for (size_t i = 0; i < n; ++i) out[i] = set_apply(s, ORC_CONTAINS, keys[i]);
}

void orc_set_remove(orc_set* s, const uint32_t* keys, uint8_t* out, size_t n) {
  for (size_t i = 0; i < n; ++i) out[i] = set_apply(s, ORC_SET_REMOVE, keys[i]);
}

void orc_set_mixed(orc_set* s, const uint8_t* types, const uint32_t* keys, uint8_t* out,
                   size_t n) {
  set_reserve(s, n);
  for (size_t i = 0; i < n; ++i) out[i] = set_apply(s, types[i], keys[i]);
}

static void* set_shard(void* arg) {
  shard_job* j = (shard_job*)arg;
  for (size_t i = 0; i < j->n; ++i) {
    uint32_t k = j->keys32[i];
    if ((int)(set_bucket(j->s, k) % (uint64_t)j->threads) != j->tid) continue;
    j->out8[i] = set_apply(j->s, j->types[i], k);
  }
  return NULL;
}

int orc_set_mixed_mt(orc_set* s, const uint8_t* types, const uint32_t* keys, uint8_t* out,
                     size_t n, int threads) {
  if (threads <= 1) {
    orc_set_mixed(s, types, keys, out, n);
    return 1;
  }
  if (set_reserve(s, n)) return -1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * threads);
  shard_job* jobs = (shard_job*)calloc(threads, sizeof(shard_job));
  int started = 0;
  for (int t = 0; t < threads; ++t) {
    jobs[t] = (shard_job){NULL, s, types, NULL, keys, NULL, NULL, out, n, t, threads};
    if (pthread_create(&th[t], NULL, set_shard, &jobs[t]) != 0) break;
    ++started;
  }
  for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
  for (int t = started; t < threads; ++t) set_shard(&jobs[t]);
  free(th);
  free(jobs);
  return started ? started : 1;
}

size_t orc_set_dump(const orc_set* s, uint32_t* keys_out, size_t cap) {
  size_t nb = (size_t)1 << s->log2, w = 0;
  for (size_t b = 0; b < nb; ++b) {
    const set_slab* sl = &s->heads[b];
    for (;;) {
      for (int lane = 0; lane < LANES; ++lane) {
        if ((sl->valid >> lane) & 1u) {
          if (w < cap) keys_out[w] = sl->key[lane];
          ++w;
        }
      }
      if (sl->next == NO_NEXT) break;
      sl = &s->pool[sl->next];
    }
  }
  return w;
}

size_t orc_set_size(const orc_set* s) { return orc_set_dump(s, NULL, 0); }
uint64_t orc_set_slabs_used(const orc_set* s) { return atomic_load(&((orc_set*)s)->pool_used); }
int orc_set_error(const orc_set* s) { return s->error; }
