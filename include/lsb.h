/*
 * lsb — a B200-native (sm_100a) slab-list hash map (uint64 -> uint64) and
 * set (uint32) with the batched API of depaulmillz/lslab.
 *
 * Plain C ABI: opaque handles, device pointers, sizes, a CUDA stream.  Every
 * batched call is asynchronous and stream-ordered, like the reference's
 * <<<...>>> launches, and returns an int status for what can be checked on
 * the host (LSB_ERR_ARG, launch failures).  Errors raised on the device
 * (slab pool exhausted, a bounded wait that gave up) are recorded in the
 * table's status word and read with lsb_map_status / lsb_set_status.  The
 * reference has no error return at all: it exits or traps
 * (include/lslab/lslab.h:28-41, include/lslab/detail/device_allocator.h:65-68).
 *
 * Batch semantics (all entry points): the ops of one call take effect as if
 * run one at a time in index order.  The reference gives that order within
 * each warp (lane order, include/lslab/detail/traverse.h:45-48) and an
 * unspecified order across warps; this library gives it across the whole
 * call, so results are deterministic, equal to a sequential replay, and for
 * batches without same-key conflicts equal to the reference's.
 *
 * Concurrency: calls on one table must be ordered on one stream when any of
 * them mutates.  Concurrent read-only calls are fine.
 */
#ifndef LSB_H
#define LSB_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define LSB_OK 0
#define LSB_ERR_ARG 1     /* bad handle, null pointer, size over a limit   */
#define LSB_ERR_OOM 2     /* slab pool or device memory exhausted          */
#define LSB_ERR_TIMEOUT 3 /* a bounded device wait gave up (lock, barrier) */
#define LSB_ERR_CUDA 4    /* a CUDA runtime call failed                    */
#define LSB_ERR_STATE 5   /* call not valid in the object's current state  */
#define LSB_ERR_IO 6      /* checkpoint file unreadable, unwritable or corrupt */

/* Device status bits (lsb_map_status / lsb_set_status). */
#define LSB_STATUS_OOM 0x1u
#define LSB_STATUS_TIMEOUT 0x2u
#define LSB_STATUS_CHAIN 0x4u   /* a chain walk hit its hop limit */
#define LSB_STATUS_BARRIER 0x8u /* a grid barrier gave up          */
#define LSB_STATUS_SCRATCH 0x10u /* window scratch read back out of range; access skipped */

/* ---- op codes of mixed batches -------------------------------------- */
#define LSB_OP_GET 0u
#define LSB_OP_PUT 1u
#define LSB_OP_REMOVE 2u
#define LSB_OP_UPDATE 3u /* map: overwrite a present key's value; an absent key stays absent */
#define LSB_OP_CONTAINS 0u /* set */
#define LSB_OP_INSERT 1u   /* set */

/* Result of a map get/remove (and of every op of a mixed batch).  Layout of
 * cuda::std::pair<bool, uint64_t> as written by the reference's get kernel
 * (include/lslab/detail/map_kernels.h:53-70): bool at byte 0, value at 8.
 * On a miss the value is 0 (the reference leaves it unwritten).  For a put in
 * a mixed batch: found = the key existed, value = the old value or 0. */
typedef struct lsb_result {
  uint8_t found;
  uint8_t pad[7];
  uint64_t value;
} lsb_result;

/* Layout of cuda::std::pair<uint64_t, uint64_t> (AoS put input,
 * include/lslab/map.h:189-192). */
typedef struct lsb_kv {
  uint64_t key;
  uint64_t value;
} lsb_kv;

/* Maps with 32-bit values (lslab::map<K, unsigned>, the shape the reference's
 * own benchmark uses, benchmark/benchmark.cu:56): results in the layout of
 * cuda::std::pair<bool, uint32_t> (bool at byte 0, value at 4, 8 bytes) and
 * AoS inputs in that of cuda::std::pair<uint64_t, uint32_t> (16 bytes). */
typedef struct lsb_result32 {
  uint8_t found;
  uint8_t pad[3];
  uint32_t value;
} lsb_result32;

typedef struct lsb_kv32 {
  uint64_t key;
  uint32_t value;
  uint32_t pad;
} lsb_kv32;

typedef struct lsb_map lsb_map;
typedef struct lsb_set lsb_set;

/* Creation options; zero-initialise and set what you need. */
typedef struct lsb_options {
  uint64_t pool_slabs;   /* overflow slab pool; 0 = default (see lsb_map_create) */
  uint32_t max_window;   /* ops per internal window (scratch size); 0 = 2^20     */
  uint32_t lock_mode;    /* LSB_LOCK_*; 0 = LSB_LOCK_WRITER                     */
  int device;            /* CUDA device; -1 = current                            */
} lsb_options;

/* Launch tuning of a table (see lsb_*_set_tuning); the autotuner picks it. */
typedef struct lsb_tuning {
  uint32_t block_threads; /* threads per block: 128, 256, 512 or 1024 (4..32 warps) */
  uint32_t chunk;         /* ops a block claims per step in the probe phase (its warps
                             share them out), multiple of 32 up to 2^20; 0 = static
                             grid stride.  With fused_split 0: the claim size of the
                             reads of the fused path; 0 = one tile per warp */
  uint32_t prefetch;      /* extra lookups a thread keeps in flight: 0, 1 or 2 */
  uint32_t dedup;         /* 1: lanes of a warp carrying the same key share one lookup */
  uint32_t fused_split;   /* fused path: percent of a window's reads probed before the
                             same-key ordering pass (the rest run during it), 0..100,
                             default 100; 0 = the mutations are listed and probed first
                             while blocks take reads, the remaining reads run during the
                             ordering (faster on batches with interleaved op types) */
  uint32_t region_order;  /* fused path: 1 = probe a window in table-region order */
  uint32_t warp_probe;    /* read-only batches: 1 = the warp-cooperative slab probe (a
                             warp serves its lanes' distinct keys one at a time, lanes
                             reading a slab's slots together); 0 = one op per thread,
                             tag sector then candidate slot (default, faster) */
  uint32_t overlap;       /* mixed batches (execute, execute_fused): 1 = each window runs
                             as launches on two streams, the reads through the lean read
                             kernel while the mutations are listed, probed, grouped and
                             ordered on a higher-priority stream; the mutations are applied
                             after both (read-mostly windows of many ops); 0 = per-phase
                             launches on the caller's stream (execute) and the persistent
                             kernel (execute_fused) */
  uint32_t read_order;    /* the lean read kernel (get / contains calls, the reads of the
                             two-stream form): 0 = in op order (default), 1 = in table-region
                             order built on the device first (measured slower: the ordering
                             steps cost more than the locality saves) */
} lsb_tuning;

#define LSB_LOCK_WRITER 0u   /* writers take a per-bucket lock; readers never lock   */
#define LSB_LOCK_FREE 1u     /* writers claim slots with CAS on slab words; growing a
                                full chain takes the bucket lock */
#define LSB_LOCK_RW 2u       /* reference-style: readers take a shared bucket lock too */

/* ---- map<uint64_t, uint64_t> ------------------------------------------
 * Replaces lslab::map<K,V>::map(unsigned n_log_2) (include/lslab/map.h:43-52)
 * and map(n_log_2, Allocator&&) (include/lslab/map.h:57-66): 2^log2_buckets
 * head slabs plus an overflow pool of pool_slabs slabs (the reference's
 * device_allocator(stack_size), include/lslab/device_allocator.h:16;
 * default when 0: 2^log2_buckets / 4 + 4096). */
int lsb_map_create(unsigned log2_buckets, uint64_t pool_slabs, lsb_map** out);
int lsb_map_create_ex(unsigned log2_buckets, const lsb_options* opt, lsb_map** out);
int lsb_map_destroy(lsb_map* m);

/* lslab::map::get<bs>(K*, pair<bool,V>*, size_t, cudaStream_t),
 * include/lslab/map.h:208-211 -> map_kernels::get_, map_kernels.h:53-70. */
int lsb_map_get(lsb_map* m, const uint64_t* keys, lsb_result* out, size_t n,
                cudaStream_t stream);

/* lslab::map::put<bs>(K*, V*, V* old, size_t, cudaStream_t),
 * include/lslab/map.h:198-201 -> map_kernels::put_ (SoA), map_kernels.h:32-50.
 * old_out[i] = value before put i (0 if the key was absent); may be NULL. */
int lsb_map_put(lsb_map* m, const uint64_t* keys, const uint64_t* vals, uint64_t* old_out,
                size_t n, cudaStream_t stream);

/* lslab::map::put<bs>(pair<K,V>*, V*, size_t, cudaStream_t),
 * include/lslab/map.h:189-192 -> map_kernels::put_ (AoS), map_kernels.h:12-30. */
int lsb_map_put_pairs(lsb_map* m, const lsb_kv* ops, uint64_t* old_out, size_t n,
                      cudaStream_t stream);

/* lslab::map::update<bs>(pair<K,V>*, pair<bool,V>*, size_t, cudaStream_t),
 * include/lslab/map.h:217-220 -> map_kernels::update_, map_kernels.h:72-89,
 * with the semantics the reference intends (map.h:154-183, the UPDATE branch
 * of traverse.h:127-130) and does not deliver (its kernel calls put,
 * map_kernels.h:85): update-if-present.  out[i] = {1, old value} and the
 * value becomes ops[i].value when the key is present; {0, 0} and no change
 * when it is absent.  out may be NULL. */
int lsb_map_update(lsb_map* m, const lsb_kv* ops, lsb_result* out, size_t n,
                   cudaStream_t stream);

/* The same calls for maps whose values are 32-bit: lslab::map<K, unsigned>'s
 * get<bs> (include/lslab/map.h:208-211), put<bs> SoA and AoS (map.h:198-201,
 * 189-192) and update<bs> (map.h:217-220, update-if-present as above).  The
 * table stores the values zero-extended, so the 64-bit calls read them too;
 * values above 2^32 - 1 stored through the 64-bit calls come back truncated
 * here. */
int lsb_map_get_v32(lsb_map* m, const uint64_t* keys, lsb_result32* out, size_t n,
                    cudaStream_t stream);
int lsb_map_put_v32(lsb_map* m, const uint64_t* keys, const uint32_t* vals, uint32_t* old_out,
                    size_t n, cudaStream_t stream);
int lsb_map_put_pairs_v32(lsb_map* m, const lsb_kv32* ops, uint32_t* old_out, size_t n,
                          cudaStream_t stream);
int lsb_map_update_v32(lsb_map* m, const lsb_kv32* ops, lsb_result32* out, size_t n,
                       cudaStream_t stream);

/* Map remove: the REMOVE branch of detail::traverse
 * (include/lslab/detail/traverse.h:88-91), which the reference map does not
 * expose.  out[i] = {found, old value or 0}; out may be NULL. */
int lsb_map_remove(lsb_map* m, const uint64_t* keys, lsb_result* out, size_t n,
                   cudaStream_t stream);

/* Mixed batch (types[i] in LSB_OP_GET/PUT/REMOVE/UPDATE), run as internal
 * windows of per-phase launches.  vals is read for puts and updates only and
 * may be NULL when the batch has none.  out[i] as described at lsb_result
 * (an update: {present before it, old value or 0}); may be NULL. */
int lsb_map_execute(lsb_map* m, const uint8_t* types, const uint64_t* keys,
                    const uint64_t* vals, lsb_result* out, size_t n, cudaStream_t stream);

/* The same batch through one persistent cooperative launch (every phase of
 * every window inside one kernel, grid-wide barriers between phases). */
int lsb_map_execute_fused(lsb_map* m, const uint8_t* types, const uint64_t* keys,
                          const uint64_t* vals, lsb_result* out, size_t n,
                          cudaStream_t stream);

/* lslab::map::buckets(), include/lslab/map.h:225-227. */
uint32_t lsb_map_buckets(const lsb_map* m);

/* Launch tuning (no reference counterpart: the reference fixes the launch as a
 * template block size, include/lslab/map.h:189-220). */
int lsb_map_get_tuning(const lsb_map* m, lsb_tuning* out);
int lsb_map_set_tuning(lsb_map* m, const lsb_tuning* t);

/* Phase tracing of the fused path (no reference counterpart; the reference
 * only brackets whole launches with cudaProfilerStart/Stop,
 * benchmark/benchmark.cu:91,119).  With tracing on, each fused launch records
 * one %globaltimer stamp per phase boundary per window: entry = ns << 8 |
 * (window & 63) << 2 | phase, phase 0 window start, 1 probe done, 2 ordering
 * done, 3 resolve done.  read_trace copies the last launch's entries to host
 * memory (synchronises the stream).  When the last call ran two-stream
 * windows (tuning overlap), the entries come from timing events instead, ns
 * counted from the first window's start, for each window (< 16, window field
 * = window & 31): phase 0 start, 1 read kernel done, 2 mutation steps
 * (listing, probing, ordering) done, 3 resolve done, and with window field
 * | 32: phase 1 listing done, phase 2 probing done.  Calls issued while the
 * stream is being captured record none. */
int lsb_map_set_trace(lsb_map* m, int on);
int lsb_map_read_trace(lsb_map* m, uint64_t* out, size_t cap, size_t* count,
                       cudaStream_t stream);

/* Device status bits seen since the last call (synchronises the stream),
 * then clears them. */
int lsb_map_status(lsb_map* m, uint32_t* flags, cudaStream_t stream);

/* Overflow slabs in use (handed out and not returned by compaction), and
 * the pool's capacity (synchronises the stream). */
int lsb_map_pool_usage(lsb_map* m, uint64_t* used, uint64_t* capacity, cudaStream_t stream);

/* Number of live entries (synchronises the stream). */
int lsb_map_size(lsb_map* m, uint64_t* count, cudaStream_t stream);

/* Compaction, the slab reclamation the reference lacks (its deallocate is a
 * no-op, include/lslab/detail/device_allocator.h:73, and it reuses no slot
 * outside a chain's tail slab, include/lslab/detail/traverse.h:54-55).  Each
 * chain's live entries move into as few slabs as hold them, removed slots
 * become empty, and the emptied overflow slabs go back to the pool, which
 * hands them out again before any fresh slab.  (Inserts also reuse removed
 * slots in place, except in LSB_LOCK_FREE maps.)  Like a mutating call it
 * must be stream-ordered with every other call on the table.  *freed
 * (optional; synchronises the stream) receives the slabs returned. */
int lsb_map_compact(lsb_map* m, uint64_t* freed, cudaStream_t stream);

/* Number of live entries, written to *count_out, a DEVICE word the caller
 * provides, asynchronously on `stream`, without allocating any memory (no
 * counterpart in the reference: it is the allocation-free form of
 * lsb_map_size for callers that must not allocate, e.g. while recording a
 * stream capture or under a fully pre-reserved memory budget).  Its scratch is
 * one static device array shared by all calls: maps of at most 2^20 buckets
 * (larger ones return LSB_ERR_ARG); calls that overlap on the GPU race on the
 * array; the first call on each device resolves the array's address and
 * should come before any stream capture (the address is cached for the
 * process: do not use the library on a device again after cudaDeviceReset).
 * The current device must be the map's own device (else LSB_ERR_ARG). */
int lsb_map_size_noalloc(lsb_map* m, uint64_t* count_out, cudaStream_t stream);

/* Copy every live (key, value) pair to HOST arrays, in key order.  *count
 * receives the number of live entries; at most cap pairs are written.
 * Synchronises the stream. */
int lsb_map_dump(lsb_map* m, uint64_t* keys_out, uint64_t* vals_out, size_t cap,
                 uint64_t* count, cudaStream_t stream);

/* ---- checkpoints --------------------------------------------------------
 * No reference counterpart (lslab has no persistence).  save writes the
 * table's live entries as records sorted by key (map: u64 key, u64 value;
 * set: u32 key) after a 56-byte header (magic "LSBCKPT1", version, container,
 * log2 buckets, key and value bytes, lock mode, pool slabs, record count, and
 * a checksum of the records); the format does not depend on the slab layout
 * or bucket count.  load creates a table (the saved shape, or `opt` when not
 * NULL; a zero opt->pool_slabs takes the saved pool size) and inserts the
 * records; it returns LSB_ERR_IO for a missing, truncated or corrupt file
 * (bad magic, version, container, count or checksum) and creates nothing.
 * Both synchronise `stream`. */
int lsb_map_save(lsb_map* m, const char* path, cudaStream_t stream);
int lsb_map_load(const char* path, const lsb_options* opt, lsb_map** out, cudaStream_t stream);
int lsb_set_save(lsb_set* s, const char* path, cudaStream_t stream);
int lsb_set_load(const char* path, const lsb_options* opt, lsb_set** out, cudaStream_t stream);

/* ---- set<uint32_t> ---------------------------------------------------
 * Replaces lslab::set<K>::set(n_log_2) (include/lslab/set.h:31-40) and
 * set(n_log_2, Allocator&&) (include/lslab/set.h:42-51). */
int lsb_set_create(unsigned log2_buckets, uint64_t pool_slabs, lsb_set** out);
int lsb_set_create_ex(unsigned log2_buckets, const lsb_options* opt, lsb_set** out);
int lsb_set_destroy(lsb_set* s);

/* lslab::set::insert<bs>(const K*, bool*, size_t, cudaStream_t),
 * include/lslab/set.h:103-106 -> set_kernels::insert_, set_kernels.h:47-63.
 * Like the reference, out[i] is true for a new AND for an existing key
 * (include/lslab/detail/traverse.h:204-212,226-232). */
int lsb_set_insert(lsb_set* s, const uint32_t* keys, bool* out, size_t n, cudaStream_t stream);

/* lslab::set::contains<bs>, include/lslab/set.h:92-95 -> set_kernels.h:28-44. */
int lsb_set_contains(lsb_set* s, const uint32_t* keys, bool* out, size_t n,
                     cudaStream_t stream);

/* lslab::set::remove<bs>, include/lslab/set.h:114-117 -> set_kernels.h:10-26.
 * out[i] = the key was present. */
int lsb_set_remove(lsb_set* s, const uint32_t* keys, bool* out, size_t n, cudaStream_t stream);

/* Mixed set batch (types[i] in LSB_OP_CONTAINS/INSERT/REMOVE). */
int lsb_set_execute(lsb_set* s, const uint8_t* types, const uint32_t* keys, bool* out,
                    size_t n, cudaStream_t stream);
int lsb_set_execute_fused(lsb_set* s, const uint8_t* types, const uint32_t* keys, bool* out,
                          size_t n, cudaStream_t stream);

uint32_t lsb_set_buckets(const lsb_set* s); /* lslab::set::buckets(), set.h:125-127 */
int lsb_set_get_tuning(const lsb_set* s, lsb_tuning* out);
int lsb_set_set_tuning(lsb_set* s, const lsb_tuning* t);
int lsb_set_set_trace(lsb_set* s, int on);
int lsb_set_read_trace(lsb_set* s, uint64_t* out, size_t cap, size_t* count,
                       cudaStream_t stream);
int lsb_set_status(lsb_set* s, uint32_t* flags, cudaStream_t stream);
int lsb_set_pool_usage(lsb_set* s, uint64_t* used, uint64_t* capacity, cudaStream_t stream);
int lsb_set_size(lsb_set* s, uint64_t* count, cudaStream_t stream);
int lsb_set_compact(lsb_set* s, uint64_t* freed, cudaStream_t stream); /* as lsb_map_compact */
int lsb_set_dump(lsb_set* s, uint32_t* keys_out, size_t cap, uint64_t* count,
                 cudaStream_t stream);

/* ---- batching: CUDA graphs and the autotuner ---------------------------
 * No reference counterpart (the reference launches one kernel per op-type
 * batch, include/lslab/map.h:189-220).  A batch may be any concatenation of
 * smaller batches: results equal running them one after another. */
typedef struct lsb_graph lsb_graph;

/* Capture lsb_map_execute_fused on these buffers into an instantiated CUDA
 * graph (one cooperative kernel; its counters are left zero by the previous
 * launch, so no memset precedes it).  Each lsb_graph_launch runs
 * the batch currently in the buffers; the window epochs live on the device,
 * so replays never reuse one. */
int lsb_map_capture_fused(lsb_map* m, const uint8_t* types, const uint64_t* keys,
                          const uint64_t* vals, lsb_result* out, size_t n, lsb_graph** graph);
int lsb_set_capture_fused(lsb_set* s, const uint8_t* types, const uint32_t* keys, bool* out,
                          size_t n, lsb_graph** graph);
int lsb_graph_launch(lsb_graph* g, cudaStream_t stream);
int lsb_graph_destroy(lsb_graph* g);

/* Autotuner: times the fused path on a sample batch for every block size
 * (128, 256, 512, 1024 threads = 4, 8, 16, 32 warps), lookahead (0, 1, 2)
 * and probe order: mutations listed and probed first, reads meanwhile and
 * after; or all ops in one pass with the probe's claim size static, 32, 128,
 * 512, 1024, 2048 or 4096 ops; the median of three timings each.  It
 * keeps the fastest on the table
 * and in a process-wide cache by table size that tables created later with
 * the same log2_buckets start from.  The sample is applied once per
 * candidate: the final table contents equal one application (a key's final
 * state is its last mutation in the batch), `out` is scratch.  Synchronises
 * the stream. */
int lsb_map_autotune(lsb_map* m, const uint8_t* types, const uint64_t* keys,
                     const uint64_t* vals, lsb_result* out, size_t n, cudaStream_t stream,
                     lsb_tuning* best);
int lsb_set_autotune(lsb_set* s, const uint8_t* types, const uint32_t* keys, bool* out,
                     size_t n, cudaStream_t stream, lsb_tuning* best);
/* container: 0 map, 1 set.  LSB_ERR_STATE when that size was never tuned. */
int lsb_autotune_lookup(int container, unsigned log2_buckets, lsb_tuning* out);

/* ---- serving: a device-resident request loop over one map ---------------
 * No counterpart in the reference (lslab only has batched host calls); this
 * is the KV-store serving form.  lsb_serve_start launches one persistent
 * kernel that admits waves of queued requests in FIFO order (continuous
 * batching: requests that arrive while a wave runs join the next one), runs
 * each wave through the same engine as lsb_map_execute_fused and publishes
 * completions.  A wave admits the longest queue prefix that fits
 * max_wave_ops and whose worst-case new slabs (one per put) fit the pool's
 * free slabs; a request that can never fit (slabs are not returned to the
 * pool) completes with status LSB_ERR_OOM and no effect.  Ops of a wave run
 * in request order, so results equal running the requests one after another
 * in submission order.  Requests, ops and results live in GPU-mapped pinned
 * host memory; the table and each wave's working copy stay in device memory.
 * While the loop runs, no other call may use the map.  The loop ends on
 * lsb_serve_stop (after draining the queue) or after idle_ms without
 * requests. */
typedef struct lsb_server lsb_server;

typedef struct lsb_serve_options {
  uint32_t max_wave_ops;  /* ops per wave; 0 = 2^16; at most the map's max_window */
  uint32_t ring_requests; /* request slots; 0 = 16384 */
  uint64_t arena_ops;     /* ops the host-mapped arena holds; 0 = 2^22 */
  uint32_t idle_ms;       /* loop ends after about this long without requests; 0 = 10000 */
  uint32_t pad;
} lsb_serve_options;

typedef struct lsb_serve_stats {
  uint64_t waves;     /* waves run */
  uint64_t ops;       /* ops run */
  uint64_t requests;  /* requests completed (refused ones included) */
  uint32_t state;     /* 0 never ran, 1 running, 2 drained after stop, 3 idle limit,
                         4 a grid barrier gave up (see lsb_map_status) */
  uint32_t pad;
  /* Device time of the loop by step, ns summed over all waves (one device
   * thread's %globaltimer): gathering a wave's ops from the host-mapped
   * arena; the engine (probe, ordering, resolve); the tail (the rest of the
   * resolve, admitting the next wave, the last barrier); waiting for
   * requests while the queue was empty. */
  uint64_t gather_ns;
  uint64_t engine_ns;
  uint64_t tail_ns;
  uint64_t wait_ns;
} lsb_serve_stats;

int lsb_serve_create(lsb_map* m, const lsb_serve_options* opt, lsb_server** out);
/* Launches the loop on the server's own stream. */
int lsb_serve_start(lsb_server* s);
/* Queues one request of n ops (host pointers; types NULL = all gets, vals
 * NULL = zeros).  LSB_ERR_STATE when the queue or arena is full: take
 * results of finished requests, then retry.  *ticket numbers requests from 0. */
int lsb_serve_submit(lsb_server* s, const uint8_t* types, const uint64_t* keys,
                     const uint64_t* vals, uint32_t n, uint64_t* ticket);
/* *done = 1 once the request has finished. */
int lsb_serve_poll(lsb_server* s, uint64_t ticket, int* done);
/* Copies a finished request's n results to host memory `out` (may be NULL)
 * and its status (LSB_OK or LSB_ERR_OOM) to *status, then frees its slot.
 * Once per ticket; LSB_ERR_STATE when it has not finished. */
int lsb_serve_take(lsb_server* s, uint64_t ticket, lsb_result* out, int* status);
/* Drains the queue, ends the loop, waits for it.  Synchronises. */
int lsb_serve_stop(lsb_server* s, lsb_serve_stats* stats);
/* The loop's counters so far, read while it runs (no synchronisation; each
 * field is as of the last completed wave).  Differences of two snapshots
 * give the counts and step times of the waves in between.  No reference
 * counterpart (serving has none). */
int lsb_serve_query(lsb_server* s, lsb_serve_stats* stats);
int lsb_serve_destroy(lsb_server* s);

/* Open-loop load generator for the serving benchmark: issues nreq requests
 * at scheduled times (request i repeats pooled request pool_index[i] and is
 * due at start + arrival_ns[i]; a full queue delays issue, not the schedule),
 * takes every result on a second thread and writes each request's latency
 * (scheduled arrival to observed completion, ns) to latency_ns[i].
 * results (optional) receives every issued request's results in issue order.
 * The loop must be running.  Returns the wall time of the run in *wall_ns. */
typedef struct lsb_serve_load {
  uint64_t nreq;
  const uint64_t* arrival_ns;
  const uint32_t* pool_index;
  uint32_t pool_size;
  uint32_t pad;
  const uint64_t* pool_off; /* first op of each pooled request in the arrays below */
  const uint32_t* pool_n;   /* ops of each pooled request */
  const uint8_t* types;
  const uint64_t* keys;
  const uint64_t* vals;
  lsb_result* results;
} lsb_serve_load;
int lsb_serve_run_load(lsb_server* s, const lsb_serve_load* load, uint64_t* latency_ns,
                       uint64_t* wall_ns);

/* ---- KV store: variable-size byte values --------------------------------
 * A caller layer over the map (no counterpart in the reference library; its
 * KVCG tests keep value pointers in the map, test/slabunified_test.cu:
 * 360-380): values live in one device byte heap of heap_bytes (at most 2^40),
 * the map holds key -> heap offset and length (values up to 2^24 - 1 bytes).
 * All arrays are device memory; calls are stream-ordered like the map's. */
typedef struct lsb_kvs lsb_kvs;
int lsb_kvs_create(unsigned log2_buckets, uint64_t heap_bytes, const lsb_options* opt,
                   lsb_kvs** out);
int lsb_kvs_destroy(lsb_kvs* s);
/* The map underneath (for lsb_map_size, _status, _compact...). */
lsb_map* lsb_kvs_map(lsb_kvs* s);
/* Put n values: op i's bytes are vals[val_off[i] .. val_off[i+1]) (n + 1
 * offsets, non-decreasing).  Ops run in index order; the space of a replaced
 * value becomes garbage (lsb_kvs_usage) until lsb_kvs_compact.  LSB_ERR_OOM
 * (no effect) when the heap cannot take the batch; LSB_ERR_ARG when a value
 * is too long.  Synchronises the stream (the batch's size is read). */
int lsb_kvs_put(lsb_kvs* s, const uint64_t* keys, const uint8_t* vals, const uint64_t* val_off,
                size_t n, cudaStream_t stream);
/* Get n values: found_out[i] (optional) = the key is present, len_out[i] =
 * the value's length (0 when absent), dst_off_out[i] = its offset in dst (the
 * exclusive prefix sums of the lengths), and the bytes copied to dst when it
 * is not NULL (values that would end past dst_cap are not copied).
 * *total_out (optional; synchronises) receives the bytes all found values
 * need. */
int lsb_kvs_get(lsb_kvs* s, const uint64_t* keys, uint8_t* found_out, uint32_t* len_out,
                uint64_t* dst_off_out, uint8_t* dst, uint64_t dst_cap, size_t n,
                uint64_t* total_out, cudaStream_t stream);
/* Remove n keys; found_out[i] (optional) = the key was present. */
int lsb_kvs_remove(lsb_kvs* s, const uint64_t* keys, uint8_t* found_out, size_t n,
                   cudaStream_t stream);
/* Heap bytes handed out, bytes of replaced or removed values among them, and
 * the capacity (synchronises). */
int lsb_kvs_usage(lsb_kvs* s, uint64_t* heap_used, uint64_t* heap_dead, uint64_t* heap_cap,
                  cudaStream_t stream);
/* Move the live values to the front of the heap (key order) and drop the
 * garbage; must not overlap other calls on the store.  Synchronises. */
int lsb_kvs_compact(lsb_kvs* s, cudaStream_t stream);

/* ---- device per-warp API -------------------------------------------------
 * The device methods of the reference (map::get/put/update, map.h:92-183;
 * set::contains/insert/remove, set.h:64-90) are in include/lsb_device.cuh,
 * used from a caller's own kernels on a view of a table's device memory.
 * The view is plain data: pass it to kernels by value.  It stays valid until
 * the table is destroyed. */
typedef struct lsb_table_view {
  void* slabs;
  int32_t* locks;
  uint32_t* status;
  uint64_t* pool;
  uint32_t* free_stack;
  uint32_t mask;
  uint32_t lock_mode;
  uint32_t chunk;
  uint32_t pad;
} lsb_table_view;
int lsb_map_device_view(const lsb_map* m, lsb_table_view* out);
int lsb_set_device_view(const lsb_set* s, lsb_table_view* out);

/* ---- measuring ---------------------------------------------------------- */
/* Probe-rate calibration (no reference counterpart): for i < n, read req[i],
 * pick a slab of the array `slabs` (nslabs slabs of slab_bytes each)
 * uniformly at random, load its 32-byte meta sector, then, dependent on it,
 * one 16-byte slot of the same slab, and store 16 bytes to out[2i..2i+1]: the
 * accesses of one get at a uniformly random key and nothing else.  Its rate
 * is the ceiling that address translation and DRAM latency put on random
 * lookups over an array of that size (pass a table's slab array from
 * lsb_*_device_view; only reads it).  Async on `s`. */
int lsb_probe_calibrate(const void* slabs, uint64_t nslabs, uint32_t slab_bytes,
                        const uint64_t* req, uint64_t* out, size_t n, uint64_t seed,
                        cudaStream_t s);

/* ---- misc ------------------------------------------------------------- */
const char* lsb_error_string(int code);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int lsb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LSB_H */
