/* Test infrastructure, not product code: the CPU oracle.
 *
 * A plain-C restatement of the reference library's slab-list hash map and
 * set (depaulmillz/lslab), run sequentially in op-index order.  It is the
 * checker for the CUDA path (tests/, __graft_entry__.smoke) and the timed CPU
 * baseline in bench.py; nothing in the product links or calls it.
 *
 * Pinned against outputs of the reference's own kernels built for sm_100a
 * (oracle/_ref, fixtures under tests/golden/) and against the reference's own
 * known-answer tests (test/set_test.cu:40-81, test/slabunified_test.cu:42-89).
 */
#ifndef LSB_ORACLE_H
#define LSB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Op codes of a mixed batch (same numbering as the product's lsb.h). */
enum { ORC_GET = 0, ORC_PUT = 1, ORC_REMOVE = 2, ORC_UPDATE = 3 };
enum { ORC_CONTAINS = 0, ORC_INSERT = 1, ORC_SET_REMOVE = 2 };

/* 16-byte result, layout of cuda::std::pair<bool, uint64_t>. */
typedef struct {
  uint8_t found;
  uint8_t pad[7];
  uint64_t value;
} orc_result;

typedef struct orc_map orc_map;
typedef struct orc_set orc_set;

orc_map* orc_map_create(unsigned log2_buckets, uint64_t pool_capacity);
void orc_map_destroy(orc_map* m);
void orc_map_get(orc_map* m, const uint64_t* keys, orc_result* out, size_t n);
void orc_map_put(orc_map* m, const uint64_t* keys, const uint64_t* vals, uint64_t* old_out,
                 size_t n);
void orc_map_remove(orc_map* m, const uint64_t* keys, orc_result* out, size_t n);
/* Update-if-present: {1, old value} and the new value stored, or {0, 0}. */
void orc_map_update(orc_map* m, const uint64_t* keys, const uint64_t* vals, orc_result* out,
                    size_t n);
/* Mixed batch in op-index order (types ORC_GET/PUT/REMOVE/UPDATE); put and
 * update results report {existed, old value or 0}. */
void orc_map_mixed(orc_map* m, const uint8_t* types, const uint64_t* keys,
                   const uint64_t* vals, orc_result* out, size_t n);
/* Same, with ops sharded by bucket over `threads` host threads; each thread
 * walks the whole stream in index order and applies the ops of its buckets,
 * so every result equals the single-threaded one. */
int orc_map_mixed_mt(orc_map* m, const uint8_t* types, const uint64_t* keys,
                     const uint64_t* vals, orc_result* out, size_t n, int threads);
size_t orc_map_size(const orc_map* m);
/* Writes all live (key, value) pairs, unsorted; returns the count. */
size_t orc_map_dump(const orc_map* m, uint64_t* keys_out, uint64_t* vals_out, size_t cap);
uint64_t orc_map_slabs_used(const orc_map* m);
int orc_map_error(const orc_map* m);

orc_set* orc_set_create(unsigned log2_buckets, uint64_t pool_capacity);
void orc_set_destroy(orc_set* s);
void orc_set_insert(orc_set* s, const uint32_t* keys, uint8_t* out, size_t n);
void orc_set_contains(orc_set* s, const uint32_t* keys, uint8_t* out, size_t n);
void orc_set_remove(orc_set* s, const uint32_t* keys, uint8_t* out, size_t n);
void orc_set_mixed(orc_set* s, const uint8_t* types, const uint32_t* keys, uint8_t* out,
                   size_t n);
int orc_set_mixed_mt(orc_set* s, const uint8_t* types, const uint32_t* keys, uint8_t* out,
                     size_t n, int threads);
size_t orc_set_size(const orc_set* s);
size_t orc_set_dump(const orc_set* s, uint32_t* keys_out, size_t cap);
uint64_t orc_set_slabs_used(const orc_set* s);
int orc_set_error(const orc_set* s);

#ifdef __cplusplus
}
#endif
#endif
