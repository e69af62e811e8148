/*
 * hg_oracle.h -- CPU oracle for the HashGraph build + intersect path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: a plain-C restatement of the
 * reference's algorithm (alokpathy/hashgraph), used by tests/, by
 * __graft_entry__.smoke() and by the CPU-baseline leg of bench.py.  Nothing in
 * the product library links, loads or calls it.
 *
 * Parity is pinned by tests/golden/: murmur known answers produced by the
 * reference's own hash_murmur compiled on the host (oracle/ref_hash_driver.cpp),
 * and CSR / intersect outputs produced by the reference's MultiHashGraph run on
 * a B200 (oracle/ref_multi_driver.cu).
 */
#ifndef HG_ORACLE_H
#define HG_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* murmur3_x86_32 of the low 4 bytes of the key, seed 0
 * (reference include/SingleHashGraphOperators.cuh:18-69). */
uint32_t or_murmur3_low32(uint64_t key);
/* bucket = murmur % n_buckets  (reference SingleHashGraphOperators.cuh:76,
 * MultiHashGraphDeviceOperators.cuh:81). */
uint64_t or_bucket(uint64_t key, uint64_t n_buckets);
void or_buckets(const void* keys, uint64_t n, int key_bytes, uint64_t n_buckets, uint64_t* out);

/* Lemire-Kaser-Kurz "fastmod" (2019) restated for checking the device form. */
uint64_t or_fastmod_magic(uint32_t d);
uint32_t or_fastmod(uint32_t a, uint64_t magic, uint32_t d);

/* Seeded counter-based generators (the workload definitions). */
uint64_t or_mix64(uint64_t x);
uint64_t or_rand64(uint64_t seed, uint64_t stream, uint64_t i);
uint64_t or_perm(uint64_t i, uint64_t n, uint64_t seed);
void or_gen_uniform(void* out, uint64_t n, int key_bytes, uint64_t seed);
void or_gen_overlap(void* out, uint64_t n, int key_bytes, const void* a_keys, uint64_t n_a,
                    double frac, uint64_t seed);
int or_zipf_cdf(uint64_t* cdf, uint64_t universe, double s);
void or_gen_zipf(void* out, uint64_t n, int key_bytes, const uint64_t* cdf, uint64_t universe,
                 uint64_t seed);

/* Stable counting-sort CSR build: offsets[n_buckets+1], keys_out[n],
 * idx_out[n] (input position; may be NULL).  Reference semantics:
 * src/SingleHashGraph.cu:187-213 and include/MultiHashGraphHostOperators.cuh:316-343. */
int or_build(const void* keys, uint64_t n, int key_bytes, uint64_t n_buckets,
             uint32_t* offsets, void* keys_out, uint32_t* idx_out);
/* Same result, multithreaded (the CPU baseline). */
int or_build_mt(const void* keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                uint32_t* offsets, void* keys_out, uint32_t* idx_out, int threads);
/* Sort every bucket by (key, idx): the canonical form used for parity. */
void or_canonicalize(const uint32_t* offsets, uint64_t n_buckets, void* keys, int key_bytes,
                     uint32_t* idx);

/* Probe intersect of queries against table A (bucket-aligned multiset join;
 * reference include/MultiHashGraphDeviceOperators.cuh:513-543).  Returns the
 * match count; writes up to pair_cap pairs (a_ref, q_ref) where a_ref is
 * a_idx[j] (or the CSR position j when a_idx is NULL) and q_ref is q_idx[i]
 * (or the query position i). */
uint64_t or_intersect(const uint32_t* a_offsets, uint64_t n_buckets, const void* a_keys,
                      const uint32_t* a_idx, int key_bytes, const void* q_keys, uint64_t nq,
                      const uint32_t* q_idx, uint32_t* pairs, uint64_t pair_cap);
uint64_t or_intersect_mt(const uint32_t* a_offsets, uint64_t n_buckets, const void* a_keys,
                         const uint32_t* a_idx, int key_bytes, const void* q_keys, uint64_t nq,
                         uint32_t* pairs, uint64_t pair_cap, int threads);
/* sum_k multA(k) * multB(k) by sort-merge (reference test/MultiHashGraphTest.cu:340-425
 * restated as sort + merge-join). */
uint64_t or_join_count_sorted(const void* a_sorted, uint64_t na, const void* b_sorted,
                              uint64_t nb, int key_bytes);
/* The same count through a hash map of A's distinct keys (at most
 * max_distinct of them): linear time for skewed inputs.  UINT64_MAX if the map
 * cannot be allocated or fills. */
uint64_t or_join_count_hashed(const void* a, uint64_t na, const void* b, uint64_t nb, int key_bytes,
                              uint64_t max_distinct, int threads);
int or_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
