/*
 * hashgraph_b200.h -- C ABI of the B200 (sm_100a) HashGraph build + intersect path.
 *
 * A HashGraph is a hash table stored as a CSR graph: bucket b of a table with
 * n_buckets buckets holds the keys whose murmur3_x86_32 hash (of the key's low
 * 32 bits, seed 0) modulo n_buckets equals b.  The table is three SoA arrays in
 * device memory:
 *     offsets[n_buckets + 1]  uint32   bucket b is [offsets[b], offsets[b+1])
 *     keys[n]                 uint32 or uint64 (key_bytes 4 or 8)
 *     idx[n]                  uint32   input position of each key (optional)
 *
 * Conventions for every entry point:
 *   - All device pointers are plain CUDA device addresses; no framework types.
 *   - Calls are stream-ordered and asynchronous on `stream` (NULL = legacy
 *     default stream) unless stated; the returned status covers argument
 *     checks and launch errors.  Failures detected on the device (a bounded
 *     wait that ran out, a pair buffer too small) are recorded in a per-device
 *     error word read by hg_device_error().
 *   - Nothing the caller owns is freed or resized.  Buffers the library
 *     allocates belong to an hg_table and are released by hg_table_free().
 *   - n < 2^32, 1 <= n_buckets <= 2^32.
 *
 * Reference interfaces replaced (alokpathy/hashgraph, path:line):
 *   SingleHashGraph::build               src/SingleHashGraph.cu:216-232
 *   MultiHashGraph::build (gpuCount = 1) src/MultiHashGraph.cu:408-629
 *   MultiHashGraph::intersect            src/MultiHashGraph.cu:631-740
 *   hash_murmur                          include/SingleHashGraphOperators.cuh:31-69
 * The C++ classes of include/hashgraph_b200/ keep the reference's class API on
 * top of these calls.
 */
#ifndef HASHGRAPH_B200_H
#define HASHGRAPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* hg_stream_t;
typedef int32_t hg_status;

#define HG_OK                   0
#define HG_ERR_INVALID_ARGUMENT (-1)
#define HG_ERR_CUDA             (-2)
#define HG_ERR_OUT_OF_MEMORY    (-3)
#define HG_ERR_PAIR_CAPACITY    (-4) /* more matches than pair_cap: count is exact, pairs truncated */
#define HG_ERR_DEVICE_TIMEOUT   (-5) /* a bounded device-side wait gave up */
#define HG_ERR_TOO_LARGE        (-6) /* n >= 2^32 or n_buckets > 2^32, or workspace too small */
#define HG_ERR_NO_DEVICE        (-7)
#define HG_ERR_KEY_WIDTH        (-8) /* key_bytes not 4 or 8, or tables of different key width */
#define HG_ERR_BUCKET_MISMATCH  (-9) /* tables built with different n_buckets */
#define HG_ERR_DEVICE_STATE     (-10) /* a kernel found a position outside its output (device state
                                        * inconsistent, e.g. after a wait that gave up) and wrote nothing */

/* Human-readable text for a status code (static storage). */
const char* hg_status_str(hg_status status);

/* Library version, e.g. "hashgraph_b200 0.1 sm_100a". */
const char* hg_version(void);

/* Description of the last failure inside the library on this host thread
 * (the call site and the CUDA error string), or "" (thread-local storage). */
const char* hg_last_error(void);

/* Host form of the bucket hash: murmur3_x86_32 of the low 32 bits of `key`,
 * seed 0.  Replaces the __host__ side of hash_murmur
 * (include/SingleHashGraphOperators.cuh:31-69). */
uint32_t hg_hash(uint64_t key);

/* Reads (then clears) the per-device error words after synchronising `stream`.
 * *code receives HG_OK, the fault (HG_ERR_DEVICE_TIMEOUT: a bounded device-side
 * wait gave up; HG_ERR_DEVICE_STATE: a position outside its output) when one
 * was recorded, else the first HG_ERR_* recorded by a kernel (for instance
 * HG_ERR_PAIR_CAPACITY).  After a fault every kernel of the library on the
 * device returns at entry, writing nothing, until this call clears it: every
 * result produced since the fault is invalid.  The reference has no device
 * error path (it prints and calls exit(0), include/MultiHashGraph.cuh:56-57). */
hg_status hg_device_error(hg_stream_t stream, hg_status* code);

/* Test hook (no counterpart in the reference): the number of polls a
 * decoupled look-back makes before it gives up and records
 * HG_ERR_DEVICE_TIMEOUT.  0 restores the default (2^22).  Lowering it makes
 * the bounded wait run out on purpose, to test the error path. */
hg_status hg_debug_set_wait_limit(uint32_t polls, hg_stream_t stream);

/* ------------------------------------------------------------------------
 * Build with caller-owned outputs and workspace.
 * ---------------------------------------------------------------------- */

/* Device scratch bytes hg_build_into needs for this shape. */
hg_status hg_build_workspace_size(uint64_t n, int key_bytes, uint64_t n_buckets, int with_index,
                                  size_t* bytes);

/* Builds the CSR of `d_keys` (n keys of key_bytes each) into caller buffers.
 * d_offsets: n_buckets+1 uint32; d_keys_out: n keys; d_idx_out: n uint32 or
 * NULL (no index).  Replaces SingleHashGraph::build (src/SingleHashGraph.cu:216-232:
 * hashValuesD, lrbCountHashD, scans, lrbRehashD, lrbCountHashGlobalD,
 * lrbCopyToGraphD) and the per-GPU build of MultiHashGraph::build
 * (src/MultiHashGraph.cu:408-629, lrbBuildMultiTable :303-375).  Bucket
 * contents are the reference's; the order inside a bucket is unspecified,
 * as in the reference. */
hg_status hg_build_into(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                        uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                        void* d_workspace, size_t workspace_bytes, hg_stream_t stream);

/* Same as hg_build_into / hg_build_workspace_size with the build path fixed:
 * path 0 = direct (one count pass with global per-bucket counters, a scan,
 * one scatter pass: the reference's non-LRB buildTable,
 * src/SingleHashGraph.cu:187-213), 1 = partitioned (bucket-range partition
 * pass, then one shared-memory build per partition: the role of the
 * reference's LRB build, src/SingleHashGraph.cu:129-181, chosen there by
 * #define LRB_BUILD, :64), -1 = planner's choice.  A table too dense for the
 * partitioned path's shared-memory staging (nearly all keys in a few buckets)
 * is built by the direct path even when path 1 is asked for. */
hg_status hg_build_workspace_size_path(uint64_t n, int key_bytes, uint64_t n_buckets, int with_index,
                                       int path, size_t* bytes);
hg_status hg_build_into_path(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                             uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                             void* d_workspace, size_t workspace_bytes, int path, hg_stream_t stream);

/* Allocation-free build (no counterpart in the reference).  For callers that
 * must not allocate device memory when they build a table: a process whose
 * HBM is handed out by its own pool allocator, code running inside another
 * allocator's callback, or a loop that forbids cudaMalloc after start-up.
 * Same arguments and result as hg_build_into on the direct path, but the
 * scratch is a fixed 64 KiB array inside this library (held on every GPU
 * that loads it), so n_buckets is limited to 2^25 = 33554432; larger values
 * return HG_ERR_TOO_LARGE.  The caller provides keys and outputs.  The first
 * call on a device looks up the array's device address; make it before any
 * stream capture.  All calls share the array: calls whose work overlaps on
 * the GPU race and must be serialised by the caller. */
hg_status hg_build_into_noalloc(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                                uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                                hg_stream_t stream);

/* ------------------------------------------------------------------------
 * Library-owned tables.
 * ---------------------------------------------------------------------- */
typedef struct hg_table hg_table;

/* Allocates a table able to hold up to `capacity` keys in n_buckets buckets,
 * with its build workspace.  No build happens. */
hg_status hg_table_create(uint64_t capacity, int key_bytes, uint64_t n_buckets, int with_index,
                          hg_table** out);

/* (Re)builds `table` from n <= capacity device keys. */
hg_status hg_table_build(hg_table* table, const void* d_keys, uint64_t n, hg_stream_t stream);

/* hg_table_create(n, ...) + hg_table_build. */
hg_status hg_build(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                   int with_index, hg_table** out, hg_stream_t stream);

/* Device views of a built table (any output pointer may be NULL). */
hg_status hg_table_view(const hg_table* table, const uint32_t** d_offsets, const void** d_keys,
                        const uint32_t** d_idx, uint64_t* n, uint64_t* n_buckets, int* key_bytes);

/* Bytes of device memory the table holds (arrays + workspace). */
hg_status hg_table_device_bytes(const hg_table* table, size_t* bytes);

void hg_table_free(hg_table* table);

/* ------------------------------------------------------------------------
 * Table files: a built table saved to disk and loaded back onto the current
 * device (no counterpart in the reference, whose tables live in one process).
 * Layout: a 64-byte header (magic "HGB2TBL", version 1, key width, index
 * flag, hash id, n, n_buckets, FNV-1a 64 checksum of the payload), then
 * offsets[n_buckets + 1] (uint32), keys[n], idx[n] (uint32, when indexed),
 * little-endian.  Loading checks the magic, version, sizes against the file
 * length, offsets[0] == 0, offsets[n_buckets] == n and the checksum.
 * The copies run on `stream` through a pinned staging buffer; the calls
 * return when the data is on disk / on the device.
 * ---------------------------------------------------------------------- */
hg_status hg_table_save(const hg_table* table, const char* path, hg_stream_t stream);
hg_status hg_table_load(const char* path, hg_table** out, hg_stream_t stream);
/* The same on caller-owned device arrays (d_idx NULL: no index saved). */
hg_status hg_table_save_arrays(const char* path, const uint32_t* d_offsets, const void* d_keys,
                               const uint32_t* d_idx, uint64_t n, uint64_t n_buckets, int key_bytes,
                               hg_stream_t stream);
/* Header of a table file (host only, no device work). */
hg_status hg_table_file_info(const char* path, uint64_t* n, uint64_t* n_buckets, int* key_bytes,
                             int* with_index);
/* Loads into caller-owned arrays sized by hg_table_file_info; n, n_buckets
 * and key_bytes must match the file's. */
hg_status hg_table_load_arrays(const char* path, uint32_t* d_offsets, void* d_keys, uint32_t* d_idx,
                               uint64_t n, uint64_t n_buckets, int key_bytes, hg_stream_t stream);

/* ------------------------------------------------------------------------
 * Intersect.  Multiset join on equal keys, bucket by bucket, as
 * MultiHashGraph::intersect (src/MultiHashGraph.cu:631-740, simpleIntersect
 * include/MultiHashGraphDeviceOperators.cuh:513-543): every (a, q) with
 * key(a) == key(q) is one match, so duplicates multiply.
 *
 * Pairs are written as uint32 [a_ref, q_ref] couples into d_pairs[2*pair_cap]:
 *   a_ref = A's idx[j] when A has an index, else the CSR position j in A;
 *   q_ref = d_query_idx[i] when given, else the query position i.
 * *d_count (uint64, device) receives the exact number of matches even when it
 * exceeds pair_cap; then only pair_cap pairs are written and the device error
 * word records HG_ERR_PAIR_CAPACITY.  d_pairs == NULL counts only.
 * ---------------------------------------------------------------------- */

/* Device scratch bytes for hg_intersect_into against a table of n_a keys
 * (with or without an index). */
hg_status hg_intersect_workspace_size(uint64_t n_a, int a_has_index, uint64_t n_buckets, uint64_t nq,
                                      int key_bytes, int emit_pairs, size_t* bytes);

/* Probes nq query keys (same key width as A) against table A. */
hg_status hg_intersect_into(const uint32_t* d_a_offsets, const void* d_a_keys,
                            const uint32_t* d_a_idx, uint64_t n_a, uint64_t n_buckets,
                            int key_bytes, const void* d_query, uint64_t nq,
                            const uint32_t* d_query_idx, uint32_t* d_pairs, uint64_t pair_cap,
                            unsigned long long* d_count, void* d_workspace,
                            size_t workspace_bytes, hg_stream_t stream);

/* Same with the probe path fixed: 0 = direct (every query reads its bucket
 * from A in HBM), 1 = partitioned (queries are split by bucket range, A's
 * slice of each range is staged in shared memory), 2 = coarse (queries are
 * grouped by bucket ranges whose slice of A fits in L2, and every range is
 * probed from L2), -1 = planner's choice.  As for the build, paths 1 and 2
 * fall back to the direct probe when the buckets are too few to split the
 * queries; any other value is HG_ERR_INVALID_ARGUMENT. */
hg_status hg_intersect_workspace_size_path(uint64_t n_a, int a_has_index, uint64_t n_buckets,
                                           uint64_t nq, int key_bytes, int emit_pairs, int path,
                                           size_t* bytes);
hg_status hg_intersect_into_path(const uint32_t* d_a_offsets, const void* d_a_keys,
                                 const uint32_t* d_a_idx, uint64_t n_a, uint64_t n_buckets,
                                 int key_bytes, const void* d_query, uint64_t nq,
                                 const uint32_t* d_query_idx, uint32_t* d_pairs, uint64_t pair_cap,
                                 unsigned long long* d_count, void* d_workspace,
                                 size_t workspace_bytes, int path, hg_stream_t stream);

/* Same, on an hg_table; allocates its scratch per call (stream-ordered). */
hg_status hg_intersect(const hg_table* a, const void* d_query, uint64_t nq,
                       const uint32_t* d_query_idx, uint32_t* d_pairs, uint64_t pair_cap,
                       unsigned long long* d_count, hg_stream_t stream);

/* Table-vs-table form of MultiHashGraph::intersect: the keys of B (in B's CSR
 * order) are the queries; q_ref is B's idx (or B's CSR position). */
hg_status hg_intersect_tables(const hg_table* a, const hg_table* b, uint32_t* d_pairs,
                              uint64_t pair_cap, unsigned long long* d_count, hg_stream_t stream);

/* ------------------------------------------------------------------------
 * Batched build + intersect: many independent (table, queries) pairs in one
 * launch sequence.  No counterpart in the reference, which builds and
 * intersects one MultiHashGraph at a time (test/MultiHashGraphTest.cu:288-338,
 * src/MultiHashGraph.cu:408-740); each pair's result equals the one
 * hg_build_into + hg_intersect_into would give it: the same offsets, the
 * same buckets, the same count and the same pairs (keys inside one bucket in
 * unspecified order, as for every build).  Pairs of 2^14 or more keys
 * (queries) whose buckets form at most 512 partitions of 2048 (4096)
 * buckets run in a partitioned form and emit their pairs grouped by
 * partition; the others emit them in query order.
 *
 * For each pair i: build table i from d_keys[0..n) into d_offsets
 * [n_buckets + 1], d_keys_out [n] and, when d_idx_out is not NULL, d_idx_out
 * [n] (input positions); then probe d_query[0..nq) against it: *d_count gets
 * the exact match count and, when d_pairs is not NULL, the first pair_cap
 * (a_ref, q_ref) pairs are written (a_ref = index or CSR position, q_ref =
 * query position).  A pair whose count exceeds pair_cap sets
 * HG_ERR_PAIR_CAPACITY in the device error word.  All pairs share the key
 * width.  Every pointer is device memory owned by the caller; the buffers
 * must not overlap between pairs.
 *
 * Probe-only and build-only pairs: a pair whose d_keys is NULL while n > 0
 * names a table already built (by hg_build_into, an earlier batch or a table
 * file) in d_offsets / d_keys_out / d_idx_out; the batch only probes it, and
 * it may be the table another pair of the same batch builds (every build of
 * a run finishes before its first probe).  A pair with nq = 0 is only built;
 * its d_count may then be NULL.  The serving engine coalesces its queued
 * requests into such batches.
 * ---------------------------------------------------------------------- */
typedef struct hg_batch_pair {
  const void* d_keys;
  uint64_t n;
  uint64_t n_buckets;
  const void* d_query;
  uint64_t nq;
  uint32_t* d_offsets;
  void* d_keys_out;
  uint32_t* d_idx_out;
  uint32_t* d_pairs;
  uint64_t pair_cap;
  unsigned long long* d_count;
} hg_batch_pair;

typedef struct hg_batch hg_batch;

/* Plans the batch (tile lists per kernel), allocates its device workspace
 * (stream-ordered) and uploads the pair descriptors on `stream`.  The
 * descriptors are copied: `pairs` may be reused after the call returns. */
hg_status hg_batch_create(const hg_batch_pair* pairs, int n_pairs, int key_bytes, hg_stream_t stream,
                          hg_batch** out);
/* Launches the batch's kernels on `stream` (a fixed sequence of at most
 * eleven launches and one memset, whatever the number of pairs).  Issues no
 * allocation, no host copy and no synchronisation, so it can be captured
 * into a CUDA graph and the graph replayed after the callers' input buffers
 * are refilled. */
hg_status hg_batch_run(const hg_batch* batch, hg_stream_t stream);
/* The size classes of a batch: pairs of at least part_min keys take the
 * partitioned build, and (queries) the L2 form of the probe when their whole
 * table (offsets, keys, index) is at most l2_table_bytes (0: never), the
 * partitioned probe otherwise; smaller pairs take the direct form. */
typedef struct hg_batch_params {
  uint64_t part_min;        /* default 2^14 */
  uint64_t l2_table_bytes;  /* default 24 MB */
} hg_batch_params;
hg_status hg_batch_params_default(hg_batch_params* params);
/* hg_batch_create with explicit size classes (params NULL: the defaults). */
hg_status hg_batch_create_params(const hg_batch_pair* pairs, int n_pairs, int key_bytes,
                                 const hg_batch_params* params, hg_stream_t stream, hg_batch** out);
/* Autotuner of the size classes: times candidate boundaries on this batch
 * (it runs the batch: the outputs hold its results) and returns the fastest
 * in *best and its time in *best_ms (optional).  Synchronises the stream. */
hg_status hg_batch_autotune(const hg_batch_pair* pairs, int n_pairs, int key_bytes, hg_stream_t stream,
                            hg_batch_params* best, float* best_ms);
/* Device bytes the batch holds (workspace and descriptors). */
hg_status hg_batch_device_bytes(const hg_batch* batch, size_t* bytes);
/* Frees the batch's device memory stream-ordered on `stream`. */
void hg_batch_free(hg_batch* batch, hg_stream_t stream);
/* create + run + free in one call. */
hg_status hg_batch_build_intersect(const hg_batch_pair* pairs, int n_pairs, int key_bytes, hg_stream_t stream);

/* ------------------------------------------------------------------------
 * One table sharded over several devices by bucket range: MultiHashGraph
 * with gpuCount > 1 (src/MultiHashGraph.cu:408-629 build, :631-740
 * intersect).  Shard r holds buckets [splits[r], splits[r+1]) of a table of
 * n_buckets; one process drives each device and the caller moves the routed
 * keys between devices with its own collective (an NCCL all-to-all).  A
 * shard's table is the global table's CSR restricted to its range:
 * offsets[b - lo] for b in [lo, hi], rebased to start at 0.
 * ---------------------------------------------------------------------- */
#define HG_MAX_SHARDS 64

/* Adds the bucket-id histogram of d_keys into d_bins[n_bins] (uint64):
 * bin = bucket / ceil(n_buckets / n_bins) -- countBinSizes,
 * include/MultiHashGraphDeviceOperators.cuh:153-163.  n_bins <= 32768. */
hg_status hg_shard_histogram(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                             uint32_t n_bins, unsigned long long* d_bins, hg_stream_t stream);
/* Host only: splits[0..n_shards] from the summed histogram of every
 * device's keys -- the reference's rule, include/MultiHashGraphHostOperators.cuh:80-88
 * (about n/n_shards keys per shard; splits[0] = 0, splits[n_shards] = n_buckets). */
hg_status hg_shard_splits(const unsigned long long* h_bins, uint32_t n_bins, uint64_t n_buckets,
                          int n_shards, uint64_t* h_splits);
/* Groups d_keys by destination shard (countKeyBuffSizes + binKeyValues,
 * include/MultiHashGraphDeviceOperators.cuh:220-246): d_keys_out holds
 * shard 0's keys, then shard 1's, ..., each group in input order;
 * d_idx_out (optional) the keys' global indices index_base + position;
 * d_shard_offsets[n_shards + 1] (uint64, device) the group boundaries.
 * `splits` is a host array. */
hg_status hg_shard_route_workspace_size(uint64_t n, int n_shards, size_t* bytes);
hg_status hg_shard_route(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                         const uint64_t* splits, int n_shards, uint32_t index_base, void* d_keys_out,
                         uint32_t* d_idx_out, unsigned long long* d_shard_offsets, void* d_workspace,
                         size_t workspace_bytes, hg_stream_t stream);
/* Builds the shard [bucket_lo, bucket_hi) of a table of n_buckets from keys
 * whose buckets all lie in that range (a shard's routed keys); d_offsets
 * holds bucket_hi - bucket_lo + 1 entries.  With d_idx_out, the index holds
 * d_key_idx[position] (the keys' global indices) when d_key_idx is given,
 * else the position.  Workspace: hg_build_workspace_size(n, key_bytes,
 * bucket_hi - bucket_lo, with_index). */
hg_status hg_shard_build_into(const void* d_keys, const uint32_t* d_key_idx, uint64_t n, int key_bytes,
                              uint64_t n_buckets, uint64_t bucket_lo, uint64_t bucket_hi,
                              uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                              void* d_workspace, size_t workspace_bytes, hg_stream_t stream);
/* Probes queries whose buckets lie in the shard's range against the shard
 * (as hg_intersect_into; q_ref = d_query_idx[i] when given).  Workspace:
 * hg_intersect_workspace_size(n_a, a_has_index, bucket_hi - bucket_lo, nq,
 * key_bytes, emit_pairs). */
hg_status hg_shard_intersect_into(const uint32_t* d_a_offsets, const void* d_a_keys, const uint32_t* d_a_idx,
                                  uint64_t n_a, uint64_t n_buckets, uint64_t bucket_lo, uint64_t bucket_hi,
                                  int key_bytes, const void* d_query, uint64_t nq, const uint32_t* d_query_idx,
                                  uint32_t* d_pairs, uint64_t pair_cap, unsigned long long* d_count,
                                  void* d_workspace, size_t workspace_bytes, hg_stream_t stream);
/* Internal: the same with an explicit path (-1 = planner's choice). */
hg_status hg_shard_build_into_path(const void* d_keys, const uint32_t* d_key_idx, uint64_t n, int key_bytes,
                                   uint64_t n_buckets, uint64_t bucket_lo, uint64_t bucket_hi,
                                   uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                                   void* d_workspace, size_t workspace_bytes, int path, hg_stream_t stream);
hg_status hg_shard_intersect_into_path(const uint32_t* d_a_offsets, const void* d_a_keys,
                                       const uint32_t* d_a_idx, uint64_t n_a, uint64_t n_buckets,
                                       uint64_t bucket_lo, uint64_t bucket_hi, int key_bytes,
                                       const void* d_query, uint64_t nq, const uint32_t* d_query_idx,
                                       uint32_t* d_pairs, uint64_t pair_cap, unsigned long long* d_count,
                                       void* d_workspace, size_t workspace_bytes, int path,
                                       hg_stream_t stream);

/* ------------------------------------------------------------------------
 * Serving engine (no counterpart in the reference, whose tables are built
 * and intersected once per process): resident tables under a device-memory
 * budget and a table limit, evicted least recently used first; requests
 * spread over a pool of CUDA streams; each request's latency from its
 * arrival stamp to the device completion of its last operation.  One host
 * thread drives a server.  Tables hold up to max_keys keys and buckets.
 * ---------------------------------------------------------------------- */
typedef struct hg_server hg_server;

/* A completed request, as hg_server_poll reports it. */
typedef struct hg_server_done {
  uint64_t ticket;
  int kind;                  /* 0 build, 1 intersect */
  int missed;                /* intersect: the table was not resident */
  unsigned long long count;  /* intersect: exact match count */
  double latency_s;          /* arrival to device completion */
} hg_server_done;

/* The clock arrival stamps use (CLOCK_MONOTONIC, seconds). */
double hg_server_now(void);
hg_status hg_server_create(size_t budget_bytes, int max_tables, int n_streams, uint64_t max_keys,
                           int key_bytes, hg_server** out);
/* Maps `bytes` (at most the budget) of device memory into the server's table
 * pool up front, so that builds do not wait on the host while the pool
 * grows.  The pool keeps up to the budget mapped for reuse. */
hg_status hg_server_reserve(hg_server* server, size_t bytes);
/* Builds (or replaces) table `table_id` from d_keys[0..n); the keys must be
 * written before the call (the server's streams do not wait on the caller's)
 * and stay valid until the request completes.  Evicts tables to make room. */
hg_status hg_server_build(hg_server* server, uint64_t table_id, const void* d_keys, uint64_t n,
                          uint64_t n_buckets, int with_index, double arrival_s, uint64_t* ticket);
/* Probes d_query[0..nq) (the same rules as the keys of a build) against
 * table `table_id`; pairs go to d_pairs (or, when NULL, nowhere for a
 * batched request and to a per-stream buffer the next request overwrites for
 * one launched on its own). */
hg_status hg_server_intersect(hg_server* server, uint64_t table_id, const void* d_query, uint64_t nq,
                              uint32_t* d_pairs, uint64_t pair_cap, double arrival_s, uint64_t* ticket);
/* One request of hg_server_submit. */
typedef struct hg_server_request {
  int kind;              /* 0 build, 1 intersect */
  int with_index;        /* build */
  uint64_t table_id;
  const void* d_data;    /* build: the keys; intersect: the queries */
  uint64_t n;            /* keys or queries */
  uint64_t n_buckets;    /* build */
  uint32_t* d_pairs;     /* intersect: as for hg_server_intersect */
  uint64_t pair_cap;     /* intersect */
  double arrival_s;
} hg_server_request;
/* Submits reqs[0..n) in order, exactly as that many hg_server_build /
 * hg_server_intersect calls would (one call for a whole arrival burst, so
 * the host's per-call cost does not bound a saturated server).  Stops at the
 * first request refused: *n_done gets the requests submitted, tickets[i]
 * their tickets, and the refusal's status is returned. */
hg_status hg_server_submit(hg_server* server, const hg_server_request* reqs, int n, uint64_t* tickets,
                           int* n_done);
/* Reports up to max_out completed requests (block: wait for the oldest). */
hg_status hg_server_poll(hg_server* server, int block, hg_server_done* out, int max_out, int* n_out);
hg_status hg_server_stats(const hg_server* server, uint64_t* resident_tables, size_t* resident_bytes,
                          uint64_t* evictions, uint64_t* inflight);
/* Continuous batching (no counterpart in the reference, which has no serving
 * path).  Requests of at most small_max keys (queries) are queued and
 * launched together as one batched launch sequence (see hg_batch): when
 * max_queued are queued, when the oldest has waited max_wait_s (checked by
 * hg_server_poll), before a request launched on its own, and when
 * hg_server_poll blocks.  Defaults: enabled, 2^16 keys, 256 requests, 100 us.
 * enabled = 0 launches every request on its own. */
hg_status hg_server_set_batching(hg_server* server, int enabled, uint64_t small_max, uint32_t max_queued,
                                 double max_wait_s);
/* Batched launches so far and the requests they carried. */
hg_status hg_server_batch_stats(const hg_server* server, uint64_t* batches, uint64_t* batched_requests);
/* Waits for all work, frees every table and the server. */
void hg_server_free(hg_server* server);

/* ------------------------------------------------------------------------
 * Instrumentation (no counterpart in the reference, which prints host wall
 * times under HOST_PROFILE, src/MultiHashGraph.cu:55-57,431-615).
 * ---------------------------------------------------------------------- */
/* Turns per-phase CUDA-event timing on/off and drops unread records.  Events
 * are recorded on the launching stream; no host synchronisation is added. */
hg_status hg_profile_enable(int on);
/* Waits for and returns up to `cap` recorded phases (name, milliseconds) in
 * launch order; *count gets the number recorded.  Clears the records. */
hg_status hg_profile_read(int cap, int* count, const char** names, float* ms);
/* Kernels this library has launched in this process. */
unsigned long long hg_launch_count(void);

/* ------------------------------------------------------------------------
 * Seeded workload generators (device), matching the oracle's definitions.
 * ---------------------------------------------------------------------- */
/* key[i] = splitmix-stream(seed, 0, i) (top 32 bits for 4-byte keys). */
hg_status hg_gen_uniform(void* d_out, uint64_t n, int key_bytes, uint64_t seed, hg_stream_t stream);
/* n keys: n_from_a of them distinct draws from d_a (n_a keys), the rest fresh,
 * shuffled by a seeded bijection. */
hg_status hg_gen_overlap(void* d_out, uint64_t n, int key_bytes, const void* d_a, uint64_t n_a,
                         uint64_t n_from_a, uint64_t seed, hg_stream_t stream);
/* Zipf draws through a u64 fixed-point CDF table (universe entries, device). */
hg_status hg_gen_zipf(void* d_out, uint64_t n, int key_bytes, const uint64_t* d_cdf,
                      uint64_t universe, uint64_t seed, hg_stream_t stream);
/* key[i] = splitmix-stream(seed, 0, i) mod bound: uniform keys in [0, bound),
 * the key range of the reference's SingleHashGraph generator
 * (src/SingleHashGraph.cu:66-77,116-119, thrust draws in [0, maxkey]). */
hg_status hg_gen_bounded(void* d_out, uint64_t n, int key_bytes, uint64_t seed, uint64_t bound,
                         hg_stream_t stream);
/* d_out[i] = (int64) d_keys[d_pairs[2*i + which]] for i < count: the key side
 * of intersect pairs, e.g. B's key per match as MultiHashGraph::intersect
 * outputs it (keypair{right}, include/MultiHashGraph.cuh:89-93). */
hg_status hg_gather_pair_keys(const void* d_keys, int key_bytes, const uint32_t* d_pairs,
                              uint64_t count, int which, int64_t* d_out, hg_stream_t stream);
/* Writes a built table in the reference's layout: n 16-byte records
 * {key (8 bytes, or 4 + 4 padding for 32-bit keys), int64 index} into d_kv16
 * (the index is the stored input position, or the CSR position without an
 * index) and n_buckets+1 int64 offsets into d_offsets64 -- keyval_ind and
 * index_t of include/MultiHashGraph.cuh:82-87,66-74, as MultiHashGraph keeps
 * them at h_dFinalKeys + h_edgesOff / h_offsetOff (src/MultiHashGraph.cu:549-566). */
hg_status hg_export_reference_layout(const uint32_t* d_offsets, const void* d_keys,
                                     const uint32_t* d_idx, uint64_t n, uint64_t n_buckets,
                                     int key_bytes, void* d_kv16, int64_t* d_offsets64,
                                     hg_stream_t stream);
/* Host: fills cdf[universe] for Zipf(s). */
hg_status hg_zipf_cdf(uint64_t* cdf, uint64_t universe, double s);

#ifdef __cplusplus
}
#endif
#endif /* HASHGRAPH_B200_H */
