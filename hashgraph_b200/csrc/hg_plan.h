// hg_plan.h -- host-side planning of build / intersect launches and the
// workspace layout they use.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "hashgraph_b200.h"
#include "hg_device.cuh"

namespace hg {

constexpr size_t WS_ALIGN = 256;
inline size_t align_up(size_t x, size_t a = WS_ALIGN) { return (x + a - 1) / a * a; }

constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_ITEMS = 16;
constexpr uint64_t SCAN_TILE = uint64_t(SCAN_BLOCK) * SCAN_ITEMS;

enum BuildPath : int { BUILD_DIRECT = 0, BUILD_PARTITIONED = 1 };

constexpr size_t SMEM_BUDGET = 220 * 1024;  // dynamic shared memory per CTA (B200 opt-in max 227 KB)
constexpr size_t FINE_SMEM_BUDGET = 100 * 1024;        // pass-3 build CTAs: two per SM (double-buffered)
constexpr size_t FINE_PROBE_SMEM_BUDGET = 220 * 1024;  // pass-3 probe CTAs: one per SM (double-buffered)
// coarse probe: bytes of the table per bucket range, read from L2 by every CTA at once
constexpr size_t COARSE_SLICE_BUDGET = size_t(24) << 20;
constexpr int PASS1_BLOCK = 512;                 // pass-1 CTA for 8-byte keys (and every batch)
constexpr int PASS1_KPT = 8;                     // pass-1 keys per thread per tile (registers)
constexpr int PASS1_TILE = PASS1_BLOCK * PASS1_KPT;
constexpr uint64_t PASS1_MAX_PARTS = 2048;       // coarse partitions pass 1 can reserve runs in
constexpr uint64_t PASS1_GOOD_PARTS = 512;       // above this many, runs get short and pass 1 slow
// Pass 1 of a table or a query set: 4-byte keys take one 1024-thread CTA per
// SM over 8192-key tiles, so that a tile's run in each of 512 partitions is
// 16 keys (64 bytes per array) instead of 8 (2^30 u32 keys + index: 8.47 ->
// 5.56 ms for the table, 8.45 -> 5.56 ms for the queries); 8-byte keys keep
// two 512-thread CTAs over 4096-key tiles (the larger tile measured 1.26 ->
// 1.31 ms at 2^28 u64, and 1.37 -> 1.51 ms for the queries).
constexpr int pass1_block(int key_bytes) { return key_bytes == 4 ? 1024 : PASS1_BLOCK; }
constexpr int pass1_tile(int key_bytes) { return pass1_block(key_bytes) * PASS1_KPT; }
constexpr int SPLIT_BLOCK = 512;
constexpr int SPLIT_TILE = 8 * SPLIT_BLOCK;     // k_split sorts a tile in registers: 8 records per thread
constexpr int SPLIT_BLOCK_WIDE = 1024;
constexpr int FINE_BLOCK = 512;
constexpr int FINE_PROBE_BLOCK = 1024;          // one 1024-thread probe CTA per SM
constexpr uint32_t SPLIT_LOG2_MAX = 8;          // pass 2 splits a coarse partition 256 ways (up to 1024)

// Geometry of the partitioned (three-pass) paths, shared by build and probe:
// pass 1 splits the keys into n_parts coarse partitions of 2^coarse_log2
// buckets (cluster multisplit), pass 2 splits each coarse partition into
// 2^split_log2 fine partitions of 2^fine_log2 buckets, pass 3 works on one
// fine partition per CTA in shared memory.
struct PartGeometry {
  uint32_t fine_log2 = 0, split_log2 = 0, coarse_log2 = 0;
  uint64_t n_parts = 0, part_cap = 0;   // coarse partitions and their record slots
  uint64_t n_fine = 0, fine_cap = 0;    // fine partitions and their record slots
  uint32_t smem_cap = 0;                // records pass 3 stages in shared memory
  uint32_t tile1 = 0;                   // pass-1 keys per CTA per tile
  size_t smem1 = 0, smem2 = 0, smem3 = 0;
  int split_block = SPLIT_BLOCK;        // k_split CTA (SPLIT_BLOCK or SPLIT_BLOCK_WIDE threads, 8 records each)
  uint64_t pscan_tiles = 0, fscan_tiles = 0;
};

struct BuildPlan {
  int path = BUILD_DIRECT;
  uint64_t n = 0, n_buckets = 0;
  // a shard of a larger table: buckets [range_lo, range_lo + n_buckets) of
  // range_total (0: the table is whole)
  uint64_t range_total = 0, range_lo = 0;
  BucketMap bucket_map() const {
    return range_total ? BucketMap::make_range(range_total, range_lo, n_buckets) : BucketMap::make(n_buckets);
  }
  int key_bytes = 8;
  bool with_index = false;
  // with an index: the indices to store for the input keys (input key i gets
  // key_idx[i]); NULL stores the input position i
  const uint32_t* key_idx = nullptr;
  uint64_t scan_tiles = 0;  // direct path: in-place scan over offsets[1..B]
  PartGeometry g;           // partitioned path
  // workspace byte offsets
  size_t off_status = 0, off_ticket = 0, off_flags = 0;
  size_t off_pcount = 0, off_pstatus = 0, off_fcount = 0, off_fstatus = 0;
  size_t off_gcount = 0, off_gstatus = 0;  // partitioned path's fallback: exact partition counts
  size_t off_pkeys = 0, off_pidx = 0, off_fkeys = 0, off_fidx = 0;
  size_t total = 0;
};

// Chooses the path and lays out the workspace.  `force_path` < 0 lets the
// planner decide.
hg_status plan_build(uint64_t n, int key_bytes, uint64_t n_buckets, bool with_index,
                     BuildPlan* plan, int force_path = -1);

// PROBE_COARSE: pass 1 into bucket ranges whose slice of the table stays in
// L2, then every range probed from L2 (no split pass, no staging).
enum ProbePath : int { PROBE_DIRECT = 0, PROBE_PARTITIONED = 1, PROBE_COARSE = 2 };

struct ProbePlan {
  int path = PROBE_DIRECT;
  uint64_t n_a = 0, nq = 0, n_buckets = 0;
  uint64_t range_total = 0, range_lo = 0;  // as in BuildPlan
  BucketMap bucket_map() const {
    return range_total ? BucketMap::make_range(range_total, range_lo, n_buckets) : BucketMap::make(n_buckets);
  }
  int key_bytes = 8;
  bool a_idx = false;
  bool emit = false;
  uint64_t tiles = 0;  // direct path: tiles of queries
  PartGeometry g;      // partitioned path (pass 3 stages A's slice)
  size_t off_status = 0, off_ticket = 0, off_flags = 0;
  size_t off_heavy = 0;  // count only: heavy-key set of the direct probe
  size_t off_pcount = 0, off_pstatus = 0, off_fcount = 0, off_fstatus = 0;
  size_t off_pkeys = 0, off_pidx = 0, off_fkeys = 0, off_fidx = 0;
  size_t total = 0;
};

hg_status plan_probe(uint64_t n_a, bool a_idx, uint64_t n_buckets, uint64_t nq, int key_bytes, bool emit,
                     ProbePlan* plan, int force_path = -1);

// Partition geometry for `n_stream` streamed records of stream_rec bytes
// (pass 1/2) over n_buckets buckets, with pass 3 staging per fine partition
// `per_bucket` bytes per bucket plus up to smem_cap records of smem_rec bytes
// sized for n_staged records in the table.  Returns false if infeasible.
// With staged_may_spill, a table too dense to stage still gets the narrowest
// fine width and as many staged records as fit (the rest is read in place).
// Pass 3 also keeps stream_smem bytes per streamed record of a fine partition.
bool plan_geometry(uint64_t n_stream, size_t stream_rec, uint64_t n_staged, size_t smem_rec, size_t per_bucket,
                   size_t stream_smem, uint64_t n_buckets, bool staged_may_spill, PartGeometry* g,
                   size_t fine_budget = FINE_SMEM_BUDGET);
uint64_t slack_capacity(double mean, uint64_t margin, double sigmas = 8.0);
size_t pass1_smem(uint64_t n_parts, int key_bytes, int tile);
// Sets g.split_block and g.smem2 for a split of g.split_log2 ways.
void plan_split(PartGeometry& g, int key_bytes, bool with_index);
size_t split_smem(uint32_t split_log2, int key_bytes, bool with_index, uint64_t n_parts, int tile);

// Kernel launchers (hg_build.cu / hg_probe.cu).  Workspace pointers are
// already carved by the caller; all launches go to `stream`.
hg_status launch_build(const BuildPlan& plan, const void* d_keys, uint32_t* d_offsets,
                       void* d_keys_out, uint32_t* d_idx_out, void* d_ws, cudaStream_t stream);

hg_status launch_probe(const ProbePlan& plan, const uint32_t* a_off, const void* a_keys,
                       const uint32_t* a_idx, const void* q_keys, const uint32_t* q_idx,
                       uint32_t* pairs, uint64_t pair_cap, unsigned long long* d_count, void* d_ws,
                       cudaStream_t stream);

int device_sm_count();

}  // namespace hg
