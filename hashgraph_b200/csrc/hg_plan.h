// hg_plan.h -- host-side planning of build / intersect launches and the
// workspace layout they use.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "hashgraph_b200.h"

namespace hg {

constexpr size_t WS_ALIGN = 256;
inline size_t align_up(size_t x, size_t a = WS_ALIGN) { return (x + a - 1) / a * a; }

constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_ITEMS = 16;
constexpr uint64_t SCAN_TILE = uint64_t(SCAN_BLOCK) * SCAN_ITEMS;

enum BuildPath : int { BUILD_DIRECT = 0, BUILD_PARTITIONED = 1 };

struct BuildPlan {
  int path = BUILD_DIRECT;
  uint64_t n = 0, n_buckets = 0;
  int key_bytes = 8;
  bool with_index = false;
  // direct path: in-place scan over offsets[1..B]
  uint64_t scan_tiles = 0;
  // partitioned path
  uint32_t part_log2 = 0;     // buckets per partition = 2^part_log2
  uint64_t n_parts = 0;
  uint64_t part_cap = 0;      // record slots per partition
  uint64_t pscan_tiles = 0;   // tiles of the partition-count scan
  // workspace byte offsets
  size_t off_status = 0, off_ticket = 0, off_flags = 0;
  size_t off_pcount = 0, off_pkeys = 0, off_pidx = 0;
  size_t total = 0;
};

// Chooses the path and lays out the workspace.  `force_path` < 0 lets the
// planner decide.
hg_status plan_build(uint64_t n, int key_bytes, uint64_t n_buckets, bool with_index,
                     BuildPlan* plan, int force_path = -1);

struct ProbePlan {
  int path = 0;               // 0 direct
  uint64_t nq = 0, n_buckets = 0;
  int key_bytes = 8;
  bool emit = false;
  uint64_t tiles = 0;
  size_t off_status = 0, off_ticket = 0;
  size_t total = 0;
};

hg_status plan_probe(uint64_t n_buckets, uint64_t nq, int key_bytes, bool emit, ProbePlan* plan);

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
