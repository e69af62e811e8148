// hg_build.cu -- CSR build kernels for sm_100a.
//
// Two paths produce the same table (offsets / keys / optional idx):
//
// Direct (tables whose working set sits in L2):
//   1. k_count:   hash each key, warp-aggregated atomicAdd of the bucket count
//                 into offsets[b+1] (replaces hashValuesD + countHashD,
//                 include/SingleHashGraphOperators.cuh:71-87).
//   2. k_scan_u32: decoupled look-back exclusive scan of offsets[1..B] in place
//                 (replaces cub::DeviceScan::ExclusiveSum + the host write of
//                 offsets[B], src/SingleHashGraph.cu:199-207).
//   3. k_scatter: rehash, warp-aggregated cursor bump on offsets[b+1], write key
//                 (+ input position) -- replaces copyToGraphD (:89-100).  Each
//                 cursor ends at the start of bucket b+1, so offsets[] is the
//                 final CSR offset array without a second counter array.
//
// Partitioned (large tables; replaces the LRB locality pass
// lrbCountHashD/lrbRehashD/lrbCountHashGlobalD/lrbCopyToGraphD,
// include/SingleHashGraphOperators.cuh:102-154, and the 1-GPU multi pipeline):
//   0. k_skew_check: 8192 sampled keys; a partition certain to overflow
//                 sets the overflow flag before any pass runs.
//   1. k_multisplit: tiles of 4096 keys (8-byte keys) or 8192 keys (4-byte
//                 keys) per CTA are ranked per coarse partition
//                 (2^coarse_log2 buckets) in shared memory, one global atomic
//                 per (tile, partition) reserves the run, and the tile leaves
//                 partition-sorted as coalesced runs.
//   2. k_scan_u32 over the coarse partition sizes.
//   3. k_split:   each coarse partition is split 256 ways (up to 1024) into
//                 fine partitions of W = 2^fine_log2 buckets the same way.
//   4. k_scan_u32 over the fine partition sizes.
//   5. k_fine_build: one CTA per fine partition: bucket histogram in shared
//                 memory, segmented block scan, coalesced offsets write, then
//                 the scatter of the partition's keys into its output slice.
//   If any partition overflowed its slot range (heavy duplicates), pass 5
//   stands down and a gated fallback rebuilds the table: the keys grouped by
//   coarse partition into exactly sized runs (k_part_hist, a scan,
//   k_multisplit in exact mode), then the direct kernels over the grouped
//   keys.  The decision is taken on the device, so the launch sequence is
//   fixed.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

#include "hg_device.cuh"
#include "hg_bulk.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"
#include "hg_scan.cuh"

namespace hg {

constexpr uint32_t FLAG_OVERFLOW = 1u;

// Gate: kernels handed a non-null gate run only when the overflow flag is set.
__device__ __forceinline__ bool gated_off(const uint32_t* gate) {
  return gate != nullptr && (*reinterpret_cast<const volatile uint32_t*>(gate) & FLAG_OVERFLOW) == 0;
}

// Entry test of every kernel that reads other kernels' results or writes at
// computed positions: true when a device fault is pending or the gate is
// closed.  One thread decides and the CTA follows, so every thread of the CTA
// returns together (the fault word may be set by another stream's kernel at
// any moment, and a CTA split between returning and running would leave its
// barriers and warp collectives short).  Contains __syncthreads().
__device__ __forceinline__ bool entry_skip(const uint32_t* gate) {
  __shared__ int s_skip;
  if (threadIdx.x == 0) s_skip = (device_faulted() || gated_off(gate)) ? 1 : 0;
  __syncthreads();
  return s_skip != 0;
}

// The same for the partitioned paths' kernels, which run only while the
// overflow flag is clear (the gated direct kernels take over once it is set).
__device__ __forceinline__ bool entry_skip_on_overflow(const uint32_t* flags) {
  __shared__ int s_skip;
  if (threadIdx.x == 0)
    s_skip = (device_faulted() || (*reinterpret_cast<const volatile uint32_t*>(flags) & FLAG_OVERFLOW)) ? 1 : 0;
  __syncthreads();
  return s_skip != 0;
}

// Loads the V keys lane `lane` owns in chunk [base, base + 32V); marks which
// exist.  Full chunks use one or two 16-byte vector loads per lane.
template <typename KeyT, int V>
__device__ __forceinline__ void load_chunk(const KeyT* __restrict__ keys, uint64_t n, uint64_t base,
                                           KeyT (&k)[V], bool (&ok)[V]) {
  const uint64_t first = base + static_cast<uint64_t>(lane_id()) * V;
  if (base + 32ull * V <= n) {
    if constexpr (V * sizeof(KeyT) == 16) {
      const uint4 u = __ldcs(reinterpret_cast<const uint4*>(keys + first));
      const KeyT* e = reinterpret_cast<const KeyT*>(&u);
#pragma unroll
      for (int j = 0; j < V; j++) { k[j] = e[j]; ok[j] = true; }
    } else {
#pragma unroll
      for (int j = 0; j < V; j++) { k[j] = __ldcs(keys + first + j); ok[j] = true; }
    }
  } else {
#pragma unroll
    for (int j = 0; j < V; j++) {
      ok[j] = first + j < n;
      k[j] = ok[j] ? __ldcs(keys + first + j) : KeyT(0);
    }
  }
}

// ---------------------------------------------------------------------------
// Direct path
// ---------------------------------------------------------------------------
template <typename KeyT, int V>
__global__ void __launch_bounds__(256) k_count(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm,
                                               uint32_t* __restrict__ cnt, const uint32_t* gate) {
  if (entry_skip(gate)) return;
  const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  const uint64_t nchunks = (n + 32ull * V - 1) / (32ull * V);
  for (uint64_t c = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; c < nchunks;
       c += warps) {
    KeyT k[V];
    bool ok[V];
    load_chunk<KeyT, V>(keys, n, c * 32ull * V, k, ok);
#pragma unroll
    for (int j = 0; j < V; j++) warp_aggregated_count(cnt, bm.of_key(k[j]), ok[j]);
  }
}

template <typename KeyT, int V, bool WITH_IDX>
__global__ void __launch_bounds__(256) k_scatter(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm,
                                                 uint32_t* __restrict__ cursor, KeyT* __restrict__ keys_out,
                                                 uint32_t* __restrict__ idx_out, const uint32_t* __restrict__ key_idx,
                                                 const uint32_t* gate) {
  if (entry_skip(gate)) return;
  const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  const uint64_t nchunks = (n + 32ull * V - 1) / (32ull * V);
  for (uint64_t c = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; c < nchunks;
       c += warps) {
    KeyT k[V];
    bool ok[V];
    const uint64_t base = c * 32ull * V;
    load_chunk<KeyT, V>(keys, n, base, k, ok);
#pragma unroll
    for (int j = 0; j < V; j++) {
      const uint32_t pos = warp_aggregated_inc(cursor, bm.of_key(k[j]), ok[j]);
      if (ok[j] && pos >= n) record_fault(HG_ERR_DEVICE_STATE);  // offsets past n: write nothing
      else if (ok[j]) {
        keys_out[pos] = k[j];
        if constexpr (WITH_IDX) {
          const uint64_t i = base + lane_id() * V + j;
          idx_out[pos] = key_idx ? key_idx[i] : static_cast<uint32_t>(i);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Direct path under skew.  The gated direct kernels run when the partitioned
// path overflowed, that is when some buckets are far above their expected
// size (heavy duplicates, Zipf keys).  Then a few buckets take most of the
// keys, and even warp-aggregated global atomics serialise on them: at 2^28
// Zipf(1.1) keys the hottest counter gets one atomic from nearly every warp.
// These forms aggregate per CTA first, in a shared-memory table of the
// chunk's buckets (open addressing, bucket id -> count): each chunk of
// SKEW_CHUNK keys costs one global atomic per distinct bucket in it, so a hot
// bucket gets one per chunk.  A key whose bucket finds no slot within
// SKEW_PROBES steps takes a global atomic of its own.
// ---------------------------------------------------------------------------
constexpr int SKEW_BLOCK = 256;
constexpr int SKEW_KPT = 8;
constexpr uint32_t SKEW_CHUNK = uint32_t(SKEW_BLOCK) * SKEW_KPT;
constexpr uint32_t SKEW_SLOTS = 4096;
constexpr uint32_t SKEW_PROBES = 8;
constexpr uint32_t SKEW_EMPTY = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t skew_slot(uint32_t b) { return (b * 0x9E3779B1u) >> 20; }

// Slot of bucket b in the chunk's table (claimed if new), or SKEW_SLOTS.
__device__ __forceinline__ uint32_t skew_place(uint32_t* s_b, uint32_t b) {
  if (b == SKEW_EMPTY) return SKEW_SLOTS;
  uint32_t h = skew_slot(b);
  for (uint32_t p = 0; p < SKEW_PROBES; p++) {
    const uint32_t prev = atomicCAS(s_b + h, SKEW_EMPTY, b);
    if (prev == SKEW_EMPTY || prev == b) return h;
    h = (h + 1) & (SKEW_SLOTS - 1);
  }
  return SKEW_SLOTS;
}

template <typename KeyT>
__global__ void __launch_bounds__(SKEW_BLOCK) k_count_skew(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm,
                                                           uint32_t* __restrict__ cnt, const uint32_t* gate) {
  if (entry_skip(gate)) return;
  __shared__ uint32_t s_b[SKEW_SLOTS], s_c[SKEW_SLOTS];
  for (uint32_t i = threadIdx.x; i < SKEW_SLOTS; i += SKEW_BLOCK) {
    s_b[i] = SKEW_EMPTY;
    s_c[i] = 0;
  }
  __syncthreads();
  const unsigned lane = lane_id();
  for (uint64_t base = uint64_t(blockIdx.x) * SKEW_CHUNK; base < n; base += uint64_t(gridDim.x) * SKEW_CHUNK) {
#pragma unroll
    for (int u = 0; u < SKEW_KPT; u++) {
      const uint64_t i = base + uint64_t(u) * SKEW_BLOCK + threadIdx.x;
      const bool valid = i < n;
      const uint32_t b = valid ? bm.of_key(__ldcs(keys + i)) : 0u;
      // a warp whose 32 keys share one bucket (a hot key's run in grouped
      // input) counts them with one atomic; other warps key by key
      const uint32_t b0 = __shfl_sync(FULL_MASK, b, 0);
      if (__all_sync(FULL_MASK, valid && b == b0)) {
        if (lane == 0) {
          const uint32_t h = skew_place(s_b, b0);
          if (h < SKEW_SLOTS) atomicAdd(s_c + h, 32u);
          else atomicAdd(cnt + b0, 32u);
        }
      } else if (valid) {
        const uint32_t h = skew_place(s_b, b);
        if (h < SKEW_SLOTS) atomicAdd(s_c + h, 1u);
        else atomicAdd(cnt + b, 1u);
      }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < SKEW_SLOTS; i += SKEW_BLOCK) {
      const uint32_t c = s_c[i];
      if (c) {
        atomicAdd(cnt + s_b[i], c);
        s_c[i] = 0;
      }
      s_b[i] = SKEW_EMPTY;
    }
    __syncthreads();
  }
}

// Scatter: a chunk's keys take a rank in their bucket's slot, one global
// atomic per slot reserves the bucket's run for the chunk, then every key is
// written at run start + rank.
template <typename KeyT, bool WITH_IDX>
__global__ void __launch_bounds__(SKEW_BLOCK) k_scatter_skew(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm,
                                                             uint32_t* __restrict__ cursor, KeyT* __restrict__ keys_out,
                                                             uint32_t* __restrict__ idx_out,
                                                             const uint32_t* __restrict__ key_idx,
                                                             const uint32_t* gate) {
  if (entry_skip(gate)) return;
  __shared__ uint32_t s_b[SKEW_SLOTS], s_c[SKEW_SLOTS];  // s_c: the chunk's count, then its run start
  for (uint32_t i = threadIdx.x; i < SKEW_SLOTS; i += SKEW_BLOCK) {
    s_b[i] = SKEW_EMPTY;
    s_c[i] = 0;
  }
  __syncthreads();
  const unsigned lane = lane_id();
  for (uint64_t base = uint64_t(blockIdx.x) * SKEW_CHUNK; base < n; base += uint64_t(gridDim.x) * SKEW_CHUNK) {
    KeyT k[SKEW_KPT];
    uint32_t where[SKEW_KPT];  // slot << 16 | rank, or the position taken by a global atomic
    uint32_t direct = 0;       // bit u: where[u] is a position
#pragma unroll
    for (int u = 0; u < SKEW_KPT; u++) {
      const uint64_t i = base + uint64_t(u) * SKEW_BLOCK + threadIdx.x;
      k[u] = i < n ? __ldcs(keys + i) : KeyT(0);
    }
#pragma unroll
    for (int u = 0; u < SKEW_KPT; u++) {
      // the warp's lanes with the same bucket take consecutive ranks: their
      // lowest lane claims the slot and reserves the group's ranks at once
      const bool valid = base + uint64_t(u) * SKEW_BLOCK + threadIdx.x < n;
      const uint32_t b = valid ? bm.of_key(k[u]) : 0u;
      const unsigned peers = __match_any_sync(FULL_MASK, valid ? uint64_t(b) : (1ull << 40));
      const unsigned leader = __ffs(peers) - 1;
      uint32_t h = SKEW_SLOTS, first = 0;
      if (valid && lane == leader) {
        h = skew_place(s_b, b);
        first = h < SKEW_SLOTS ? atomicAdd(s_c + h, uint32_t(__popc(peers)))
                               : atomicAdd(cursor + b, uint32_t(__popc(peers)));
      }
      h = __shfl_sync(FULL_MASK, h, leader);
      first = __shfl_sync(FULL_MASK, first, leader) + __popc(peers & lanemask_lt());
      where[u] = 0;
      if (valid) {
        if (h < SKEW_SLOTS) {
          where[u] = (h << 16) | first;
        } else {
          where[u] = first;
          direct |= 1u << u;
        }
      }
    }
    __syncthreads();
    // the chunk's run reservations: each thread's slots in groups of eight,
    // all eight atomics in flight before their results are stored
    constexpr uint32_t SPT = SKEW_SLOTS / SKEW_BLOCK;
#pragma unroll
    for (uint32_t g0 = 0; g0 < SPT; g0 += 8) {
      uint32_t c8[8], used = 0;
#pragma unroll
      for (uint32_t u = 0; u < 8; u++) {
        c8[u] = s_c[(g0 + u) * SKEW_BLOCK + threadIdx.x];
        used |= (c8[u] != 0u) << u;
      }
#pragma unroll
      for (uint32_t u = 0; u < 8; u++) {
        const uint32_t i = (g0 + u) * SKEW_BLOCK + threadIdx.x;
        if ((used >> u) & 1u) c8[u] = atomicAdd(cursor + s_b[i], c8[u]);
      }
#pragma unroll
      for (uint32_t u = 0; u < 8; u++)
        if ((used >> u) & 1u) s_c[(g0 + u) * SKEW_BLOCK + threadIdx.x] = c8[u];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < SKEW_KPT; u++) {
      const uint64_t i = base + uint64_t(u) * SKEW_BLOCK + threadIdx.x;
      if (i < n) {
        const uint32_t pos = (direct >> u) & 1u ? where[u] : s_c[where[u] >> 16] + (where[u] & 0xffffu);
        if (pos < n) {
          keys_out[pos] = k[u];
          if constexpr (WITH_IDX) idx_out[pos] = key_idx ? key_idx[i] : static_cast<uint32_t>(i);
        } else {
          record_fault(HG_ERR_DEVICE_STATE);  // offsets past n: write nothing
        }
      }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < SKEW_SLOTS; i += SKEW_BLOCK) {
      s_c[i] = 0;
      s_b[i] = SKEW_EMPTY;
    }
    __syncthreads();
  }
}

// In-place exclusive scan of data[0..count) (uint32 values, total < 2^32).
// first_slot (optional) receives 0; total_out (optional) receives the sum.
// Persistent: each CTA takes tiles in ticket order until none is left.  Four
// CTAs per SM (64 registers) and the L2 prefetch of the tile one ticket round
// ahead: 2^28 counts 1.27 -> 1.04 ms.
template <int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK, 4) k_scan_u32(uint32_t* __restrict__ data, uint64_t count,
                                                    uint64_t* __restrict__ status, unsigned* ticket,
                                                    uint32_t* first_slot, uint32_t* total_out,
                                                    const uint32_t* gate) {
  if (entry_skip(gate)) return;
  constexpr int TILE = BLOCK * ITEMS;
  __shared__ uint32_t s[TILE + TILE / 32];
  __shared__ uint32_t red[BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
  const uint64_t ntiles = (count + TILE - 1) / TILE;
  constexpr int LINES = TILE * 4 / 128;  // 128-byte lines of a tile
  static_assert(LINES <= BLOCK, "one prefetch per thread");
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= ntiles) break;
    const uint64_t base = tile * TILE;
    // the tile a CTA takes about one round of tickets from now (tile +
    // gridDim.x) is brought into L2 here, so that whoever takes it loads from
    // L2; no ticket is held ahead, so every look-back still waits only on
    // tiles that have started
    if (threadIdx.x < LINES) {
      const uint64_t e = (tile + gridDim.x) * TILE + uint64_t(threadIdx.x) * 32;
      if (e < count) asm volatile("prefetch.global.L2 [%0];" ::"l"(data + e));
    }
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      const int si = k * BLOCK + threadIdx.x;
      const uint64_t i = base + si;
      s[si + si / 32] = i < count ? data[i] : 0u;
    }
    __syncthreads();
    uint32_t v[ITEMS];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      const int si = threadIdx.x * ITEMS + k;
      v[k] = s[si + si / 32];
      sum += v[k];
    }
    uint32_t tile_total;
    const uint32_t excl = block_exclusive_scan<BLOCK>(sum, red, &tile_total);
    if (threadIdx.x < 32) {
      const uint64_t p = lookback_exclusive(status, tile, tile_total);
      if (threadIdx.x == 0) s_prefix = p;
    }
    __syncthreads();
    uint32_t run = static_cast<uint32_t>(s_prefix) + excl;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      const int si = threadIdx.x * ITEMS + k;
      s[si + si / 32] = run;
      run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      const int si = k * BLOCK + threadIdx.x;
      const uint64_t i = base + si;
      if (i < count) data[i] = s[si + si / 32];
    }
    if (threadIdx.x == 0) {
      if (tile == 0 && first_slot) *first_slot = 0u;
      if (tile == ntiles - 1 && total_out) *total_out = static_cast<uint32_t>(s_prefix) + tile_total;
    }
    __syncthreads();
  }
}

__global__ void k_fill_u32(uint32_t* p, uint64_t count, uint32_t value, const uint32_t* gate) {
  if (entry_skip(gate)) return;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    p[i] = value;
}

// ---------------------------------------------------------------------------
// Partitioned path (cluster kernels)
// ---------------------------------------------------------------------------

// Pass 1: multisplit into coarse partitions.  Each CTA takes tiles of TILE
// consecutive keys (KPT per thread, in registers), ranks them per coarse
// partition with shared-memory atomics, reserves its run in every partition
// with ONE global atomic per (tile, partition), and writes its keys
// partition-sorted (in-place counting sort in shared memory) so the runs
// leave as coalesced stores.  The reservations are issued before the local
// scan and sort and their results are consumed only after them, which hides
// the atomics' round trip.  With BULK, the CTA's next tile is prefetched into
// shared memory by a bulk copy (TMA) while the current one is processed.
// Dynamic smem: eoff[P] (i64) | hist[P] | lp[P] | raw[2][TILE] | si[TILE] | sp[TILE] (u16)

constexpr int64_t EOFF_NONE = INT64_MIN;      // a dropped (overflowing) run

// One pass-1 tile: where its keys come from and where its partitions go.
template <typename KeyT>
struct SplitTile {
  const KeyT* keys;         // source array; the tile is keys[base .. base + cnt)
  const uint32_t* key_idx;  // optional positions of the source keys (else base + r)
  uint64_t base;
  uint32_t cnt;
  BucketMap bm;
  uint32_t shift;           // partition = bucket >> shift
  uint32_t n_parts;
  uint64_t cap;             // record slots per partition
  uint32_t* pcount;         // per-partition counters
  KeyT* pkeys;              // partition p's slots start at p * cap
  uint32_t* pidx;
};

// Pass-1 tiles of one table: tile t holds keys [t*TILE, (t+1)*TILE).
template <typename KeyT, uint32_t TILE>
struct TableTiles {
  const KeyT* keys;
  const uint32_t* key_idx;
  uint64_t n;
  BucketMap bm;
  uint32_t shift, n_parts;
  uint64_t cap;
  uint32_t* pcount;
  KeyT* pkeys;
  uint32_t* pidx;
  __device__ __forceinline__ uint64_t ntiles() const { return (n + TILE - 1) / TILE; }
  __device__ __forceinline__ SplitTile<KeyT> at(uint64_t t) const {
    const uint64_t b = t * TILE;
    const uint32_t c = b < n ? static_cast<uint32_t>(umin64(TILE, n - b)) : 0u;
    return SplitTile<KeyT>{keys, key_idx, b, c, bm, shift, n_parts, cap, pcount, pkeys, pidx};
  }
};

// The partitioned build's fallback (gated: runs only after an overflow)
// first counts the keys of every coarse partition: a shared-memory histogram
// per CTA, one global add per partition and CTA.
constexpr int PART_HIST_BLOCK = 512;
template <typename KeyT>
__global__ void __launch_bounds__(PART_HIST_BLOCK)
    k_part_hist(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm, uint32_t shift, uint32_t n_parts,
                uint32_t* __restrict__ hist, const uint32_t* gate) {
  if (entry_skip(gate)) return;
  __shared__ uint32_t h[PASS1_MAX_PARTS];
  for (uint32_t j = threadIdx.x; j < n_parts; j += PART_HIST_BLOCK) h[j] = 0u;
  __syncthreads();
  constexpr int PER = 8;  // keys per thread and step, all loaded before any is counted
  const uint64_t stride = uint64_t(gridDim.x) * PART_HIST_BLOCK;
  for (uint64_t i0 = uint64_t(blockIdx.x) * PART_HIST_BLOCK + threadIdx.x; i0 < n; i0 += PER * stride) {
    KeyT k[PER];
#pragma unroll
    for (int u = 0; u < PER; u++) k[u] = i0 + u * stride < n ? __ldcs(keys + i0 + u * stride) : KeyT(0);
#pragma unroll
    for (int u = 0; u < PER; u++) {
      if (i0 + u * stride < n) {
        const uint32_t p = bm.of_key(k[u]) >> shift;
        if (p < n_parts) atomicAdd(&h[p], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < n_parts; j += PART_HIST_BLOCK)
    if (h[j]) atomicAdd(hist + j, h[j]);
}

// Before pass 1: SKEW_SAMPLES evenly spaced keys are histogrammed by coarse
// partition.  A partition whose sampled count passes c + 8 sqrt(c) + 8, c =
// the samples its slots would hold (cap * S / n), overflows for certain, so
// the overflow flag is set at once: pass 1 and the partitioned kernels then
// return at entry and the gated direct kernels do the work without a wasted
// pass (2^28 Zipf keys: 1.2 ms saved on each side of a build + probe).  A
// partition that fits its slots draws at most c samples on average (a
// binomial count; c >= 4 with at most 2048 partitions) and passes the bound
// with a probability below 10^-10 (Chernoff); a skew the sample misses
// still overflows in pass 1, which the fallback handles as before.
constexpr uint32_t SKEW_SAMPLES = 8192;
constexpr int SKEW_CHECK_BLOCK = 1024;

template <typename KeyT>
__global__ void __launch_bounds__(SKEW_CHECK_BLOCK)
    k_skew_check(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm, uint32_t shift, uint32_t n_parts,
                 uint64_t cap, uint32_t* flags) {
  if (entry_skip(nullptr)) return;
  __shared__ uint32_t h[PASS1_MAX_PARTS];
  for (uint32_t j = threadIdx.x; j < n_parts; j += SKEW_CHECK_BLOCK) h[j] = 0u;
  __syncthreads();
  const uint64_t S = n < SKEW_SAMPLES ? n : SKEW_SAMPLES;
  constexpr int PER = SKEW_SAMPLES / SKEW_CHECK_BLOCK;
  KeyT k[PER];
#pragma unroll
  for (int u = 0; u < PER; u++) {  // every sample's load in flight before any is used
    const uint64_t x = uint64_t(u) * SKEW_CHECK_BLOCK + threadIdx.x;
    k[u] = x < S ? keys[x * n / S] : KeyT(0);
  }
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const uint64_t x = uint64_t(u) * SKEW_CHECK_BLOCK + threadIdx.x;
    const uint32_t p = bm.of_key(k[u]) >> shift;
    if (x < S && p < n_parts) atomicAdd(&h[p], 1u);
  }
  __syncthreads();
  const double c = double(cap) * double(S) / double(n);
  const double bound = c + 8.0 * sqrt(c) + 8.0;
  for (uint32_t j = threadIdx.x; j < n_parts; j += SKEW_CHECK_BLOCK)
    if (double(h[j]) > bound) atomicOr(flags, FLAG_OVERFLOW);
}

// EXACT: the partitions' counts are known and pcount holds their starts in
// one flat record array (the fallback after an overflow groups the keys that
// way, every partition exactly sized): the kernel then runs only while the
// overflow flag is set, and no run can overflow.
template <typename KeyT, bool WITH_IDX, int BLOCK, int KPT, bool BULK, typename Src, bool EXACT = false>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) k_multisplit(Src src, uint32_t max_parts, uint32_t* flags) {
  if (EXACT ? entry_skip(flags) : entry_skip_on_overflow(flags)) return;
  constexpr uint32_t TILE = BLOCK * KPT;
  constexpr uint32_t APT = PASS1_MAX_PARTS / BLOCK;  // partition reservations per thread and tile
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int64_t* eoff = reinterpret_cast<int64_t*>(smem_raw);  // element offset of sorted position 0, per partition
  uint32_t* hist = reinterpret_cast<uint32_t*>(eoff + max_parts);
  uint32_t* lp = hist + max_parts;
  KeyT* raw = reinterpret_cast<KeyT*>(smem_raw + align_up_dev(size_t(max_parts) * 16, 16));
  uint32_t* si = reinterpret_cast<uint32_t*>(raw + 2 * TILE);
  uint16_t* sp = reinterpret_cast<uint16_t*>(si + TILE);
  __shared__ uint32_t wsum[BLOCK / 32 + 1];
  __shared__ uint64_t bar[2];
  const uint64_t ntiles = src.ntiles();
  // bulk part of a tile: whole 16-byte units; the ragged tail is read with plain loads
  auto bulk_bytes = [&](uint32_t cnt) -> uint32_t { return (cnt * uint32_t(sizeof(KeyT))) & ~15u; };
  for (uint32_t j = threadIdx.x; j < max_parts; j += BLOCK) hist[j] = 0u;
  if constexpr (BULK) {
    if (threadIdx.x == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      fence_mbar_init();
      if (blockIdx.x < ntiles) {
        const SplitTile<KeyT> v = src.at(blockIdx.x);
        bulk_load(raw, v.keys + v.base, bulk_bytes(v.cnt), &bar[0]);
      }
    }
  }
  __syncthreads();
  bool overflow = false;
  uint32_t it = 0;
  for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
    const SplitTile<KeyT> v = src.at(t);
    const KeyT* keys = v.keys;
    const uint32_t* key_idx = v.key_idx;
    const uint64_t base = v.base;
    const uint32_t cnt = v.cnt;
    const BucketMap bm = v.bm;
    const uint32_t coarse_log2 = v.shift;
    const uint32_t n_parts = v.n_parts;
    const uint64_t cap = v.cap;
    uint32_t* pcount = v.pcount;
    KeyT* pkeys = v.pkeys;
    uint32_t* pidx = v.pidx;
    KeyT* cur = raw + (it & 1) * TILE;
    if constexpr (BULK) {
      // prefetch the next tile into the other buffer (its readers finished at
      // the __syncthreads that closed the previous iteration)
      if (threadIdx.x == 0 && t + gridDim.x < ntiles) {
        fence_proxy_async_smem();
        const SplitTile<KeyT> nv = src.at(t + gridDim.x);
        bulk_load(raw + ((it + 1) & 1) * TILE, nv.keys + nv.base, bulk_bytes(nv.cnt), &bar[(it + 1) & 1]);
      }
    }
    KeyT k[KPT];
    uint32_t pr[KPT];
    if constexpr (BULK) {
      // one thread waits for the copy; the barrier publishes it to the rest
      if (threadIdx.x == 0) mbar_wait(&bar[it & 1], (it >> 1) & 1);
      __syncthreads();
      const uint32_t nb = bulk_bytes(cnt) / uint32_t(sizeof(KeyT));
#pragma unroll
      for (int u = 0; u < KPT; u++) {
        const uint32_t r = u * BLOCK + threadIdx.x;
        k[u] = r < nb ? cur[r] : (r < cnt ? keys[base + r] : KeyT(0));
      }
    } else {
#pragma unroll
      for (int u = 0; u < KPT; u++) {
        const uint32_t r = u * BLOCK + threadIdx.x;
        k[u] = r < cnt ? __ldcs(keys + base + r) : KeyT(0);
      }
    }
#pragma unroll
    for (int u = 0; u < KPT; u++) {
      const uint32_t r = u * BLOCK + threadIdx.x;
      if (r < cnt) {
        const uint32_t p = bm.of_key(k[u]) >> coarse_log2;
        pr[u] = (p << 16) | atomicAdd(&hist[p], 1u);
      }
    }
    __syncthreads();
    // reservations: issued now, consumed after the local scan and sort
    // (n_parts <= APT * BLOCK)
    uint32_t g[APT], hh[APT];
#pragma unroll
    for (uint32_t a = 0; a < APT; a++) {
      const uint32_t j = a * BLOCK + threadIdx.x;
      hh[a] = j < n_parts ? hist[j] : 0u;
      g[a] = hh[a] ? atomicAdd(pcount + j, hh[a]) : 0u;
      if (j < n_parts) {
        lp[j] = hh[a];
        hist[j] = 0u;  // ready for the next tile
      }
    }
    if (n_parts <= BLOCK) {
      // one partition per thread: warp scans, then every warp adds the
      // totals of the warps before it (two barriers in all)
      const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
      const uint32_t inc = warp_inclusive_scan(hh[0]);
      if (lane == 31) wsum[warp] = inc;
      __syncthreads();
      const uint32_t before = warp_sum((lane < (BLOCK / 32) && lane < warp) ? wsum[lane] : 0u);
      if (threadIdx.x < n_parts) lp[threadIdx.x] = before + inc - hh[0];
      __syncthreads();
    } else {
      __syncthreads();
      block_scan_segments<BLOCK>(lp, n_parts, 0u, 0u, wsum, [](uint32_t, uint32_t) {});
    }
#pragma unroll
    for (int u = 0; u < KPT; u++) {
      const uint32_t r = u * BLOCK + threadIdx.x;
      if (r < cnt) {
        const uint32_t p = pr[u] >> 16;
        const uint32_t pos = lp[p] + (pr[u] & 0xffffu);
        cur[pos] = k[u];
        sp[pos] = static_cast<uint16_t>(p);
        if constexpr (WITH_IDX) si[pos] = key_idx ? key_idx[base + r] : static_cast<uint32_t>(base + r);
      }
    }
    // sorted position s of partition p goes to element eoff[p] + s; a run
    // that would pass the partition's slots is dropped (EOFF_NONE) and flags
    // the overflow
#pragma unroll
    for (uint32_t a = 0; a < APT; a++) {
      const uint32_t j = a * BLOCK + threadIdx.x;
      if (j < n_parts) {
        if constexpr (EXACT) {
          eoff[j] = int64_t(g[a]) - int64_t(lp[j]);
        } else {
          const bool fits = uint64_t(g[a]) + hh[a] <= cap;
          overflow |= !fits;
          eoff[j] = fits ? int64_t(j) * int64_t(cap) + int64_t(g[a]) - int64_t(lp[j]) : EOFF_NONE;
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < KPT; u++) {
      const uint32_t s = u * BLOCK + threadIdx.x;
      if (s < cnt) {
        const int64_t e = eoff[sp[s]];
        if (e != EOFF_NONE) {
          pkeys[e + s] = cur[s];
          if constexpr (WITH_IDX) pidx[e + s] = si[s];
        }
      }
    }
    __syncthreads();
  }
  if (overflow) atomicOr(flags, FLAG_OVERFLOW);
}

// Pass 2: split every coarse partition S ways into fine partitions of W
// buckets.  One CTA per tile of a coarse partition's records (bulk-copied,
// the next tile prefetched while this one is sorted): a shared-memory
// counting sort by fine partition, one global atomic per (tile, fine
// partition) to reserve the run, coalesced run writes.
// Dynamic smem: eoff[S] (i64) | hist[S] | lp[S] | rk[2][TILE] | ri[2][TILE] | sp[TILE] (u16) | pstart[P+1]
template <typename KeyT, bool WITH_IDX, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_split(const KeyT* __restrict__ pkeys, const uint32_t* __restrict__ pidx,
                                                 const uint32_t* __restrict__ pstart, uint32_t n_parts, uint64_t cap1,
                                                 Div32 tpp, BucketMap bm, uint32_t fine_log2,
                                                 uint32_t split_log2, uint64_t capf, uint32_t* __restrict__ fcount,
                                                 KeyT* __restrict__ fkeys, uint32_t* __restrict__ fidx,
                                                 uint32_t* flags) {
  constexpr uint32_t KPT = 8;
  constexpr uint32_t TILE = BLOCK * KPT;
  if (entry_skip_on_overflow(flags)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t S = 1u << split_log2;
  int64_t* eoff = reinterpret_cast<int64_t*>(smem_raw);  // element offset of sorted position 0, per fine partition
  uint32_t* hist = reinterpret_cast<uint32_t*>(eoff + S);
  uint32_t* lp = hist + S;
  KeyT* rk = reinterpret_cast<KeyT*>(smem_raw + align_up_dev(size_t(S) * 16, 16));
  uint32_t* ri = reinterpret_cast<uint32_t*>(rk + 2 * TILE);
  uint16_t* sp = reinterpret_cast<uint16_t*>(ri + (WITH_IDX ? 2 * TILE : 0));
  uint32_t* sps = reinterpret_cast<uint32_t*>(sp + TILE);  // partition starts (n_parts + 1)
  for (uint32_t j = threadIdx.x; j <= n_parts; j += BLOCK) sps[j] = pstart[j];
  __syncthreads();
  __shared__ uint64_t bar[2];
  __shared__ uint64_t s_next;
  __shared__ uint32_t s_next_cnt;
  __shared__ uint32_t s_wsum[BLOCK / 32];
  const uint32_t coarse_log2 = fine_log2 + split_log2;
  const uint32_t tiles_per_part = tpp.d;
  const uint64_t vtiles = uint64_t(n_parts) * tiles_per_part;  // below 2^32 (the planner keeps it so)
  // first valid virtual tile at or after vt (stepping by the grid); vtiles if none
  auto next_valid = [&](uint64_t vt, uint32_t* cnt) -> uint64_t {
    for (; vt < vtiles; vt += gridDim.x) {
      const uint32_t q = tpp.div(static_cast<uint32_t>(vt));
      const uint32_t r0 = (static_cast<uint32_t>(vt) - q * tiles_per_part) * TILE;
      const uint32_t m = sps[q + 1] - sps[q];
      if (r0 < m) {
        *cnt = min(TILE, m - r0);
        return vt;
      }
    }
    *cnt = 0;
    return vtiles;
  };
  auto issue = [&](uint64_t vt, uint32_t cnt, uint32_t buf) {
    const uint64_t q = tpp.div(static_cast<uint32_t>(vt));
    const uint64_t r0 = uint64_t(static_cast<uint32_t>(vt) - static_cast<uint32_t>(q) * tiles_per_part) * TILE;
    const uint32_t bk = (cnt * uint32_t(sizeof(KeyT)) + 15u) & ~15u;  // stays inside the partition's slots
    const uint32_t bi = WITH_IDX ? ((cnt * 4u + 15u) & ~15u) : 0u;
    mbar_arrive_expect_tx(&bar[buf], bk + bi);
    bulk_g2s(rk + buf * TILE, pkeys + q * cap1 + r0, bk, &bar[buf]);
    if constexpr (WITH_IDX) bulk_g2s(ri + buf * TILE, pidx + q * cap1 + r0, bi, &bar[buf]);
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
    uint32_t c0;
    const uint64_t v0 = next_valid(blockIdx.x, &c0);
    if (v0 < vtiles) issue(v0, c0, 0);
    s_next = v0;
    s_next_cnt = c0;
  }
  __syncthreads();
  bool overflow = false;
  uint32_t it = 0;
  while (true) {
    const uint64_t vt = s_next;
    const uint32_t cnt = s_next_cnt;
    if (vt >= vtiles) break;
    const uint32_t buf = it & 1;
    __syncthreads();  // everyone has read s_next before thread 0 moves it
    if (threadIdx.x == 0) {
      uint32_t cn;
      const uint64_t nx = next_valid(vt + gridDim.x, &cn);
      if (nx < vtiles) {
        fence_proxy_async_smem();
        issue(nx, cn, buf ^ 1u);
      }
      s_next = nx;
      s_next_cnt = cn;
    }
    const uint64_t q = tpp.div(static_cast<uint32_t>(vt));
    const uint64_t b0 = q << coarse_log2;
    KeyT* ck = rk + buf * TILE;
    uint32_t* ci = ri + buf * TILE;
    for (uint32_t j = threadIdx.x; j < S; j += BLOCK) hist[j] = 0u;
    if (threadIdx.x == 0) mbar_wait(&bar[buf], (it >> 1) & 1);  // published by the barrier below
    __syncthreads();
    KeyT kk[KPT];
    uint32_t ii[KPT], pp[KPT];
#pragma unroll
    for (int u = 0; u < KPT; u++) {
      const uint32_t r = u * BLOCK + threadIdx.x;
      if (r < cnt) {
        kk[u] = ck[r];
        if constexpr (WITH_IDX) ii[u] = ci[r];
        const uint32_t f = static_cast<uint32_t>(bm.of_key(kk[u]) - b0) >> fine_log2;
        pp[u] = (f << 16) | atomicAdd(&hist[f], 1u);
      }
    }
    __syncthreads();
    // reservations (S <= 2 * BLOCK): issued now, consumed after the local
    // scan and sort, which hides the atomics' round trip
    uint32_t g[2], hh[2];
#pragma unroll
    for (uint32_t a = 0; a < 2; a++) {
      const uint32_t f = a * BLOCK + threadIdx.x;
      hh[a] = f < S ? hist[f] : 0u;
      g[a] = hh[a] ? atomicAdd(fcount + (q << split_log2) + f, hh[a]) : 0u;
    }
    if (S <= BLOCK) {
      // one fine partition per thread: warp scans, then every warp adds the
      // totals of the warps before it
      const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
      const uint32_t inc = warp_inclusive_scan(hh[0]);
      if (lane == 31) s_wsum[warp] = inc;
      __syncthreads();
      const uint32_t before = warp_sum((lane < (BLOCK / 32) && lane < warp) ? s_wsum[lane] : 0u);
      if (threadIdx.x < S) lp[threadIdx.x] = before + inc - hh[0];
    } else if (threadIdx.x < 32) {  // exclusive scan of S <= 1024 counts by one warp
      uint32_t run = 0;
      for (uint32_t j0 = 0; j0 < S; j0 += 32) {
        const uint32_t j = j0 + threadIdx.x;
        const uint32_t v = j < S ? hist[j] : 0u;
        const uint32_t inc = warp_inclusive_scan(v);
        if (j < S) lp[j] = run + inc - v;
        run += __shfl_sync(FULL_MASK, inc, 31);
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < KPT; u++) {
      const uint32_t r = u * BLOCK + threadIdx.x;
      if (r < cnt) {
        const uint32_t f = pp[u] >> 16;
        const uint32_t pos = lp[f] + (pp[u] & 0xffffu);
        ck[pos] = kk[u];
        sp[pos] = static_cast<uint16_t>(f);
        if constexpr (WITH_IDX) ci[pos] = ii[u];
      }
    }
    // sorted position s of fine partition f goes to element eoff[f] + s; a
    // run that would pass the partition's slots is dropped and flags the
    // overflow
#pragma unroll
    for (uint32_t a = 0; a < 2; a++) {
      const uint32_t f = a * BLOCK + threadIdx.x;
      if (f < S) {
        const bool fits = uint64_t(g[a]) + hh[a] <= capf;
        overflow |= !fits;
        eoff[f] = fits ? int64_t((q << split_log2) + f) * int64_t(capf) + int64_t(g[a]) - int64_t(lp[f]) : EOFF_NONE;
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < KPT; u++) {
      const uint32_t s = u * BLOCK + threadIdx.x;
      if (s < cnt) {
        const int64_t e = eoff[sp[s]];
        if (e != EOFF_NONE) {
          fkeys[e + s] = ck[s];
          if constexpr (WITH_IDX) fidx[e + s] = ci[s];
        }
      }
    }
    __syncthreads();
    it++;
  }
  if (overflow) atomicOr(flags, FLAG_OVERFLOW);
}

// Pass 3: one CTA per fine partition of W buckets.  The partition's records
// are bulk-copied into shared memory (the next partition's copy is in flight
// meanwhile).  Each record is hashed once: a shared-memory atomic on its
// bucket's counter gives its rank, kept with the bucket as (bucket << 16 |
// rank).  The counters are scanned into the partition's offsets (coalesced
// write) and every record goes to offsets[bucket] + rank in the partition's
// output slice (a few tens of KB, completed while resident in L2).
// Dynamic smem: ctr[2][W] | sk[2][capf] | si[2][capf] | sr[capf]
// One pass-3 partition of a build: its records and the table they go to.
template <typename KeyT>
struct FinePart {
  const KeyT* rkeys;      // the partition's record slots
  const uint32_t* ridx;
  uint64_t b0;            // first bucket of the partition in its table
  uint32_t nb;            // buckets of the partition
  BucketMap bm;
  uint32_t* offsets;      // the table's arrays
  KeyT* keys_out;
  uint32_t* idx_out;
};

// Pass-3 partitions of one table: partition f holds buckets [f*W, (f+1)*W);
// its records sit at slot f*capf and its output starts at fstart[f].
template <typename KeyT>
struct TableFine {
  const KeyT* fkeys;
  const uint32_t* fidx;
  const uint32_t* fstart;
  uint64_t n_fine, capf;
  uint32_t fine_log2;
  BucketMap bm;
  uint64_t n_buckets;
  uint32_t* offsets;
  KeyT* keys_out;
  uint32_t* idx_out;
  __device__ __forceinline__ uint64_t count() const {
    return umin64(n_fine, (n_buckets + (1ull << fine_log2) - 1) >> fine_log2);  // partitions holding buckets
  }
  // (first, end) of partition f's records in the table's CSR order
  __device__ __forceinline__ uint2 meta(uint64_t f) const { return make_uint2(fstart[f], fstart[f + 1]); }
  __device__ __forceinline__ FinePart<KeyT> at(uint64_t f) const {
    const uint64_t b0 = f << fine_log2;
    const uint32_t nb = static_cast<uint32_t>(umin64(1ull << fine_log2, n_buckets - b0));
    return FinePart<KeyT>{fkeys + f * capf, fidx + f * capf, b0, nb, bm, offsets, keys_out, idx_out};
  }
  // thread 0 of the CTA that takes partition f: the table's last offset
  __device__ __forceinline__ void finish(uint64_t f) const {
    if (f == 0) offsets[n_buckets] = fstart[n_fine];
  }
};

template <typename KeyT, bool WITH_IDX, int BLOCK, typename Src>
__global__ void __launch_bounds__(BLOCK) k_fine_build(Src src, uint64_t capf, uint32_t fine_log2,
                                                      const uint32_t* flags) {
  if (entry_skip_on_overflow(flags)) return;
  constexpr int NW = BLOCK / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t W = 1u << fine_log2;
  uint32_t* ctr2 = reinterpret_cast<uint32_t*>(smem_raw);
  KeyT* sk = reinterpret_cast<KeyT*>(smem_raw + align_up_dev(size_t(W) * 8, 16));
  uint32_t* si = reinterpret_cast<uint32_t*>(sk + 2 * capf);
  uint32_t* sr = si + (WITH_IDX ? 2 * capf : 0);
  uint16_t* sperm = reinterpret_cast<uint16_t*>(sr + capf);  // record at each output position
  __shared__ uint32_t wsum[NW + 1];
  __shared__ uint64_t bar[2];
  __shared__ uint32_t s_base[2], s_m[2];
  const uint64_t n_live = src.count();
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  // thread 0 loads a partition's start and size one iteration before it issues its copy
  auto load_meta = [&](uint64_t f) -> uint2 { return f < n_live ? src.meta(f) : make_uint2(0u, 0u); };
  auto issue = [&](uint64_t f, uint32_t buf, uint2 mt) {
    uint32_t m = mt.y - mt.x;
    if (mt.y < mt.x || m > capf) {  // a partition larger than its slots: bad device state
      record_fault(HG_ERR_DEVICE_STATE);
      m = 0;
    }
    s_base[buf] = mt.x;
    s_m[buf] = m;
    const FinePart<KeyT> fp = src.at(f);
    const uint32_t bk = (m * uint32_t(sizeof(KeyT)) + 15u) & ~15u;  // stays inside the partition's slots
    const uint32_t bi = WITH_IDX ? ((m * 4u + 15u) & ~15u) : 0u;
    mbar_arrive_expect_tx(&bar[buf], bk + bi);
    if (bk) bulk_g2s(sk + buf * capf, fp.rkeys, bk, &bar[buf]);
    if constexpr (WITH_IDX) {
      if (bi) bulk_g2s(si + buf * capf, fp.ridx, bi, &bar[buf]);
    }
  };
  uint2 next_meta = make_uint2(0u, 0u);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
    if (blockIdx.x < n_live) issue(blockIdx.x, 0, load_meta(blockIdx.x));
    next_meta = load_meta(blockIdx.x + gridDim.x);
  }
  for (uint32_t j = threadIdx.x; j < W; j += BLOCK) ctr2[j] = 0u;
  uint32_t it = 0;
  for (uint64_t f = blockIdx.x; f < n_live; f += gridDim.x, it++) {
    const uint32_t buf = it & 1;
    const FinePart<KeyT> fp = src.at(f);
    const uint64_t b0 = fp.b0;
    const uint32_t nb = fp.nb;
    const BucketMap bm = fp.bm;
    uint32_t* offsets = fp.offsets;
    KeyT* keys_out = fp.keys_out;
    uint32_t* idx_out = fp.idx_out;
    const bool off_vec = (reinterpret_cast<uintptr_t>(offsets) & 15u) == 0;
    if (threadIdx.x == 0) {
      src.finish(f);
      mbar_wait(&bar[buf], (it >> 1) & 1);
    }
    // the copy landed (published by this barrier) and every thread finished
    // the previous partition: its buffer and counters are free
    __syncthreads();
    if (threadIdx.x == 0 && f + gridDim.x < n_live) {
      fence_proxy_async_smem();
      issue(f + gridDim.x, buf ^ 1u, next_meta);
      next_meta = load_meta(f + 2 * uint64_t(gridDim.x));  // consumed next iteration
    }
    uint32_t* ctr = ctr2 + buf * W;
    uint32_t* ctr_next = ctr2 + (buf ^ 1u) * W;
    const KeyT* ck = sk + buf * capf;
    const uint32_t* ci = si + buf * capf;
    const uint32_t base = s_base[buf];
    const uint32_t m = s_m[buf];
    for (uint32_t j = threadIdx.x; j < W; j += BLOCK) ctr_next[j] = 0u;  // for the next partition
    for (uint32_t r = threadIdx.x; r < m; r += BLOCK) {
      const uint32_t lb = static_cast<uint32_t>(bm.of_key(ck[r]) - b0);
      sr[r] = (lb << 16) | atomicAdd(&ctr[lb], 1u);
    }
    __syncthreads();
    if (nb == 4 * BLOCK) {
      // four counters per thread: warp scans of the thread sums; after one
      // barrier every warp sums the totals of the warps before it itself
      // (wsum is next written after the next partition's first barrier)
      const uint4 v = reinterpret_cast<const uint4*>(ctr)[threadIdx.x];
      const uint32_t sum = v.x + v.y + v.z + v.w;
      const uint32_t inc = warp_inclusive_scan(sum);
      if (lane == 31) wsum[warp] = inc;
      __syncthreads();
      const uint32_t wt = (lane < NW && lane < warp) ? wsum[lane] : 0u;
      const uint32_t before = warp_sum(wt);
      uint4 o;
      o.x = base + before + inc - sum;
      o.y = o.x + v.x;
      o.z = o.y + v.y;
      o.w = o.z + v.z;
      reinterpret_cast<uint4*>(ctr)[threadIdx.x] = o;
      uint32_t* dst = offsets + b0 + 4 * threadIdx.x;
      if (off_vec) {
        *reinterpret_cast<uint4*>(dst) = o;
      } else {
        dst[0] = o.x;
        dst[1] = o.y;
        dst[2] = o.z;
        dst[3] = o.w;
      }
      __syncthreads();  // the scatter reads any bucket's start
    } else if (nb == 8 * BLOCK) {
      // eight counters per thread, the same scheme with two vectors
      const uint4 v0 = reinterpret_cast<const uint4*>(ctr)[2 * threadIdx.x];
      const uint4 v1 = reinterpret_cast<const uint4*>(ctr)[2 * threadIdx.x + 1];
      const uint32_t s0 = v0.x + v0.y + v0.z + v0.w;
      const uint32_t sum = s0 + v1.x + v1.y + v1.z + v1.w;
      const uint32_t inc = warp_inclusive_scan(sum);
      if (lane == 31) wsum[warp] = inc;
      __syncthreads();
      const uint32_t wt = (lane < NW && lane < warp) ? wsum[lane] : 0u;
      const uint32_t before = warp_sum(wt);
      uint4 o0, o1;
      o0.x = base + before + inc - sum;
      o0.y = o0.x + v0.x;
      o0.z = o0.y + v0.y;
      o0.w = o0.z + v0.z;
      o1.x = o0.w + v0.w;
      o1.y = o1.x + v1.x;
      o1.z = o1.y + v1.y;
      o1.w = o1.z + v1.z;
      reinterpret_cast<uint4*>(ctr)[2 * threadIdx.x] = o0;
      reinterpret_cast<uint4*>(ctr)[2 * threadIdx.x + 1] = o1;
      uint32_t* dst = offsets + b0 + 8 * threadIdx.x;
      if (off_vec) {
        reinterpret_cast<uint4*>(dst)[0] = o0;
        reinterpret_cast<uint4*>(dst)[1] = o1;
      } else {
        dst[0] = o0.x; dst[1] = o0.y; dst[2] = o0.z; dst[3] = o0.w;
        dst[4] = o1.x; dst[5] = o1.y; dst[6] = o1.z; dst[7] = o1.w;
      }
      __syncthreads();
    } else {
      block_scan_segments<BLOCK>(ctr, nb, base, base, wsum, [&](uint32_t j, uint32_t g) { offsets[b0 + j] = g; });
    }
    // the partition's output is the contiguous range [base, base + m): each
    // record's position goes into shared memory, then the keys (and
    // indices) leave in position order with coalesced stores
    for (uint32_t r = threadIdx.x; r < m; r += BLOCK) {
      const uint32_t v = sr[r];
      sperm[ctr[v >> 16] + (v & 0xffffu) - base] = static_cast<uint16_t>(r);
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < m; q += BLOCK) {
      const uint32_t r = sperm[q];
      keys_out[base + q] = ck[r];
      if constexpr (WITH_IDX) {
        if (idx_out) idx_out[base + q] = ci[r];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
int device_sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
      sms = 148;
    cached[dev] = sms;
  }
  return cached[dev];
}

template <typename KeyT, int V>
static void launch_direct_count(const KeyT* keys, uint64_t n, BucketMap bm, uint32_t* cnt, const uint32_t* gate,
                                cudaStream_t s) {
  const uint64_t chunks = (n + 32ull * V - 1) / (32ull * V);
  const uint64_t want = (chunks + 7) / 8;
  const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(device_sm_count()) * 8)));
  Phase ph(s, gate ? "fallback_count" : "count");
  count_launch();
  if (gate) {  // the fallback runs under skew: CTA-aggregated counting
    const uint64_t cchunks = (n + SKEW_CHUNK - 1) / SKEW_CHUNK;
    const unsigned sgrid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(cchunks, uint64_t(device_sm_count()) * 4)));
    k_count_skew<KeyT><<<sgrid, SKEW_BLOCK, 0, s>>>(keys, n, bm, cnt, gate);
    return;
  }
  k_count<KeyT, V><<<grid, 256, 0, s>>>(keys, n, bm, cnt, gate);
}

template <typename KeyT, int V, bool WI>
static void launch_direct_scatter(const KeyT* keys, uint64_t n, BucketMap bm, uint32_t* cursor, KeyT* out,
                                  uint32_t* idx, const uint32_t* key_idx, const uint32_t* gate, cudaStream_t s) {
  const uint64_t chunks = (n + 32ull * V - 1) / (32ull * V);
  const uint64_t want = (chunks + 7) / 8;
  const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(device_sm_count()) * 8)));
  Phase ph(s, gate ? "fallback_scatter" : "scatter");
  count_launch();
  if (gate) {  // the fallback runs under skew: CTA-aggregated cursor bumps
    const uint64_t cchunks = (n + SKEW_CHUNK - 1) / SKEW_CHUNK;
    const unsigned sgrid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(cchunks, uint64_t(device_sm_count()) * 4)));
    k_scatter_skew<KeyT, WI><<<sgrid, SKEW_BLOCK, 0, s>>>(keys, n, bm, cursor, out, idx, key_idx, gate);
    return;
  }
  k_scatter<KeyT, V, WI><<<grid, 256, 0, s>>>(keys, n, bm, cursor, out, idx, key_idx, gate);
}

static void launch_scan(uint32_t* data, uint64_t count, uint64_t* status, unsigned* ticket, uint32_t* first_slot,
                        uint32_t* total_out, const uint32_t* gate, cudaStream_t s, const char* name = nullptr) {
  const uint64_t tiles = (count + SCAN_TILE - 1) / SCAN_TILE;
  if (tiles == 0) return;
  Phase ph(s, name ? name : (gate ? "fallback_scan" : "scan"));
  count_launch();
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(tiles, uint64_t(device_sm_count()) * 8));
  k_scan_u32<SCAN_BLOCK, SCAN_ITEMS><<<grid, SCAN_BLOCK, 0, s>>>(data, count, status, ticket, first_slot, total_out,
                                                                 gate);
}

template <typename KeyT, int V, bool WI>
static hg_status run_direct(const BuildPlan& p, const KeyT* keys, uint32_t* offsets, KeyT* keys_out, uint32_t* idx_out,
                            char* ws, const uint32_t* gate, cudaStream_t s, const uint32_t* key_idx) {
  const BucketMap bm = p.bucket_map();
  uint64_t* status = reinterpret_cast<uint64_t*>(ws + p.off_status);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  if (gate) {
    const int grid = static_cast<int>(std::min<uint64_t>((p.n_buckets + 1 + 255) / 256, uint64_t(device_sm_count()) * 8));
    Phase ph(s, "fallback_fill");
    count_launch();
    k_fill_u32<<<std::max(grid, 1), 256, 0, s>>>(offsets, p.n_buckets + 1, 0u, gate);
  } else {
    HG_CUDA(cudaMemsetAsync(offsets, 0, (p.n_buckets + 1) * sizeof(uint32_t), s), "build: offsets memset");
  }
  HG_CUDA(cudaMemsetAsync(ws + p.off_status, 0, p.off_flags - p.off_status, s), "build: scan state memset");
  if (p.n > 0) launch_direct_count<KeyT, V>(keys, p.n, bm, offsets + 1, gate, s);
  launch_scan(offsets + 1, p.n_buckets, status, ticket, offsets, nullptr, gate, s);
  if (p.n > 0) launch_direct_scatter<KeyT, V, WI>(keys, p.n, bm, offsets + 1, keys_out, idx_out, key_idx, gate, s);
  return HG_OK;
}

uint64_t slack_capacity(double mean, uint64_t margin, double sigmas) {
  const uint64_t c = static_cast<uint64_t>(std::ceil(mean + sigmas * std::sqrt(mean) + double(margin)));
  return (c + 31) & ~31ull;
}

static uint32_t ceil_log2_u64(uint64_t x) {
  uint32_t l = 0;
  while ((1ull << l) < x) l++;
  return l;
}

size_t pass1_smem(uint64_t n_parts, int key_bytes, int tile) {
  return align_up(16 * n_parts, 16) + size_t(tile) * (2 * key_bytes + 6);
}

size_t split_smem(uint32_t split_log2, int key_bytes, bool with_index, uint64_t n_parts, int tile) {
  return align_up(16 * (size_t(1) << split_log2), 16) + size_t(tile) * (2 * key_bytes + (with_index ? 8 : 0) + 2) +
         (n_parts + 1) * 4;
}

// Splits of 512 or 1024 ways take one 1024-thread CTA per SM over 8192-record
// tiles when that fits in shared memory, so that a tile's run in each fine
// partition stays 8 or more records long (2^30 u32 keys + index, 1024 ways:
// the split's runs were 4 records); narrower splits keep 512-thread CTAs.
void plan_split(PartGeometry& g, int key_bytes, bool with_index) {
  g.split_block = SPLIT_BLOCK;
  if (g.split_log2 >= 9) {
    const size_t wide = split_smem(g.split_log2, key_bytes, with_index, g.n_parts, 8 * SPLIT_BLOCK_WIDE);
    if (wide <= SMEM_BUDGET) g.split_block = SPLIT_BLOCK_WIDE;
  }
  g.smem2 = split_smem(g.split_log2, key_bytes, with_index, g.n_parts, 8 * g.split_block);
}

bool plan_geometry(uint64_t n_stream, size_t stream_rec, uint64_t n_staged, size_t smem_rec, size_t per_bucket,
                   size_t stream_smem, uint64_t n_buckets, bool staged_may_spill, PartGeometry* out,
                   size_t fine_budget) {
  PartGeometry g;
  bool found = false;
  const size_t FINE_SMEM_BUDGET = fine_budget;
  // tuning overrides: HG_FINE_LOG2 caps the fine width (W = 2^value buckets),
  // HG_SPLIT_LOG2 caps the pass-2 split factor
  uint32_t w_max = 15, s_max = SPLIT_LOG2_MAX;
  if (const char* e = std::getenv("HG_FINE_LOG2")) w_max = std::max(6, std::min(15, std::atoi(e)));
  if (const char* e = std::getenv("HG_SPLIT_LOG2")) s_max = std::max(0, std::min(10, std::atoi(e)));
  for (uint32_t w = w_max; w >= 6 && !found; w--) {
    const uint64_t W = 1ull << w;
    const double frac = double(std::min<uint64_t>(W, n_buckets)) / double(n_buckets);
    // a probe's staged slice may spill (read in place), so it takes less slack
    const uint64_t cap = slack_capacity(double(n_staged) * frac, 64, staged_may_spill ? 4.0 : 8.0);
    const uint64_t qcap = stream_smem ? slack_capacity(double(n_stream) * frac, 64) : 0;
    const size_t bytes = align_up(per_bucket * (W + 1), 16) + cap * smem_rec + qcap * stream_smem;
    if (bytes <= FINE_SMEM_BUDGET) {
      g.fine_log2 = w;
      g.smem_cap = static_cast<uint32_t>(cap);
      g.smem3 = bytes;
      found = true;
    }
  }
  if (!found) {
    if (!staged_may_spill) return false;
    g.fine_log2 = 6;
    const double frac = double(std::min<uint64_t>(64, n_buckets)) / double(n_buckets);
    const uint64_t qcap = stream_smem ? slack_capacity(double(n_stream) * frac, 64) : 0;
    const size_t head = align_up(per_bucket * ((size_t(1) << 6) + 1), 16) + qcap * stream_smem;
    if (head + 32 * smem_rec > FINE_SMEM_BUDGET) return false;
    g.smem_cap = static_cast<uint32_t>((FINE_SMEM_BUDGET - head) / smem_rec) & ~31u;
    g.smem3 = head + size_t(g.smem_cap) * smem_rec;
  }
  const uint64_t W = 1ull << g.fine_log2;
  g.split_log2 = std::min<uint32_t>(s_max, ceil_log2_u64((n_buckets + W - 1) / W));
  // Pass 1 slows down sharply above PASS1_GOOD_PARTS coarse partitions (runs
  // of a few keys per tile, more reservations): split wider, up to 1024 ways,
  // until the coarse partitions are at most that many (measured on 2^30 u32
  // keys + index: 512 partitions with a 1024-way split beat 2048 with 256-way
  // by 14%).  PASS1_MAX_PARTS is the hard limit of the pass-1 kernel.
  auto parts_at = [&](uint32_t sl) {
    return (n_buckets + (1ull << (g.fine_log2 + sl)) - 1) >> (g.fine_log2 + sl);
  };
  while (g.split_log2 < 10 && !std::getenv("HG_SPLIT_LOG2") && parts_at(g.split_log2) > PASS1_GOOD_PARTS)
    g.split_log2++;
  while (g.split_log2 < 10 && parts_at(g.split_log2) > PASS1_MAX_PARTS) g.split_log2++;
  g.coarse_log2 = g.fine_log2 + g.split_log2;
  g.n_parts = (n_buckets + (1ull << g.coarse_log2) - 1) >> g.coarse_log2;
  if (g.n_parts > PASS1_MAX_PARTS) return false;
  g.n_fine = g.n_parts << g.split_log2;
  g.part_cap = slack_capacity(double(n_stream) * double(std::min<uint64_t>(1ull << g.coarse_log2, n_buckets)) /
                                  double(n_buckets), 256);
  g.fine_cap = slack_capacity(double(n_stream) * double(std::min<uint64_t>(W, n_buckets)) / double(n_buckets), 64);
  // pass 1: hist/lp/start per coarse partition + a sorted tile (keys, index,
  // 16-bit partition ids)
  g.tile1 = PASS1_TILE;
  // pass 1: hist/lp/start, two raw key tiles, the index and the 16-bit
  // partition id of the sorted tile (sizes set by the caller, which knows the
  // key width: pass1_smem / split_smem)
  g.smem1 = 0;
  g.smem2 = 0;
  g.pscan_tiles = (g.n_parts + SCAN_TILE - 1) / SCAN_TILE;
  g.fscan_tiles = (g.n_fine + SCAN_TILE - 1) / SCAN_TILE;
  if (g.n_parts >= 65536 || g.part_cap >= (1ull << 32) || g.fine_cap >= (1ull << 32)) return false;
  *out = g;
  return true;
}

hg_status plan_build(uint64_t n, int key_bytes, uint64_t n_buckets, bool with_index, BuildPlan* plan, int force_path) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0) return HG_ERR_INVALID_ARGUMENT;
  if (n >= (1ull << 32) || n_buckets > (1ull << 32)) return HG_ERR_TOO_LARGE;
  BuildPlan p;
  p.n = n;
  p.n_buckets = n_buckets;
  p.key_bytes = key_bytes;
  p.with_index = with_index;
  const size_t rec = key_bytes + (with_index ? 4 : 0);
  // pass 3 double-buffers its partition's records (2 * rec per staged
  // record) and its bucket counters (8 bytes per bucket), and keeps a 4-byte
  // (bucket, rank) word and a 2-byte output-position entry per record
  size_t budget = FINE_SMEM_BUDGET;
  if (const char* e = std::getenv("HG_BUILD_SMEM_KB")) {  // tuning override of the fine-build CTA's budget
    const int kb = std::atoi(e);
    if (kb >= 16 && kb <= 220) budget = size_t(kb) * 1024;
  }
  bool part_ok = plan_geometry(n, rec, n, 2 * rec + 6, 8, 0, n_buckets, false, &p.g, budget);
  // ranks within a bucket and local bucket numbers are packed in 16 bits
  if (part_ok && (p.g.fine_cap >= 65536 || p.g.fine_log2 > 16)) part_ok = false;
  if (part_ok) {
    p.g.tile1 = pass1_tile(key_bytes);
    p.g.smem1 = pass1_smem(p.g.n_parts, key_bytes, p.g.tile1);
    plan_split(p.g, key_bytes, with_index);
    part_ok = p.g.smem1 <= SMEM_BUDGET && p.g.smem2 <= SMEM_BUDGET;
  }
  // the partitioned path pays off with many keys; a sparse table (few keys,
  // many buckets) stays direct, whose workspace is O(buckets / 4096) where the
  // partitioned one keeps slack slots in every partition (O(buckets))
  const uint64_t footprint = n * (key_bytes + rec);
  int path = force_path;
  if (path < 0) path = (part_ok && footprint > (48ull << 20)) ? BUILD_PARTITIONED : BUILD_DIRECT;
  // A table too dense to stage a fine partition in shared memory (a few
  // buckets holding everything) takes the direct path even when asked for
  // the partitioned one.
  if (path == BUILD_PARTITIONED && !part_ok) path = BUILD_DIRECT;
  p.path = path;
  size_t off = 0;
  p.scan_tiles = (n_buckets + SCAN_TILE - 1) / SCAN_TILE;
  p.off_status = off;  off = align_up(off + p.scan_tiles * 8);
  p.off_ticket = off;  off = align_up(off + 8 * sizeof(unsigned));
  p.off_flags = off;   off = align_up(off + sizeof(uint32_t));
  if (path == BUILD_PARTITIONED) {
    const PartGeometry& g = p.g;
    p.off_pcount = off;  off = align_up(off + (g.n_parts + 1) * 4);
    p.off_pstatus = off; off = align_up(off + g.pscan_tiles * 8);
    p.off_fcount = off;  off = align_up(off + (g.n_fine + 1) * 4);
    p.off_fstatus = off; off = align_up(off + g.fscan_tiles * 8);
    p.off_gcount = off;  off = align_up(off + (g.n_parts + 1) * 4);
    p.off_gstatus = off; off = align_up(off + g.pscan_tiles * 8);
    p.off_pkeys = off;   off = align_up(off + g.n_parts * g.part_cap * key_bytes);
    if (with_index) { p.off_pidx = off; off = align_up(off + g.n_parts * g.part_cap * 4); }
    p.off_fkeys = off;   off = align_up(off + g.n_fine * g.fine_cap * key_bytes);
    if (with_index) { p.off_fidx = off; off = align_up(off + g.n_fine * g.fine_cap * 4); }
  } else {
    p.off_pcount = p.off_pstatus = p.off_fcount = p.off_fstatus = off;
    p.off_gcount = p.off_gstatus = off;
    p.off_pkeys = p.off_pidx = p.off_fkeys = p.off_fidx = off;
  }
  p.total = std::max<size_t>(off, WS_ALIGN);
  *plan = p;
  return HG_OK;
}

// Raises a kernel's dynamic shared-memory limit to the device maximum (minus
// its static shared memory) once, and returns co-resident CTAs per SM for
// `smem` bytes (0 if it cannot run).
template <typename Kern>
static int blocks_per_sm(Kern kern, unsigned block, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, size_t, unsigned, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(reinterpret_cast<const void*>(kern), smem, block, dev);
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa = {};
  cudaFuncGetAttributes(&fa, kern);
  const int max_dyn = optin - static_cast<int>(fa.sharedSizeBytes);
  int n = 0;
  if (max_dyn >= 0 && size_t(max_dyn) >= smem &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn) == cudaSuccess)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, static_cast<int>(block), smem);
  cudaGetLastError();
  std::lock_guard<std::mutex> g(mu);
  cache[key] = n;
  return n;
}

// Pass 1 over `n` streamed keys (with their input positions when WI): the
// per-CTA multisplit into g.n_parts coarse partitions of 2^g.coarse_log2
// buckets, record slots p * g.part_cap, counts in pcount[p].
template <typename KeyT, int V, bool WI>
static hg_status launch_pass1(const PartGeometry& g, uint64_t n, const KeyT* keys, const uint32_t* key_idx,
                              BucketMap bm, uint32_t* pcount, KeyT* pkeys, uint32_t* pidx, uint32_t* flags,
                              const char* name, cudaStream_t s) {
  if (n == 0) return HG_OK;
  constexpr int BLK = pass1_block(sizeof(KeyT)), TILE = pass1_tile(sizeof(KeyT));
  auto kern = k_multisplit<KeyT, WI, BLK, PASS1_KPT, (V > 1), TableTiles<KeyT, TILE>>;
  const int bps = blocks_per_sm(kern, BLK, g.smem1);
  if (bps <= 0) return lib_fail(HG_ERR_CUDA, "multisplit kernel cannot be resident");
  const uint64_t ntiles = (n + TILE - 1) / TILE;
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(ntiles, uint64_t(device_sm_count()) * bps));
  Phase ph(s, name);
  count_launch();
  k_skew_check<KeyT><<<1, SKEW_CHECK_BLOCK, 0, s>>>(keys, n, bm, g.coarse_log2, static_cast<uint32_t>(g.n_parts),
                                                    g.part_cap, flags);
  count_launch();
  using Src = TableTiles<KeyT, TILE>;
  const Src src{keys, key_idx, n, bm, g.coarse_log2, static_cast<uint32_t>(g.n_parts), g.part_cap, pcount, pkeys, pidx};
  kern<<<grid, BLK, g.smem1, s>>>(src, static_cast<uint32_t>(g.n_parts), flags);
  HG_CUDA(cudaPeekAtLastError(), "multisplit launch");
  return HG_OK;
}

// Passes 1 and 2 of a partitioned path over `n` streamed keys (with their
// input positions when WI): cluster multisplit into coarse partitions, scan,
// split into fine partitions, scan.  Shared by the build and the probe.
template <typename KeyT, int V, bool WI>
static hg_status run_partition_passes(const PartGeometry& g, uint64_t n, const KeyT* keys, const uint32_t* key_idx,
                                      BucketMap bm, char* ws, size_t off_flags, size_t off_ticket, size_t off_pcount,
                                      size_t off_pstatus, size_t off_fcount, size_t off_fstatus, size_t off_pkeys,
                                      size_t off_pidx, size_t off_fkeys, size_t off_fidx, const char* who,
                                      cudaStream_t s) {
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + off_flags);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + off_ticket);
  uint32_t* pcount = reinterpret_cast<uint32_t*>(ws + off_pcount);
  uint64_t* pstatus = reinterpret_cast<uint64_t*>(ws + off_pstatus);
  uint32_t* fcount = reinterpret_cast<uint32_t*>(ws + off_fcount);
  uint64_t* fstatus = reinterpret_cast<uint64_t*>(ws + off_fstatus);
  KeyT* pkeys = reinterpret_cast<KeyT*>(ws + off_pkeys);
  uint32_t* pidx = WI ? reinterpret_cast<uint32_t*>(ws + off_pidx) : nullptr;
  KeyT* fkeys = reinterpret_cast<KeyT*>(ws + off_fkeys);
  uint32_t* fidx = WI ? reinterpret_cast<uint32_t*>(ws + off_fidx) : nullptr;
  hg_status st = launch_pass1<KeyT, V, WI>(g, n, keys, key_idx, bm, pcount, pkeys, pidx, flags,
                                          who[0] == 'b' ? "multisplit" : "probe_multisplit", s);
  if (st != HG_OK) return st;
  launch_scan(pcount, g.n_parts, pstatus, ticket + 1, nullptr, pcount + g.n_parts, nullptr, s,
              who[0] == 'b' ? "part_scan" : "probe_part_scan");
  auto split = [&](auto block_c) -> hg_status {
    constexpr int BLK = decltype(block_c)::value;
    auto kern = k_split<KeyT, WI, BLK>;
    const int bps = blocks_per_sm(kern, BLK, g.smem2);
    if (bps <= 0) return lib_fail(HG_ERR_CUDA, "split kernel cannot be resident");
    const uint32_t tile = 8 * BLK;
    const uint32_t tiles_per_part = static_cast<uint32_t>((g.part_cap + tile - 1) / tile);
    const uint64_t vt = g.n_parts * tiles_per_part;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(vt, uint64_t(device_sm_count()) * bps));
    Phase ph(s, who[0] == 'b' ? "split" : "probe_split");
    count_launch();
    kern<<<std::max(grid, 1u), BLK, g.smem2, s>>>(
        pkeys, pidx, pcount, static_cast<uint32_t>(g.n_parts), g.part_cap, Div32::make(tiles_per_part), bm, g.fine_log2,
        g.split_log2, g.fine_cap, fcount, fkeys, fidx, flags);
    HG_CUDA(cudaPeekAtLastError(), "split launch");
    return HG_OK;
  };
  st = g.split_block == SPLIT_BLOCK_WIDE ? split(std::integral_constant<int, SPLIT_BLOCK_WIDE>{})
                                         : split(std::integral_constant<int, SPLIT_BLOCK>{});
  if (st != HG_OK) return st;
  launch_scan(fcount, g.n_fine, fstatus, ticket + 2, nullptr, fcount + g.n_fine, nullptr, s,
              who[0] == 'b' ? "fine_scan" : "probe_fine_scan");
  return HG_OK;
}

template <typename KeyT, int V, bool WI>
static hg_status run_partitioned(const BuildPlan& p, const KeyT* keys, uint32_t* offsets, KeyT* keys_out,
                                 uint32_t* idx_out, char* ws, cudaStream_t s) {
  const BucketMap bm = p.bucket_map();
  const PartGeometry& g = p.g;
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + p.off_flags);
  // status words, tickets, flags, partition counts and their scan states
  HG_CUDA(cudaMemsetAsync(ws + p.off_status, 0, p.off_pkeys - p.off_status, s), "build: workspace memset");
  hg_status st = run_partition_passes<KeyT, V, WI>(g, p.n, keys, p.key_idx, bm, ws, p.off_flags, p.off_ticket,
                                                   p.off_pcount, p.off_pstatus, p.off_fcount, p.off_fstatus,
                                                   p.off_pkeys, p.off_pidx, p.off_fkeys, p.off_fidx, "build", s);
  if (st != HG_OK) return st;
  {
    hg_status lst = HG_OK;
    using Src = TableFine<KeyT>;
    const Src src{reinterpret_cast<const KeyT*>(ws + p.off_fkeys),
                  WI ? reinterpret_cast<const uint32_t*>(ws + p.off_fidx) : nullptr,
                  reinterpret_cast<const uint32_t*>(ws + p.off_fcount), g.n_fine, g.fine_cap, g.fine_log2, bm,
                  p.n_buckets, offsets, keys_out, idx_out};
    auto go = [&](auto kern, unsigned block) {
      const int bps = blocks_per_sm(kern, block, g.smem3);
      if (bps <= 0) {
        lst = lib_fail(HG_ERR_CUDA, "fine-build kernel cannot be resident");
        return;
      }
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(g.n_fine, uint64_t(device_sm_count()) * bps));
      Phase ph(s, "fine_build");
      count_launch();
      kern<<<std::max(grid, 1u), block, g.smem3, s>>>(src, g.fine_cap, g.fine_log2, flags);
    };
    // tuning override: HG_BUILD_BLOCK=1024 or 256 runs the fine build with that many threads per CTA
    const char* bb = std::getenv("HG_BUILD_BLOCK");
    if (bb && std::atoi(bb) == 1024) go(k_fine_build<KeyT, WI, 1024, Src>, 1024u);
    else if (bb && std::atoi(bb) == 256) go(k_fine_build<KeyT, WI, 256, Src>, 256u);
    else go(k_fine_build<KeyT, WI, FINE_BLOCK, Src>, unsigned(FINE_BLOCK));
    if (lst != HG_OK) return lst;
    HG_CUDA(cudaPeekAtLastError(), "fine-build launch");
  }
  // Fallback for an overflowed partition (heavy duplicates), gated on the
  // flag: the keys are first grouped by coarse partition into exactly sized
  // runs of the partition buffer (a histogram, its scan, pass 1 with exact
  // starts), then the direct build runs over the grouped keys, so that its
  // counter and cursor atomics and its key writes stay within the buckets of
  // the few partitions in flight, which sit in L2.
  if (p.n == 0) return run_direct<KeyT, V, WI>(p, keys, offsets, keys_out, idx_out, ws, flags, s, p.key_idx);
  uint32_t* gcount = reinterpret_cast<uint32_t*>(ws + p.off_gcount);
  uint64_t* gstatus = reinterpret_cast<uint64_t*>(ws + p.off_gstatus);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  KeyT* gkeys = reinterpret_cast<KeyT*>(ws + p.off_pkeys);
  uint32_t* gidx = WI ? reinterpret_cast<uint32_t*>(ws + p.off_pidx) : nullptr;
  {
    Phase ph(s, "fallback_group_count");
    count_launch();
    const unsigned hgrid = static_cast<unsigned>(std::max<uint64_t>(
        1, std::min<uint64_t>((p.n + PART_HIST_BLOCK - 1) / PART_HIST_BLOCK, uint64_t(device_sm_count()) * 4)));
    k_part_hist<KeyT><<<hgrid, PART_HIST_BLOCK, 0, s>>>(keys, p.n, bm, g.coarse_log2, static_cast<uint32_t>(g.n_parts),
                                                         gcount, flags);
  }
  launch_scan(gcount, g.n_parts, gstatus, ticket + 4, nullptr, gcount + g.n_parts, flags, s, "fallback_group_scan");
  {
    Phase ph(s, "fallback_group");
    constexpr int BLK = pass1_block(sizeof(KeyT)), TILE = pass1_tile(sizeof(KeyT));
    auto kern = k_multisplit<KeyT, WI, BLK, PASS1_KPT, (V > 1), TableTiles<KeyT, TILE>, true>;
    const int bps = blocks_per_sm(kern, BLK, g.smem1);
    if (bps <= 0) return lib_fail(HG_ERR_CUDA, "multisplit kernel cannot be resident");
    const uint64_t ntiles = (p.n + TILE - 1) / TILE;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(ntiles, uint64_t(device_sm_count()) * bps));
    using Src = TableTiles<KeyT, TILE>;
    const Src src{keys, p.key_idx, p.n, bm, g.coarse_log2, static_cast<uint32_t>(g.n_parts), 0, gcount, gkeys, gidx};
    count_launch();
    kern<<<grid, BLK, g.smem1, s>>>(src, static_cast<uint32_t>(g.n_parts), flags);
    HG_CUDA(cudaPeekAtLastError(), "grouping multisplit launch");
  }
  return run_direct<KeyT, 16 / sizeof(KeyT), WI>(p, gkeys, offsets, keys_out, idx_out, ws, flags, s, gidx);
}

template <typename KeyT, bool WI>
static hg_status dispatch(const BuildPlan& p, const void* keys, uint32_t* offsets, void* keys_out, uint32_t* idx_out,
                          char* ws, cudaStream_t s) {
  const KeyT* k = static_cast<const KeyT*>(keys);
  KeyT* ko = static_cast<KeyT*>(keys_out);
  constexpr int V = 16 / sizeof(KeyT);
  const bool aligned = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0;
  if (p.path == BUILD_PARTITIONED) {
    return aligned ? run_partitioned<KeyT, V, WI>(p, k, offsets, ko, idx_out, ws, s)
                   : run_partitioned<KeyT, 1, WI>(p, k, offsets, ko, idx_out, ws, s);
  }
  return aligned ? run_direct<KeyT, V, WI>(p, k, offsets, ko, idx_out, ws, nullptr, s, p.key_idx)
                 : run_direct<KeyT, 1, WI>(p, k, offsets, ko, idx_out, ws, nullptr, s, p.key_idx);
}

hg_status launch_build(const BuildPlan& p, const void* d_keys, uint32_t* d_offsets, void* d_keys_out,
                       uint32_t* d_idx_out, void* d_ws, cudaStream_t s) {
  char* ws = static_cast<char*>(d_ws);
  hg_status st;
  if (p.key_bytes == 4)
    st = p.with_index ? dispatch<uint32_t, true>(p, d_keys, d_offsets, d_keys_out, d_idx_out, ws, s)
                      : dispatch<uint32_t, false>(p, d_keys, d_offsets, d_keys_out, d_idx_out, ws, s);
  else
    st = p.with_index ? dispatch<uint64_t, true>(p, d_keys, d_offsets, d_keys_out, d_idx_out, ws, s)
                      : dispatch<uint64_t, false>(p, d_keys, d_offsets, d_keys_out, d_idx_out, ws, s);
  if (st != HG_OK) return st;
  HG_CUDA(cudaPeekAtLastError(), "build: kernel launch");
  return HG_OK;
}

}  // namespace hg
