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
//   1. k_part_scatter: hash each key, bucket range p = b >> part_log2, append
//                 (key, position) to partition p's slot range (warp-aggregated
//                 slot reservation; the open tail line of every partition stays
//                 in L2 so the scattered appends reach HBM as whole lines).
//   2. k_scan_u32 over the P partition sizes -> partition starts.
//   3. k_part_local: one CTA per partition: shared-memory bucket histogram,
//                 segmented block scan, coalesced offsets write, then the
//                 scatter of the partition's keys into its output slice.
//   If any partition overflowed its slot range (heavy duplicates), pass 3
//   stands down and gated copies of the direct kernels rebuild the table;
//   the decision is taken on the device, so the launch sequence is fixed.
#include <algorithm>
#include <cmath>

#include "hg_device.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"
#include "hg_scan.cuh"

namespace hg {

constexpr uint32_t FLAG_OVERFLOW = 1u;

// Gate: kernels handed a non-null gate run only when the overflow flag is set.
__device__ __forceinline__ bool gated_off(const uint32_t* gate) {
  return gate != nullptr && (*reinterpret_cast<const volatile uint32_t*>(gate) & FLAG_OVERFLOW) == 0;
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
  if (gated_off(gate)) return;
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
                                                 uint32_t* __restrict__ idx_out, const uint32_t* gate) {
  if (gated_off(gate)) return;
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
      if (ok[j]) {
        keys_out[pos] = k[j];
        if constexpr (WITH_IDX) idx_out[pos] = static_cast<uint32_t>(base + lane_id() * V + j);
      }
    }
  }
}

// In-place exclusive scan of data[0..count) (uint32 values, total < 2^32).
// first_slot (optional) receives 0; total_out (optional) receives the sum.
template <int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK) k_scan_u32(uint32_t* __restrict__ data, uint64_t count,
                                                    uint64_t* __restrict__ status, unsigned* ticket,
                                                    uint32_t* first_slot, uint32_t* total_out,
                                                    const uint32_t* gate) {
  if (gated_off(gate)) return;
  constexpr int TILE = BLOCK * ITEMS;
  __shared__ uint32_t s[TILE + TILE / 32];
  __shared__ uint32_t red[BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t base = tile * TILE;
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
  const uint64_t ntiles = (count + TILE - 1) / TILE;
  if (threadIdx.x == 0) {
    if (tile == 0 && first_slot) *first_slot = 0u;
    if (tile == ntiles - 1 && total_out) *total_out = static_cast<uint32_t>(s_prefix) + tile_total;
  }
}

__global__ void k_fill_u32(uint32_t* p, uint64_t count, uint32_t value, const uint32_t* gate) {
  if (gated_off(gate)) return;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    p[i] = value;
}

// ---------------------------------------------------------------------------
// Partitioned path
// ---------------------------------------------------------------------------
template <typename KeyT, int V, bool WITH_IDX>
__global__ void __launch_bounds__(256) k_part_scatter(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm,
                                                      uint32_t part_log2, uint64_t cap,
                                                      uint32_t* __restrict__ pcount, KeyT* __restrict__ pkeys,
                                                      uint32_t* __restrict__ pidx, uint32_t* flags) {
  const uint64_t warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  const uint64_t nchunks = (n + 32ull * V - 1) / (32ull * V);
  bool overflow = false;
  for (uint64_t c = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; c < nchunks;
       c += warps) {
    KeyT k[V];
    bool ok[V];
    const uint64_t base = c * 32ull * V;
    load_chunk<KeyT, V>(keys, n, base, k, ok);
#pragma unroll
    for (int j = 0; j < V; j++) {
      const uint32_t p = bm.of_key(k[j]) >> part_log2;
      const uint32_t slot = warp_aggregated_inc(pcount, p, ok[j]);
      if (ok[j]) {
        if (slot < cap) {
          const uint64_t at = static_cast<uint64_t>(p) * cap + slot;
          pkeys[at] = k[j];
          if constexpr (WITH_IDX) pidx[at] = static_cast<uint32_t>(base + lane_id() * V + j);
        } else {
          overflow = true;
        }
      }
    }
  }
  if (overflow) atomicOr(flags, FLAG_OVERFLOW);
}

// One CTA per partition (grid-stride over partitions).  Dynamic shared memory:
// 2^part_log2 uint32 counters.
template <typename KeyT, bool WITH_IDX, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_part_local(const KeyT* __restrict__ pkeys, const uint32_t* __restrict__ pidx,
                                                      const uint32_t* __restrict__ pstart, uint64_t n_parts,
                                                      uint64_t cap, uint32_t part_log2, BucketMap bm,
                                                      uint64_t n_buckets, uint32_t* __restrict__ offsets,
                                                      KeyT* __restrict__ keys_out, uint32_t* __restrict__ idx_out,
                                                      const uint32_t* flags) {
  if (*reinterpret_cast<const volatile uint32_t*>(flags) & FLAG_OVERFLOW) return;
  extern __shared__ uint32_t ctr[];
  constexpr int NW = BLOCK / 32;
  __shared__ uint32_t wsum[NW + 1];
  const unsigned warp = threadIdx.x >> 5, lane = lane_id();
  if (blockIdx.x == 0 && threadIdx.x == 0) offsets[n_buckets] = pstart[n_parts];
  for (uint64_t p = blockIdx.x; p < n_parts; p += gridDim.x) {
    const uint32_t base = pstart[p];
    const uint32_t cnt = pstart[p + 1] - base;
    const uint64_t b0 = p << part_log2;
    const uint32_t nb = static_cast<uint32_t>(min(uint64_t(1) << part_log2, n_buckets - b0));
    const KeyT* src = pkeys + p * cap;
    const uint32_t* srci = pidx + p * cap;
    for (uint32_t j = threadIdx.x; j < nb; j += BLOCK) ctr[j] = 0;
    __syncthreads();
    for (uint32_t r0 = 0; r0 < cnt; r0 += BLOCK) {
      const uint32_t r = r0 + threadIdx.x;
      const bool ok = r < cnt;
      const KeyT k = ok ? src[r] : KeyT(0);
      const uint32_t lb = ok ? static_cast<uint32_t>(bm.of_key(k) - b0) : 0u;
      warp_aggregated_count(ctr, lb, ok);
    }
    __syncthreads();
    // Segmented scan: warp w owns counters [w*seg, (w+1)*seg).
    const uint32_t seg = ((nb + NW - 1) / NW + 31) & ~31u;
    const uint32_t s0 = min(nb, warp * seg), s1 = min(nb, s0 + seg);
    uint32_t part = 0;
    for (uint32_t j = s0 + lane; j < s1; j += 32) part += ctr[j];
    part = warp_sum(part);
    if (lane == 0) wsum[warp] = part;
    __syncthreads();
    if (warp == 0) {
      const uint32_t w = lane < NW ? wsum[lane] : 0u;
      const uint32_t wi = warp_inclusive_scan(w);
      if (lane < NW) wsum[lane] = wi - w;
    }
    __syncthreads();
    uint32_t run = base + wsum[warp];
    for (uint32_t j0 = s0; j0 < s1; j0 += 32) {
      const uint32_t j = j0 + lane;
      const uint32_t v = j < s1 ? ctr[j] : 0u;
      const uint32_t inc = warp_inclusive_scan(v);
      if (j < s1) {
        const uint32_t ex = run + inc - v;
        ctr[j] = ex;
        offsets[b0 + j] = ex;
      }
      run += __shfl_sync(FULL_MASK, inc, 31);
    }
    __syncthreads();
    for (uint32_t r0 = 0; r0 < cnt; r0 += BLOCK) {
      const uint32_t r = r0 + threadIdx.x;
      const bool ok = r < cnt;
      const KeyT k = ok ? src[r] : KeyT(0);
      const uint32_t lb = ok ? static_cast<uint32_t>(bm.of_key(k) - b0) : 0u;
      const uint32_t pos = warp_aggregated_inc(ctr, lb, ok);
      if (ok) {
        keys_out[pos] = k;
        if constexpr (WITH_IDX) idx_out[pos] = srci[r];
      }
    }
    __syncthreads();
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

constexpr int PART_LOCAL_BLOCK = 512;
constexpr uint32_t PART_LOG2_DEFAULT = 14;

hg_status plan_build(uint64_t n, int key_bytes, uint64_t n_buckets, bool with_index, BuildPlan* plan,
                     int force_path) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0) return HG_ERR_INVALID_ARGUMENT;
  if (n >= (1ull << 32) || n_buckets > (1ull << 32)) return HG_ERR_TOO_LARGE;
  BuildPlan p;
  p.n = n;
  p.n_buckets = n_buckets;
  p.key_bytes = key_bytes;
  p.with_index = with_index;
  const uint64_t rec = key_bytes + (with_index ? 4 : 0);
  const uint64_t footprint = n * (key_bytes + rec) + 4 * n_buckets;
  int path = force_path;
  if (path < 0) path = (footprint <= (48ull << 20) || n_buckets <= (1ull << PART_LOG2_DEFAULT)) ? BUILD_DIRECT : BUILD_PARTITIONED;
  p.path = path;
  size_t off = 0;
  p.scan_tiles = (n_buckets + SCAN_TILE - 1) / SCAN_TILE;
  p.off_status = off;  off = align_up(off + p.scan_tiles * 8);
  p.off_ticket = off;  off = align_up(off + 2 * sizeof(unsigned));
  p.off_flags = off;   off = align_up(off + sizeof(uint32_t));
  if (path == BUILD_PARTITIONED) {
    p.part_log2 = PART_LOG2_DEFAULT;
    p.n_parts = (n_buckets + (1ull << p.part_log2) - 1) >> p.part_log2;
    const double mean = double(n) * double(1ull << p.part_log2) / double(n_buckets);
    uint64_t cap = static_cast<uint64_t>(std::ceil(mean + 8.0 * std::sqrt(mean) + 64.0));
    cap = (cap + 31) & ~31ull;
    p.part_cap = cap;
    p.pscan_tiles = (p.n_parts + SCAN_TILE - 1) / SCAN_TILE;
    // the partition scan gets its own status region after the bucket-scan one
    p.off_pcount = off;  off = align_up(off + (p.n_parts + 1) * 4 + p.pscan_tiles * 8 + 8);
    p.off_pkeys = off;   off = align_up(off + p.n_parts * cap * key_bytes);
    if (with_index) { p.off_pidx = off; off = align_up(off + p.n_parts * cap * 4); }
  }
  p.total = std::max<size_t>(off, WS_ALIGN);
  *plan = p;
  return HG_OK;
}

template <typename KeyT, int V>
static void launch_direct_count(const KeyT* keys, uint64_t n, BucketMap bm, uint32_t* cnt, const uint32_t* gate,
                                cudaStream_t s) {
  const uint64_t chunks = (n + 32ull * V - 1) / (32ull * V);
  const uint64_t want = (chunks + 7) / 8;
  const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(device_sm_count()) * 8)));
  Phase ph(s, gate ? "fallback_count" : "count");
  count_launch();
  k_count<KeyT, V><<<grid, 256, 0, s>>>(keys, n, bm, cnt, gate);
}

template <typename KeyT, int V, bool WI>
static void launch_direct_scatter(const KeyT* keys, uint64_t n, BucketMap bm, uint32_t* cursor, KeyT* out,
                                  uint32_t* idx, const uint32_t* gate, cudaStream_t s) {
  const uint64_t chunks = (n + 32ull * V - 1) / (32ull * V);
  const uint64_t want = (chunks + 7) / 8;
  const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(device_sm_count()) * 8)));
  Phase ph(s, gate ? "fallback_scatter" : "scatter");
  count_launch();
  k_scatter<KeyT, V, WI><<<grid, 256, 0, s>>>(keys, n, bm, cursor, out, idx, gate);
}

static void launch_scan(uint32_t* data, uint64_t count, uint64_t* status, unsigned* ticket, uint32_t* first_slot,
                        uint32_t* total_out, const uint32_t* gate, cudaStream_t s) {
  const uint64_t tiles = (count + SCAN_TILE - 1) / SCAN_TILE;
  if (tiles == 0) return;
  Phase ph(s, gate ? "fallback_scan" : "scan");
  count_launch();
  k_scan_u32<SCAN_BLOCK, SCAN_ITEMS><<<static_cast<unsigned>(tiles), SCAN_BLOCK, 0, s>>>(data, count, status, ticket,
                                                                                      first_slot, total_out, gate);
}

template <typename KeyT, int V, bool WI>
static hg_status run_direct(const BuildPlan& p, const KeyT* keys, uint32_t* offsets, KeyT* keys_out, uint32_t* idx_out,
                            char* ws, const uint32_t* gate, cudaStream_t s) {
  const BucketMap bm = BucketMap::make(p.n_buckets);
  uint64_t* status = reinterpret_cast<uint64_t*>(ws + p.off_status);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  if (gate) {
    const int grid = static_cast<int>(std::min<uint64_t>((p.n_buckets + 1 + 255) / 256, uint64_t(device_sm_count()) * 8));
    Phase ph(s, "fallback_fill");
    count_launch();
    k_fill_u32<<<std::max(grid, 1), 256, 0, s>>>(offsets, p.n_buckets + 1, 0u, gate);
  } else {
    if (cudaMemsetAsync(offsets, 0, (p.n_buckets + 1) * sizeof(uint32_t), s) != cudaSuccess) return HG_ERR_CUDA;
  }
  if (cudaMemsetAsync(ws + p.off_status, 0, p.off_flags - p.off_status, s) != cudaSuccess) return HG_ERR_CUDA;
  if (p.n > 0) launch_direct_count<KeyT, V>(keys, p.n, bm, offsets + 1, gate, s);
  launch_scan(offsets + 1, p.n_buckets, status, ticket, offsets, nullptr, gate, s);
  if (p.n > 0) launch_direct_scatter<KeyT, V, WI>(keys, p.n, bm, offsets + 1, keys_out, idx_out, gate, s);
  return HG_OK;
}

template <typename KeyT, int V, bool WI>
static hg_status run_partitioned(const BuildPlan& p, const KeyT* keys, uint32_t* offsets, KeyT* keys_out,
                                 uint32_t* idx_out, char* ws, cudaStream_t s) {
  const BucketMap bm = BucketMap::make(p.n_buckets);
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + p.off_flags);
  uint32_t* pcount = reinterpret_cast<uint32_t*>(ws + p.off_pcount);
  uint64_t* pstatus = reinterpret_cast<uint64_t*>(ws + p.off_pcount + align_up((p.n_parts + 1) * 4, 8));
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  KeyT* pkeys = reinterpret_cast<KeyT*>(ws + p.off_pkeys);
  uint32_t* pidx = WI ? reinterpret_cast<uint32_t*>(ws + p.off_pidx) : nullptr;
  // status words, tickets, flags, partition counts and their scan status
  if (cudaMemsetAsync(ws + p.off_status, 0, p.off_pkeys - p.off_status, s) != cudaSuccess) return HG_ERR_CUDA;
  if (p.n > 0) {
    const uint64_t chunks = (p.n + 32ull * V - 1) / (32ull * V);
    const uint64_t want = (chunks + 7) / 8;
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(want, uint64_t(device_sm_count()) * 8)));
    Phase ph(s, "part_scatter");
    count_launch();
    k_part_scatter<KeyT, V, WI><<<grid, 256, 0, s>>>(keys, p.n, bm, p.part_log2, p.part_cap, pcount, pkeys, pidx,
                                                     flags);
  }
  // partition starts: exclusive scan of pcount[0..P), total into pcount[P]
  launch_scan(pcount, p.n_parts, pstatus, ticket + 1, nullptr, pcount + p.n_parts, nullptr, s);
  {
    const size_t smem = (size_t(1) << p.part_log2) * sizeof(uint32_t);
    auto kern = k_part_local<KeyT, WI, PART_LOCAL_BLOCK>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess)
      return HG_ERR_CUDA;
    const int grid = static_cast<int>(std::min<uint64_t>(p.n_parts, uint64_t(device_sm_count()) * 4));
    Phase ph(s, "part_local");
    count_launch();
    kern<<<std::max(grid, 1), PART_LOCAL_BLOCK, smem, s>>>(pkeys, pidx, pcount, p.n_parts, p.part_cap, p.part_log2,
                                                            bm, p.n_buckets, offsets, keys_out, idx_out, flags);
  }
  // Fallback for overflowed partitions: the direct build, gated on the flag.
  return run_direct<KeyT, V, WI>(p, keys, offsets, keys_out, idx_out, ws, flags, s);
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
  return aligned ? run_direct<KeyT, V, WI>(p, k, offsets, ko, idx_out, ws, nullptr, s)
                 : run_direct<KeyT, 1, WI>(p, k, offsets, ko, idx_out, ws, nullptr, s);
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
  return cudaPeekAtLastError() == cudaSuccess ? HG_OK : HG_ERR_CUDA;
}

}  // namespace hg
