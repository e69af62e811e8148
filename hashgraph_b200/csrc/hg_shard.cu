// hg_shard.cu -- one table sharded over several devices by bucket range: the
// B200 form of MultiHashGraph with gpuCount > 1 (build
// src/MultiHashGraph.cu:408-629, intersect :631-740).
//
// The reference hashes every key into a materialised hash array
// (basicHashD), histograms the bucket ids into binCount bins (countBinSizes,
// include/MultiHashGraphDeviceOperators.cuh:153-163), sums the histograms on
// the host and picks per-GPU bucket ranges holding about n/G keys each
// (include/MultiHashGraphHostOperators.cuh:29-100), counts and buffers the
// keys bound for each GPU (countKeyBuffSizes :220-246, binKeyValues),
// copies the buffers between GPUs, subtracts the range start from every hash
// (decrHash :371-380) and builds each GPU's table over its range.
//
// Here one process drives one device and the exchange is the caller's
// collective (NCCL all-to-all over NVLink):
//   hg_shard_histogram   one kernel: bucket -> bin, shared-memory histogram,
//                        one 64-bit atomic per (CTA, non-empty bin).
//   hg_shard_splits      host: the reference's split rule, exact integers.
//   hg_shard_route       k_route_count, the look-back scan, k_route_scatter:
//                        keys grouped by destination shard, in input order
//                        inside each group, each with its global index
//                        (index_base + position) -- deterministic.
//   hg_shard_build_into  the ordinary build under the range's bucket map
//                        (no hash array, no decrHash pass), storing the
//                        carried global indices as the table's index.
//   hg_shard_intersect_into  the ordinary probe under the range's bucket map.
#include <algorithm>
#include <vector>

#include "hg_device.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"

namespace hg {

constexpr int SHARD_MAX = HG_MAX_SHARDS;
constexpr uint32_t SHARD_MAX_BINS = 32768;
constexpr int ROUTE_BLOCK = 256;
constexpr int ROUTE_WARPS = ROUTE_BLOCK / 32;
constexpr int ROUTE_V = 16;  // keys per lane: a tile is 4096 keys
constexpr uint64_t ROUTE_TILE = uint64_t(ROUTE_BLOCK) * ROUTE_V;

struct ShardSplits {
  uint64_t s[SHARD_MAX + 1];
};

// The shard whose range [s[r], s[r+1]) holds bucket b (s[0] = 0, s[G] = B,
// non-decreasing: an empty range is never chosen).
__device__ __forceinline__ int shard_of(uint32_t b, const uint64_t* s, int G) {
  int lo = 0, hi = G;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (uint64_t(b) >= s[mid]) lo = mid; else hi = mid;
  }
  return lo;
}

// Bin of a bucket: bucket / width with c = ceil(2^64 / width), exact for
// 32-bit buckets and widths (Lemire, Kaser & Kurz, "Faster remainder by
// direct computation", 2019: 64 fraction bits cover 32-bit operands);
// width 1 (c would not fit) is the bucket itself.
__device__ __forceinline__ uint32_t bin_of(uint32_t bucket, uint64_t c) {
  return c ? static_cast<uint32_t>(__umul64hi(c, bucket)) : bucket;
}

constexpr int HIST_BLOCK = 256, HIST_V = 8;

template <typename KeyT>
__global__ void __launch_bounds__(HIST_BLOCK) k_shard_hist(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm,
                                                           uint64_t bin_magic, uint32_t n_bins,
                                                           unsigned long long* __restrict__ bins) {
  if (entry_skip(nullptr)) return;
  extern __shared__ uint32_t s_bin[];
  for (uint32_t i = threadIdx.x; i < n_bins; i += HIST_BLOCK) s_bin[i] = 0;
  __syncthreads();
  // HIST_V keys per thread per round, each load coalesced across the block
  constexpr uint64_t CH = uint64_t(HIST_BLOCK) * HIST_V;
  for (uint64_t base = uint64_t(blockIdx.x) * CH; base < n; base += uint64_t(gridDim.x) * CH) {
    KeyT k[HIST_V];
#pragma unroll
    for (int j = 0; j < HIST_V; j++) {
      const uint64_t i = base + uint64_t(j) * HIST_BLOCK + threadIdx.x;
      k[j] = i < n ? __ldcs(keys + i) : KeyT(0);
    }
#pragma unroll
    for (int j = 0; j < HIST_V; j++)
      if (base + uint64_t(j) * HIST_BLOCK + threadIdx.x < n) atomicAdd(&s_bin[bin_of(bm.of_key(k[j]), bin_magic)], 1u);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n_bins; i += HIST_BLOCK)
    if (s_bin[i]) atomicAdd(bins + i, static_cast<unsigned long long>(s_bin[i]));
}

// Loads the tile's keys a warp owns: lane l holds keys base + j*32 + l, so
// walking j with the lanes in order visits the keys in input order.
template <typename KeyT>
__device__ __forceinline__ void route_load(const KeyT* __restrict__ keys, uint64_t n, uint64_t base, const BucketMap& bm,
                                           const uint64_t* s, int G, KeyT (&k)[ROUTE_V], int (&d)[ROUTE_V]) {
#pragma unroll
  for (int j = 0; j < ROUTE_V; j++) {
    const uint64_t i = base + uint64_t(j) * 32 + lane_id();
    const bool ok = i < n;
    k[j] = ok ? __ldcs(keys + i) : KeyT(0);
    d[j] = ok ? shard_of(bm.of_key(k[j]), s, G) : SHARD_MAX;  // SHARD_MAX: no key
  }
}

// Per-warp key counts of each destination shard, into s_wc[warp][shard].
template <typename KeyT>
__device__ __forceinline__ void route_count_warp(const int (&d)[ROUTE_V], uint32_t* s_wc_row) {
#pragma unroll
  for (int j = 0; j < ROUTE_V; j++) {
    const unsigned peers = __match_any_sync(FULL_MASK, d[j]);
    if (d[j] < SHARD_MAX && lane_id() == unsigned(__ffs(peers) - 1)) s_wc_row[d[j]] += __popc(peers);
    __syncwarp();
  }
}

// tile_counts[r * tiles + t] = keys of tile t bound for shard r.
template <typename KeyT>
__global__ void __launch_bounds__(ROUTE_BLOCK, 4) k_route_count(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm,
                                                             ShardSplits splits, int G,
                                                             uint32_t* __restrict__ tile_counts, uint64_t tiles) {
  if (entry_skip(nullptr)) return;
  __shared__ uint64_t s_split[SHARD_MAX + 1];
  __shared__ uint32_t s_wc[ROUTE_WARPS][SHARD_MAX];
  for (int i = threadIdx.x; i <= G; i += ROUTE_BLOCK) s_split[i] = splits.s[i];
  for (int i = threadIdx.x; i < ROUTE_WARPS * SHARD_MAX; i += ROUTE_BLOCK) (&s_wc[0][0])[i] = 0;
  __syncthreads();
  const uint64_t tile = blockIdx.x;
  const int w = threadIdx.x >> 5;
  KeyT k[ROUTE_V];
  int d[ROUTE_V];
  route_load<KeyT>(keys, n, tile * ROUTE_TILE + uint64_t(w) * 32 * ROUTE_V, bm, s_split, G, k, d);
  route_count_warp<KeyT>(d, s_wc[w]);
  __syncthreads();
  for (int r = threadIdx.x; r < G; r += ROUTE_BLOCK) {
    uint32_t c = 0;
#pragma unroll
    for (int x = 0; x < ROUTE_WARPS; x++) c += s_wc[x][r];
    tile_counts[uint64_t(r) * tiles + tile] = c;
  }
}

// After the exclusive scan of tile_counts (shard-major), every (shard, tile)
// knows where its keys start; each warp adds the counts of the warps before
// it and writes its keys in order.
template <typename KeyT, bool WITH_IDX>
__global__ void __launch_bounds__(ROUTE_BLOCK, 4) k_route_scatter(const KeyT* __restrict__ keys, uint64_t n, BucketMap bm,
                                                               ShardSplits splits, int G,
                                                               const uint32_t* __restrict__ tile_start, uint64_t tiles,
                                                               KeyT* __restrict__ keys_out,
                                                               uint32_t* __restrict__ idx_out, uint32_t index_base) {
  if (entry_skip(nullptr)) return;
  __shared__ uint64_t s_split[SHARD_MAX + 1];
  __shared__ uint32_t s_wc[ROUTE_WARPS][SHARD_MAX];
  for (int i = threadIdx.x; i <= G; i += ROUTE_BLOCK) s_split[i] = splits.s[i];
  for (int i = threadIdx.x; i < ROUTE_WARPS * SHARD_MAX; i += ROUTE_BLOCK) (&s_wc[0][0])[i] = 0;
  __syncthreads();
  const uint64_t tile = blockIdx.x;
  const int w = threadIdx.x >> 5;
  const uint64_t base = tile * ROUTE_TILE + uint64_t(w) * 32 * ROUTE_V;
  KeyT k[ROUTE_V];
  int d[ROUTE_V];
  route_load<KeyT>(keys, n, base, bm, s_split, G, k, d);
  route_count_warp<KeyT>(d, s_wc[w]);
  __syncthreads();
  // counts -> start positions, per shard down the warps
  for (int r = threadIdx.x; r < G; r += ROUTE_BLOCK) {
    uint32_t at = tile_start[uint64_t(r) * tiles + tile];
#pragma unroll
    for (int x = 0; x < ROUTE_WARPS; x++) {
      const uint32_t c = s_wc[x][r];
      s_wc[x][r] = at;
      at += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < ROUTE_V; j++) {
    const unsigned peers = __match_any_sync(FULL_MASK, d[j]);
    if (d[j] < SHARD_MAX) {
      const uint32_t at = s_wc[w][d[j]];
      const uint32_t pos = at + __popc(peers & lanemask_lt());
      if (pos < n) {
        keys_out[pos] = k[j];
        if constexpr (WITH_IDX) idx_out[pos] = index_base + static_cast<uint32_t>(base + uint64_t(j) * 32 + lane_id());
      } else {
        record_fault(HG_ERR_DEVICE_STATE);  // tile starts past n: write nothing
      }
      __syncwarp(peers);
      if (lane_id() == unsigned(__ffs(peers) - 1)) s_wc[w][d[j]] = at + __popc(peers);
    }
    __syncwarp();
  }
}

// offsets[r] = first routed key of shard r (offsets[G] = n).
__global__ void k_route_offsets(const uint32_t* __restrict__ tile_start, uint64_t tiles, int G, uint64_t n,
                                unsigned long long* __restrict__ offsets) {
  if (entry_skip(nullptr)) return;
  const int r = threadIdx.x;
  if (r < G) offsets[r] = tiles ? tile_start[uint64_t(r) * tiles] : 0ull;
  if (r == G) offsets[r] = n;
}

static int max_dyn_smem_set(const void* kern, size_t bytes) {
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)) ==
         cudaSuccess;
}

struct RouteWs {
  uint64_t tiles = 0, counts = 0, scan_tiles = 0;
  size_t off_counts = 0, off_status = 0, off_ticket = 0, total = 0;
};

static RouteWs route_ws(uint64_t n, int G) {
  RouteWs w;
  w.tiles = (n + ROUTE_TILE - 1) / ROUTE_TILE;
  w.counts = w.tiles * uint64_t(G);
  w.scan_tiles = (w.counts + SCAN_TILE - 1) / SCAN_TILE;
  w.off_counts = 0;
  w.off_status = align_up(w.off_counts + w.counts * 4);
  w.off_ticket = align_up(w.off_status + w.scan_tiles * 8);
  w.total = align_up(w.off_ticket + 16);
  return w;
}

// Checks a shard range [lo, hi) of a table of `total` buckets: the bucket
// map of an unaligned range needs the remainder form, so total < 2^32.
static hg_status check_range(uint64_t total, uint64_t lo, uint64_t hi) {
  if (total == 0 || lo >= hi || hi > total) return lib_fail(HG_ERR_INVALID_ARGUMENT, "shard: need lo < hi <= n_buckets");
  if (total > (1ull << 32)) return HG_ERR_TOO_LARGE;
  const uint64_t local = hi - lo;
  const bool aligned_p2 = (total & (total - 1)) == 0 && (local & (local - 1)) == 0 && lo % local == 0;
  if (total == (1ull << 32) && !aligned_p2 && !(lo == 0 && hi == total))
    return lib_fail(HG_ERR_TOO_LARGE, "shard: a table of 2^32 buckets shards only into aligned power-of-two ranges");
  return HG_OK;
}

static hg_status check_splits(const uint64_t* splits, int G, uint64_t n_buckets) {
  if (!splits || G < 1 || G > SHARD_MAX) return HG_ERR_INVALID_ARGUMENT;
  if (splits[0] != 0 || splits[G] != n_buckets)
    return lib_fail(HG_ERR_INVALID_ARGUMENT, "shard: splits must start at 0 and end at n_buckets");
  for (int r = 0; r < G; r++)
    if (splits[r] > splits[r + 1]) return lib_fail(HG_ERR_INVALID_ARGUMENT, "shard: splits must not decrease");
  return HG_OK;
}

}  // namespace hg

using namespace hg;

extern "C" hg_status hg_shard_histogram(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                                        uint32_t n_bins, unsigned long long* d_bins, hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0 || n_bins == 0 || !d_bins || (n > 0 && !d_keys)) return HG_ERR_INVALID_ARGUMENT;
  if (n_buckets > (1ull << 32) || n_bins > SHARD_MAX_BINS) return HG_ERR_TOO_LARGE;
  if (n == 0) return HG_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const BucketMap bm = BucketMap::make(n_buckets);
  const uint64_t width = (n_buckets + n_bins - 1) / n_bins;
  // ceil(2^64 / width) for width >= 2; 0 marks width 1
  const uint64_t magic = width == 1 ? 0ull : UINT64_MAX / width + 1;
  const size_t smem = size_t(n_bins) * 4;
  // two CTAs per SM: each CTA flushes up to n_bins 64-bit atomics at its end,
  // so fewer, longer-running CTAs keep that flush small (2^24 keys, 16000
  // bins: 6.9M L2 atomic sectors per launch with 8 CTAs per SM)
  const uint64_t chunks = (n + uint64_t(HIST_BLOCK) * HIST_V - 1) / (uint64_t(HIST_BLOCK) * HIST_V);
  const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(chunks, uint64_t(device_sm_count()) * 2)));
  Phase ph(s, "shard_histogram");
  count_launch();
  if (key_bytes == 8) {
    if (smem > 48 * 1024) max_dyn_smem_set(reinterpret_cast<const void*>(k_shard_hist<uint64_t>), smem);
    k_shard_hist<uint64_t><<<grid, HIST_BLOCK, smem, s>>>(static_cast<const uint64_t*>(d_keys), n, bm, magic, n_bins,
                                                         d_bins);
  } else {
    if (smem > 48 * 1024) max_dyn_smem_set(reinterpret_cast<const void*>(k_shard_hist<uint32_t>), smem);
    k_shard_hist<uint32_t><<<grid, HIST_BLOCK, smem, s>>>(static_cast<const uint32_t*>(d_keys), n, bm, magic, n_bins,
                                                         d_bins);
  }
  HG_CUDA(cudaPeekAtLastError(), "hg_shard_histogram");
  return HG_OK;
}

// The reference's rule (include/MultiHashGraphHostOperators.cuh:80-88):
// prefix sums ps[0..bins] of the bin counts; the upper split of shard r is
// the bin found by its binary search (:8-27, the exact-match-or-insertion
// index) for ceil(total/G) * (r+1), times the bin width, capped at B.  Kept
// alike so a sharded table's ranges are the reference's.  Two decisions of
// our own: integer arithmetic where the reference rounds through float, and
// the last split is always B (the reference can stop short of B when the top
// bins are empty, and a later table built on the same splits then has keys
// in no range).
extern "C" hg_status hg_shard_splits(const unsigned long long* h_bins, uint32_t n_bins, uint64_t n_buckets,
                                     int n_shards, uint64_t* h_splits) {
  if (!h_bins || !h_splits || n_bins == 0 || n_buckets == 0 || n_shards < 1 || n_shards > SHARD_MAX)
    return HG_ERR_INVALID_ARGUMENT;
  if (n_buckets > (1ull << 32) || n_bins > SHARD_MAX_BINS) return HG_ERR_TOO_LARGE;
  std::vector<uint64_t> ps(size_t(n_bins) + 1, 0);
  for (uint32_t i = 0; i < n_bins; i++) ps[i + 1] = ps[i] + h_bins[i];
  const uint64_t total = ps[n_bins];
  const uint64_t width = (n_buckets + n_bins - 1) / n_bins;
  const uint64_t avg = (total + uint64_t(n_shards) - 1) / uint64_t(n_shards);
  h_splits[0] = 0;
  for (int r = 0; r + 1 < n_shards; r++) {
    const uint64_t x = avg * uint64_t(r + 1);
    // binary search over ps[0..n_bins] (inclusive bounds, as the reference's)
    int64_t l = 0, h = n_bins;
    uint64_t found = 0;
    bool hit = false;
    while (h >= l) {
      const int64_t mid = l + (h - l) / 2;
      if (ps[mid] == x) { found = uint64_t(mid); hit = true; break; }
      if (ps[mid] > x) h = mid - 1; else l = mid + 1;
    }
    const uint64_t idx = hit ? found : uint64_t(l);
    h_splits[r + 1] = std::max<uint64_t>(h_splits[r], std::min<uint64_t>(idx * width, n_buckets));
  }
  h_splits[n_shards] = n_buckets;
  return HG_OK;
}

extern "C" hg_status hg_shard_route_workspace_size(uint64_t n, int n_shards, size_t* bytes) {
  if (!bytes || n_shards < 1 || n_shards > SHARD_MAX) return HG_ERR_INVALID_ARGUMENT;
  if (n >= (1ull << 32)) return HG_ERR_TOO_LARGE;
  *bytes = route_ws(n, n_shards).total;
  return HG_OK;
}

extern "C" hg_status hg_shard_route(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                                    const uint64_t* splits, int n_shards, uint32_t index_base, void* d_keys_out,
                                    uint32_t* d_idx_out, unsigned long long* d_shard_offsets, void* d_workspace,
                                    size_t workspace_bytes, hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0 || !d_shard_offsets || (n > 0 && (!d_keys || !d_keys_out))) return HG_ERR_INVALID_ARGUMENT;
  if (n >= (1ull << 32) || n_buckets > (1ull << 32)) return HG_ERR_TOO_LARGE;
  if (d_idx_out && uint64_t(index_base) + n > (1ull << 32))
    return lib_fail(HG_ERR_TOO_LARGE, "hg_shard_route: global indices must stay below 2^32");
  hg_status st = check_splits(splits, n_shards, n_buckets);
  if (st != HG_OK) return st;
  const RouteWs w = route_ws(n, n_shards);
  if (!d_workspace || workspace_bytes < w.total) return HG_ERR_TOO_LARGE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(d_workspace);
  uint32_t* counts = reinterpret_cast<uint32_t*>(ws + w.off_counts);
  ShardSplits sp = {};
  for (int r = 0; r <= n_shards; r++) sp.s[r] = splits[r];
  const BucketMap bm = BucketMap::make(n_buckets);
  if (w.tiles) {
    HG_CUDA(cudaMemsetAsync(ws + w.off_status, 0, w.total - w.off_status, s), "hg_shard_route: memset");
    {
      Phase ph(s, "shard_route_count");
      count_launch();
      if (key_bytes == 8)
        k_route_count<uint64_t><<<static_cast<unsigned>(w.tiles), ROUTE_BLOCK, 0, s>>>(
            static_cast<const uint64_t*>(d_keys), n, bm, sp, n_shards, counts, w.tiles);
      else
        k_route_count<uint32_t><<<static_cast<unsigned>(w.tiles), ROUTE_BLOCK, 0, s>>>(
            static_cast<const uint32_t*>(d_keys), n, bm, sp, n_shards, counts, w.tiles);
      HG_CUDA(cudaPeekAtLastError(), "hg_shard_route: count");
    }
    launch_scan(counts, w.counts, reinterpret_cast<uint64_t*>(ws + w.off_status),
                reinterpret_cast<unsigned*>(ws + w.off_ticket), nullptr, nullptr, nullptr, s, "shard_route_scan");
    Phase ph(s, "shard_route_scatter");
    count_launch();
#define HG_ROUTE(KT, WI)                                                                                         \
  k_route_scatter<KT, WI><<<static_cast<unsigned>(w.tiles), ROUTE_BLOCK, 0, s>>>(                                \
      static_cast<const KT*>(d_keys), n, bm, sp, n_shards, counts, w.tiles, static_cast<KT*>(d_keys_out), d_idx_out, \
      index_base)
    if (key_bytes == 8) {
      if (d_idx_out) HG_ROUTE(uint64_t, true); else HG_ROUTE(uint64_t, false);
    } else {
      if (d_idx_out) HG_ROUTE(uint32_t, true); else HG_ROUTE(uint32_t, false);
    }
#undef HG_ROUTE
    HG_CUDA(cudaPeekAtLastError(), "hg_shard_route: scatter");
  }
  count_launch();
  k_route_offsets<<<1, SHARD_MAX + 1, 0, s>>>(counts, w.tiles, n_shards, n, d_shard_offsets);
  HG_CUDA(cudaPeekAtLastError(), "hg_shard_route: offsets");
  return HG_OK;
}

extern "C" hg_status hg_shard_build_into_path(const void* d_keys, const uint32_t* d_key_idx, uint64_t n, int key_bytes,
                                              uint64_t n_buckets, uint64_t bucket_lo, uint64_t bucket_hi,
                                              uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                                              void* d_workspace, size_t workspace_bytes, int path,
                                              hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  hg_status st = check_range(n_buckets, bucket_lo, bucket_hi);
  if (st != HG_OK) return st;
  if (n >= (1ull << 32)) return HG_ERR_TOO_LARGE;
  if (!d_offsets || (n > 0 && (!d_keys || !d_keys_out)) || !d_workspace) return HG_ERR_INVALID_ARGUMENT;
  BuildPlan plan;
  st = plan_build(n, key_bytes, bucket_hi - bucket_lo, d_idx_out != nullptr, &plan, path);
  if (st != HG_OK) return st;
  if (workspace_bytes < plan.total) return HG_ERR_TOO_LARGE;
  plan.range_total = n_buckets;
  plan.range_lo = bucket_lo;
  plan.key_idx = d_key_idx;  // the partition passes (or the direct scatter) store the carried indices
  return launch_build(plan, d_keys, d_offsets, d_keys_out, d_idx_out, d_workspace,
                      reinterpret_cast<cudaStream_t>(stream));
}

extern "C" hg_status hg_shard_build_into(const void* d_keys, const uint32_t* d_key_idx, uint64_t n, int key_bytes,
                                         uint64_t n_buckets, uint64_t bucket_lo, uint64_t bucket_hi,
                                         uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                                         void* d_workspace, size_t workspace_bytes, hg_stream_t stream) {
  return hg_shard_build_into_path(d_keys, d_key_idx, n, key_bytes, n_buckets, bucket_lo, bucket_hi, d_offsets,
                                  d_keys_out, d_idx_out, d_workspace, workspace_bytes, -1, stream);
}

extern "C" hg_status hg_shard_intersect_into_path(const uint32_t* d_a_offsets, const void* d_a_keys,
                                                  const uint32_t* d_a_idx, uint64_t n_a, uint64_t n_buckets,
                                                  uint64_t bucket_lo, uint64_t bucket_hi, int key_bytes,
                                                  const void* d_query, uint64_t nq, const uint32_t* d_query_idx,
                                                  uint32_t* d_pairs, uint64_t pair_cap, unsigned long long* d_count,
                                                  void* d_workspace, size_t workspace_bytes, int path,
                                                  hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  hg_status st = check_range(n_buckets, bucket_lo, bucket_hi);
  if (st != HG_OK) return st;
  if (!d_a_offsets || !d_count || (nq > 0 && !d_query) || (n_a > 0 && !d_a_keys)) return HG_ERR_INVALID_ARGUMENT;
  ProbePlan plan;
  st = plan_probe(n_a, d_a_idx != nullptr, bucket_hi - bucket_lo, nq, key_bytes, d_pairs != nullptr, &plan, path);
  if (st != HG_OK) return st;
  if (workspace_bytes < plan.total || (!d_workspace && plan.total)) return HG_ERR_TOO_LARGE;
  plan.range_total = n_buckets;
  plan.range_lo = bucket_lo;
  return launch_probe(plan, d_a_offsets, d_a_keys, d_a_idx, d_query, d_query_idx, d_pairs, pair_cap, d_count,
                      d_workspace, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" hg_status hg_shard_intersect_into(const uint32_t* d_a_offsets, const void* d_a_keys, const uint32_t* d_a_idx,
                                             uint64_t n_a, uint64_t n_buckets, uint64_t bucket_lo, uint64_t bucket_hi,
                                             int key_bytes, const void* d_query, uint64_t nq,
                                             const uint32_t* d_query_idx, uint32_t* d_pairs, uint64_t pair_cap,
                                             unsigned long long* d_count, void* d_workspace, size_t workspace_bytes,
                                             hg_stream_t stream) {
  return hg_shard_intersect_into_path(d_a_offsets, d_a_keys, d_a_idx, n_a, n_buckets, bucket_lo, bucket_hi, key_bytes,
                                      d_query, nq, d_query_idx, d_pairs, pair_cap, d_count, d_workspace,
                                      workspace_bytes, -1, stream);
}
