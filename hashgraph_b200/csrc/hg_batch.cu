// hg_batch.cu -- batched build + intersect of many independent (table,
// queries) pairs in one fixed launch sequence.
//
// A batch of thousands of small and medium pairs (2^6 .. 2^20 keys) is
// launch-bound when every pair takes its own build + intersect calls (about
// seven launches each).  Here every kernel of the direct path runs ONCE for the
// whole batch over a flattened list of tiles: tile t belongs to pair
// tile_pair[t] (a host-built map, one 4-byte load per tile).  Tiles are
// ordered by pair, so the CTAs in flight work on a few consecutive pairs at a
// time and each pair's table (at most a few MB) stays in L2 while it is
// counted, scattered and probed.
//
// Sequence (hg_batch_run): memset of the look-back state, then
//   k_batch_clear    zero every pair's offsets, zero every pair's count
//   k_batch_count    hash + warp-aggregated bucket counts into offsets[1..B]
//   k_batch_scan     per-pair exclusive scan of offsets[1..B] in place: one
//                    decoupled look-back chain per pair over the flattened
//                    scan tiles (ticket order across the whole batch)
//   k_batch_scatter  hash + warp-aggregated cursor bump on offsets[b+1]
//                    (each cursor ends at the start of bucket b+1), write
//                    key (+ input position)
//   k_batch_probe    per query tile: count, per-pair look-back for the output
//                    offset, pairs written in query order; the pair's last
//                    tile stores its exact count
// Each pair's result is the one the single-pair direct path
// (k_count / k_scan_u32 / k_scatter / k_probe) gives.  The reference has no
// batched form; per pair it replaces build + intersect of
// src/MultiHashGraph.cu:408-740.
#include <algorithm>
#include <vector>

#include "hg_device.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"
#include "hg_scan.cuh"

struct hg_batch;

namespace hg {

constexpr int BATCH_BLOCK = 256;
constexpr uint32_t BATCH_KPT = 8;                              // keys per thread per tile
constexpr uint32_t BATCH_KTILE = BATCH_BLOCK * BATCH_KPT;      // count / scatter tile
constexpr uint32_t BATCH_QPT = 4;                              // queries per thread per tile
constexpr uint32_t BATCH_QTILE = BATCH_BLOCK * BATCH_QPT;      // probe tile
constexpr uint32_t BATCH_STILE = SCAN_TILE;                    // scan tile (offsets entries)

struct BatchPairDev {
  const void* keys;
  const void* query;
  uint32_t* offsets;
  void* keys_out;
  uint32_t* idx_out;
  uint32_t* pairs;
  unsigned long long* count;
  uint64_t n, nq, n_buckets, pair_cap;
  BucketMap bm;
  uint64_t ktile0, stile0, qtile0;  // first flattened tile of each kind
  uint64_t qtiles;                  // query tiles of this pair
};

// Every pair's offsets to zero (tile lt of a pair clears entries
// [lt*STILE, ...) of offsets[1..B]; tile 0 also offsets[0]); every count to 0.
__global__ void __launch_bounds__(BATCH_BLOCK) k_batch_clear(const BatchPairDev* __restrict__ pairs, int n_pairs,
                                                            const uint32_t* __restrict__ stile_pair, uint64_t n_stiles) {
  for (uint64_t i = uint64_t(blockIdx.x) * BATCH_BLOCK + threadIdx.x; i < uint64_t(n_pairs);
       i += uint64_t(gridDim.x) * BATCH_BLOCK)
    *pairs[i].count = 0ull;
  for (uint64_t t = blockIdx.x; t < n_stiles; t += gridDim.x) {
    const BatchPairDev& P = pairs[stile_pair[t]];
    const uint64_t lt = t - P.stile0;
    const uint64_t j0 = lt * BATCH_STILE;
    const uint64_t j1 = umin64(j0 + BATCH_STILE, P.n_buckets);
    uint32_t* data = P.offsets + 1;
    for (uint64_t j = j0 + threadIdx.x; j < j1; j += BATCH_BLOCK) data[j] = 0u;
    if (lt == 0 && threadIdx.x == 0) P.offsets[0] = 0u;
  }
}

template <typename KeyT>
__global__ void __launch_bounds__(BATCH_BLOCK) k_batch_count(const BatchPairDev* __restrict__ pairs,
                                                            const uint32_t* __restrict__ ktile_pair, uint64_t n_ktiles) {
  for (uint64_t t = blockIdx.x; t < n_ktiles; t += gridDim.x) {
    const BatchPairDev& P = pairs[ktile_pair[t]];
    const KeyT* keys = static_cast<const KeyT*>(P.keys);
    const uint64_t base = (t - P.ktile0) * BATCH_KTILE;
    const BucketMap bm = P.bm;
    uint32_t* cnt = P.offsets + 1;
#pragma unroll
    for (uint32_t u = 0; u < BATCH_KPT; u++) {
      const uint64_t i = base + u * BATCH_BLOCK + threadIdx.x;
      const bool ok = i < P.n;
      const KeyT k = ok ? keys[i] : KeyT(0);
      warp_aggregated_count(cnt, ok ? bm.of_key(k) : 0u, ok);
    }
  }
}

// Per-pair in-place exclusive scan of offsets[1..B]: the scan of k_scan_u32
// with one look-back chain per pair (status words of pair p start at its
// first scan tile).  Tiles are taken in ticket order across the batch, so
// every tile a look-back waits on is already held by a running CTA.
template <int ITEMS>
__global__ void __launch_bounds__(BATCH_BLOCK) k_batch_scan(const BatchPairDev* __restrict__ pairs,
                                                           const uint32_t* __restrict__ stile_pair, uint64_t n_stiles,
                                                           uint64_t* __restrict__ status, unsigned* ticket) {
  constexpr int TILE = BATCH_BLOCK * ITEMS;
  static_assert(TILE == BATCH_STILE, "scan tile");
  __shared__ uint32_t s[TILE + TILE / 32];
  __shared__ uint32_t red[BATCH_BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t t = s_tile;
    if (t >= n_stiles) break;
    const BatchPairDev& P = pairs[stile_pair[t]];
    const uint64_t lt = t - P.stile0;
    uint32_t* data = P.offsets + 1;
    const uint64_t count = P.n_buckets;
    const uint64_t base = lt * TILE;
#pragma unroll
    for (int k = 0; k < ITEMS; k++) {
      const int si = k * BATCH_BLOCK + threadIdx.x;
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
    const uint32_t excl = block_exclusive_scan<BATCH_BLOCK>(sum, red, &tile_total);
    if (threadIdx.x < 32) {
      const uint64_t p = lookback_exclusive(status + P.stile0, lt, tile_total);
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
      const int si = k * BATCH_BLOCK + threadIdx.x;
      const uint64_t i = base + si;
      if (i < count) data[i] = s[si + si / 32];
    }
    __syncthreads();
  }
}

template <typename KeyT>
__global__ void __launch_bounds__(BATCH_BLOCK) k_batch_scatter(const BatchPairDev* __restrict__ pairs,
                                                              const uint32_t* __restrict__ ktile_pair,
                                                              uint64_t n_ktiles) {
  for (uint64_t t = blockIdx.x; t < n_ktiles; t += gridDim.x) {
    const BatchPairDev& P = pairs[ktile_pair[t]];
    const KeyT* keys = static_cast<const KeyT*>(P.keys);
    KeyT* out = static_cast<KeyT*>(P.keys_out);
    uint32_t* idx = P.idx_out;
    const uint64_t base = (t - P.ktile0) * BATCH_KTILE;
    const BucketMap bm = P.bm;
    uint32_t* cursor = P.offsets + 1;
    // all the tile's cursor bumps are issued before any of their results is
    // used, so the warp waits for one atomic round trip, not BATCH_KPT
    KeyT k[BATCH_KPT];
    uint32_t got[BATCH_KPT], rank[BATCH_KPT], leader[BATCH_KPT];
#pragma unroll
    for (uint32_t u = 0; u < BATCH_KPT; u++) {
      const uint64_t i = base + u * BATCH_BLOCK + threadIdx.x;
      const bool ok = i < P.n;
      k[u] = ok ? keys[i] : KeyT(0);
      const uint32_t b = ok ? bm.of_key(k[u]) : 0u;
      const unsigned peers = __match_any_sync(FULL_MASK, ok ? uint64_t(b) : (1ull << 40));
      leader[u] = __ffs(peers) - 1;
      rank[u] = __popc(peers & lanemask_lt());
      got[u] = (ok && lane_id() == leader[u]) ? atomicAdd(cursor + b, uint32_t(__popc(peers))) : 0u;
    }
#pragma unroll
    for (uint32_t u = 0; u < BATCH_KPT; u++) {
      const uint64_t i = base + u * BATCH_BLOCK + threadIdx.x;
      const uint32_t pos = __shfl_sync(FULL_MASK, got[u], leader[u]) + rank[u];
      if (i < P.n) {
        out[pos] = k[u];
        if (idx) idx[pos] = static_cast<uint32_t>(i);
      }
    }
  }
}

// Probe: tiles of BATCH_QTILE queries in ticket order; thread t takes the
// BATCH_QPT consecutive queries at tile*QTILE + t*QPT, as k_probe does, so
// the pairs come out in the same order as the single-pair direct probe.
template <typename KeyT>
__global__ void __launch_bounds__(BATCH_BLOCK) k_batch_probe(const BatchPairDev* __restrict__ pairs,
                                                            const uint32_t* __restrict__ qtile_pair, uint64_t n_qtiles,
                                                            uint64_t* __restrict__ status, unsigned* ticket) {
  __shared__ uint64_t red[BATCH_BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t t = s_tile;
    if (t >= n_qtiles) break;
    const BatchPairDev& P = pairs[qtile_pair[t]];
    const uint64_t lt = t - P.qtile0;
    const KeyT* q = static_cast<const KeyT*>(P.query);
    const KeyT* a_keys = static_cast<const KeyT*>(P.keys_out);
    const uint32_t* a_off = P.offsets;
    const uint32_t* a_idx = P.idx_out;
    const BucketMap bm = P.bm;
    const uint64_t nq = P.nq;
    const uint64_t q0 = lt * BATCH_QTILE + uint64_t(threadIdx.x) * BATCH_QPT;
    KeyT key[BATCH_QPT];
    uint32_t lo[BATCH_QPT], hi[BATCH_QPT];
    uint64_t c = 0;
#pragma unroll
    for (uint32_t j = 0; j < BATCH_QPT; j++) {
      lo[j] = hi[j] = 0;
      key[j] = 0;
      if (q0 + j < nq) {
        key[j] = q[q0 + j];
        const uint32_t b = bm.of_key(key[j]);
        lo[j] = a_off[b];
        hi[j] = a_off[b + 1];
      }
    }
    // every query's first bucket entry is loaded before any is compared, so
    // the four dependent loads overlap; the rest of a bucket follows
    KeyT first[BATCH_QPT];
#pragma unroll
    for (uint32_t j = 0; j < BATCH_QPT; j++) first[j] = lo[j] < hi[j] ? a_keys[lo[j]] : KeyT(0);
#pragma unroll
    for (uint32_t j = 0; j < BATCH_QPT; j++) {
      if (lo[j] < hi[j]) {
        c += (first[j] == key[j]);
        for (uint32_t x = lo[j] + 1; x < hi[j]; x++) c += (a_keys[x] == key[j]);
      }
    }
    uint64_t tile_total;
    const uint64_t excl = block_exclusive_scan<BATCH_BLOCK>(c, red, &tile_total);
    if (threadIdx.x < 32) {
      const uint64_t p = lookback_exclusive(status + P.qtile0, lt, tile_total);
      if (threadIdx.x == 0) s_prefix = p;
    }
    __syncthreads();
    const uint64_t prefix = s_prefix;
    if (P.pairs && c) {
      uint64_t pos = prefix + excl;
      uint2* out = reinterpret_cast<uint2*>(P.pairs);
#pragma unroll
      for (uint32_t j = 0; j < BATCH_QPT; j++) {
        for (uint32_t x = lo[j]; x < hi[j]; x++) {
          if (a_keys[x] == key[j]) {
            if (pos < P.pair_cap) out[pos] = make_uint2(a_idx ? a_idx[x] : x, static_cast<uint32_t>(q0 + j));
            pos++;
          }
        }
      }
    }
    if (threadIdx.x == 0 && lt == P.qtiles - 1) {
      const uint64_t total = prefix + tile_total;
      *P.count = total;
      if (P.pairs && total > P.pair_cap) record_error(HG_ERR_PAIR_CAPACITY);
    }
    __syncthreads();
  }
}

// Host-side batch: the plan, the device workspace and the descriptors.
struct BatchPlan {
  int n_pairs = 0;
  int key_bytes = 8;
  uint64_t n_ktiles = 0, n_stiles = 0, n_qtiles = 0;
  size_t off_pairs = 0, off_kmap = 0, off_smap = 0, off_qmap = 0;
  size_t off_zero = 0, off_sstat = 0, off_qstat = 0, off_ticket = 0, total = 0;
};

}  // namespace hg

struct hg_batch {
  hg::BatchPlan plan;
  int device = 0;
  char* d_mem = nullptr;
};

namespace hg {

static hg_status batch_plan(const hg_batch_pair* pairs, int n_pairs, int key_bytes, BatchPlan* plan,
                            std::vector<BatchPairDev>* dev, std::vector<uint32_t>* kmap,
                            std::vector<uint32_t>* smap, std::vector<uint32_t>* qmap) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_pairs < 0 || (n_pairs > 0 && !pairs)) return HG_ERR_INVALID_ARGUMENT;
  BatchPlan p;
  p.n_pairs = n_pairs;
  p.key_bytes = key_bytes;
  dev->resize(n_pairs);
  for (int i = 0; i < n_pairs; i++) {
    const hg_batch_pair& a = pairs[i];
    if (a.n_buckets == 0 || !a.d_offsets || !a.d_count) return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_batch_create: pair without buckets, offsets or count");
    if ((a.n > 0 && (!a.d_keys || !a.d_keys_out)) || (a.nq > 0 && !a.d_query))
      return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_batch_create: pair with keys or queries but no buffer");
    if (a.n >= (1ull << 32) || a.nq >= (1ull << 32) || a.n_buckets > (1ull << 32))
      return lib_fail(HG_ERR_TOO_LARGE, "hg_batch_create: a pair exceeds 2^32 keys, queries or buckets");
    BatchPairDev& d = (*dev)[i];
    d.keys = a.d_keys;
    d.query = a.d_query;
    d.offsets = a.d_offsets;
    d.keys_out = a.d_keys_out;
    d.idx_out = a.d_idx_out;
    d.pairs = a.d_pairs;
    d.count = a.d_count;
    d.n = a.n;
    d.nq = a.nq;
    d.n_buckets = a.n_buckets;
    d.pair_cap = a.d_pairs ? a.pair_cap : 0;
    d.bm = BucketMap::make(a.n_buckets);
    const uint64_t kt = (a.n + BATCH_KTILE - 1) / BATCH_KTILE;
    const uint64_t st = (a.n_buckets + BATCH_STILE - 1) / BATCH_STILE;
    const uint64_t qt = (a.nq + BATCH_QTILE - 1) / BATCH_QTILE;
    d.ktile0 = p.n_ktiles;
    d.stile0 = p.n_stiles;
    d.qtile0 = p.n_qtiles;
    d.qtiles = qt;
    p.n_ktiles += kt;
    p.n_stiles += st;
    p.n_qtiles += qt;
    if (p.n_ktiles >= (1ull << 32) || p.n_stiles >= (1ull << 32) || p.n_qtiles >= (1ull << 32))
      return lib_fail(HG_ERR_TOO_LARGE, "hg_batch_create: more than 2^32 tiles");
  }
  kmap->resize(p.n_ktiles);
  smap->resize(p.n_stiles);
  qmap->resize(p.n_qtiles);
  for (int i = 0; i < n_pairs; i++) {
    const BatchPairDev& d = (*dev)[i];
    const uint64_t kt = (d.n + BATCH_KTILE - 1) / BATCH_KTILE;
    const uint64_t st = (d.n_buckets + BATCH_STILE - 1) / BATCH_STILE;
    std::fill(kmap->begin() + d.ktile0, kmap->begin() + d.ktile0 + kt, uint32_t(i));
    std::fill(smap->begin() + d.stile0, smap->begin() + d.stile0 + st, uint32_t(i));
    std::fill(qmap->begin() + d.qtile0, qmap->begin() + d.qtile0 + d.qtiles, uint32_t(i));
  }
  size_t off = 0;
  p.off_pairs = off;  off = align_up(off + sizeof(BatchPairDev) * std::max(n_pairs, 1));
  p.off_kmap = off;   off = align_up(off + 4 * std::max<uint64_t>(p.n_ktiles, 1));
  p.off_smap = off;   off = align_up(off + 4 * std::max<uint64_t>(p.n_stiles, 1));
  p.off_qmap = off;   off = align_up(off + 4 * std::max<uint64_t>(p.n_qtiles, 1));
  p.off_zero = off;   // zeroed by every run: look-back status words and tickets
  p.off_sstat = off;  off = align_up(off + 8 * std::max<uint64_t>(p.n_stiles, 1));
  p.off_qstat = off;  off = align_up(off + 8 * std::max<uint64_t>(p.n_qtiles, 1));
  p.off_ticket = off; off = align_up(off + 4 * sizeof(unsigned));
  p.total = off;
  *plan = p;
  return HG_OK;
}

template <typename KeyT>
static hg_status batch_launch(const BatchPlan& p, char* ws, cudaStream_t s) {
  const BatchPairDev* pairs = reinterpret_cast<const BatchPairDev*>(ws + p.off_pairs);
  const uint32_t* kmap = reinterpret_cast<const uint32_t*>(ws + p.off_kmap);
  const uint32_t* smap = reinterpret_cast<const uint32_t*>(ws + p.off_smap);
  const uint32_t* qmap = reinterpret_cast<const uint32_t*>(ws + p.off_qmap);
  uint64_t* sstat = reinterpret_cast<uint64_t*>(ws + p.off_sstat);
  uint64_t* qstat = reinterpret_cast<uint64_t*>(ws + p.off_qstat);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  HG_CUDA(cudaMemsetAsync(ws + p.off_zero, 0, p.total - p.off_zero, s), "hg_batch_run: state memset");
  if (p.n_pairs == 0) return HG_OK;
  const uint64_t resident = uint64_t(device_sm_count()) * 8;  // 256-thread CTAs, 8 per SM
  auto grid_for = [&](uint64_t tiles) { return static_cast<unsigned>(std::max<uint64_t>(1, std::min(tiles, resident))); };
  {
    Phase ph(s, "batch_clear");
    count_launch();
    k_batch_clear<<<grid_for(std::max<uint64_t>(p.n_stiles, (p.n_pairs + BATCH_BLOCK - 1) / BATCH_BLOCK)), BATCH_BLOCK, 0, s>>>(
        pairs, p.n_pairs, smap, p.n_stiles);
  }
  if (p.n_ktiles) {
    Phase ph(s, "batch_count");
    count_launch();
    k_batch_count<KeyT><<<grid_for(p.n_ktiles), BATCH_BLOCK, 0, s>>>(pairs, kmap, p.n_ktiles);
  }
  {
    Phase ph(s, "batch_scan");
    count_launch();
    k_batch_scan<SCAN_ITEMS><<<grid_for(p.n_stiles), BATCH_BLOCK, 0, s>>>(pairs, smap, p.n_stiles, sstat, ticket);
  }
  if (p.n_ktiles) {
    Phase ph(s, "batch_scatter");
    count_launch();
    k_batch_scatter<KeyT><<<grid_for(p.n_ktiles), BATCH_BLOCK, 0, s>>>(pairs, kmap, p.n_ktiles);
  }
  if (p.n_qtiles) {
    Phase ph(s, "batch_probe");
    count_launch();
    k_batch_probe<KeyT><<<grid_for(p.n_qtiles), BATCH_BLOCK, 0, s>>>(pairs, qmap, p.n_qtiles, qstat, ticket + 1);
  }
  HG_CUDA(cudaPeekAtLastError(), "hg_batch_run: kernel launch");
  return HG_OK;
}

}  // namespace hg

using namespace hg;

extern "C" hg_status hg_batch_create(const hg_batch_pair* pairs, int n_pairs, int key_bytes, hg_stream_t stream,
                                     hg_batch** out) {
  if (!out) return HG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  BatchPlan plan;
  std::vector<BatchPairDev> dev;
  std::vector<uint32_t> kmap, smap, qmap;
  hg_status st = batch_plan(pairs, n_pairs, key_bytes, &plan, &dev, &kmap, &smap, &qmap);
  if (st != HG_OK) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  hg_batch* b = new hg_batch();
  b->plan = plan;
  cudaGetDevice(&b->device);
  void* mem = nullptr;
  cudaError_t e = cudaMallocAsync(&mem, plan.total, s);
  if (e != cudaSuccess) {
    delete b;
    cuda_fail(e, "hg_batch_create: workspace allocation");
    return e == cudaErrorMemoryAllocation ? HG_ERR_OUT_OF_MEMORY : HG_ERR_CUDA;
  }
  b->d_mem = static_cast<char*>(mem);
  auto up = [&](size_t off, const void* src, size_t bytes) -> cudaError_t {
    return bytes ? cudaMemcpyAsync(b->d_mem + off, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
  };
  if ((e = up(plan.off_pairs, dev.data(), dev.size() * sizeof(BatchPairDev))) != cudaSuccess ||
      (e = up(plan.off_kmap, kmap.data(), kmap.size() * 4)) != cudaSuccess ||
      (e = up(plan.off_smap, smap.data(), smap.size() * 4)) != cudaSuccess ||
      (e = up(plan.off_qmap, qmap.data(), qmap.size() * 4)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {  // the host vectors go out of scope
    cudaFreeAsync(b->d_mem, s);
    delete b;
    return cuda_fail(e, "hg_batch_create: descriptor upload");
  }
  *out = b;
  return HG_OK;
}

extern "C" hg_status hg_batch_run(const hg_batch* b, hg_stream_t stream) {
  if (!b) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return b->plan.key_bytes == 4 ? batch_launch<uint32_t>(b->plan, b->d_mem, s)
                                : batch_launch<uint64_t>(b->plan, b->d_mem, s);
}

extern "C" hg_status hg_batch_device_bytes(const hg_batch* b, size_t* bytes) {
  if (!b || !bytes) return HG_ERR_INVALID_ARGUMENT;
  *bytes = b->plan.total;
  return HG_OK;
}

extern "C" void hg_batch_free(hg_batch* b, hg_stream_t stream) {
  if (!b) return;
  if (b->d_mem) cudaFreeAsync(b->d_mem, reinterpret_cast<cudaStream_t>(stream));
  delete b;
}

extern "C" hg_status hg_batch_build_intersect(const hg_batch_pair* pairs, int n_pairs, int key_bytes,
                                              hg_stream_t stream) {
  hg_batch* b = nullptr;
  hg_status st = hg_batch_create(pairs, n_pairs, key_bytes, stream, &b);
  if (st != HG_OK) return st;
  st = hg_batch_run(b, stream);
  hg_batch_free(b, stream);
  return st;
}
