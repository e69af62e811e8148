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
// Large pairs take faster forms: the table through the partitioned build,
// the queries of a pair whose table fits an L2 budget through
// k_batch_l2probe (tiles in pair order, the pair's table read from L2, one
// atomic per tile on the pair's count, pairs grouped by tile), those of a
// larger table through the partitioned probe.
// Each pair's result is the one the single-pair direct path
// (k_count / k_scan_u32 / k_scatter / k_probe) gives.  The reference has no
// batched form; per pair it replaces build + intersect of
// src/MultiHashGraph.cu:408-740.
#include <algorithm>
#include <cstring>
#include <new>
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
  // partitioned form (pb: the table, pq: the queries); the direct kernels
  // take such a pair only if its partitioned pass overflowed
  uint32_t pb, pq;
  uint32_t nfb, nfq;                // fine partitions of the table / of the queries
  uint64_t fb0, fq0;                // first fine partition in the batch's lists
  uint64_t mt0, mq0;                // first pass-1 tile of the keys / of the queries
  uint32_t a_bulk;                  // the table's arrays are 16-byte aligned
  uint32_t pl;                      // L2 form of the probe: chunks [ltile0, ltile0 + ltiles)
  uint64_t ltile0, ltiles;
  uint32_t prebuilt;                // the table is already built: the pair is only probed
};

// Flags of a batch run: [0] a table's partitioned build overflowed, [1] a
// partitioned probe overflowed; the direct kernels then redo those pairs.
__device__ __forceinline__ bool batch_skip_build(const BatchPairDev& P, const uint32_t* flags) {
  return P.pb && !(*reinterpret_cast<const volatile uint32_t*>(flags) & FLAG_OVERFLOW);
}
__device__ __forceinline__ bool batch_skip_probe(const BatchPairDev& P, const uint32_t* flags) {
  return P.pl || (P.pq && !(*reinterpret_cast<const volatile uint32_t*>(flags + 1) & FLAG_OVERFLOW));
}

// Every pair's offsets to zero (tile lt of a pair clears entries
// [lt*STILE, ...) of offsets[1..B]; tile 0 also offsets[0]); every count to 0.
__global__ void __launch_bounds__(BATCH_BLOCK) k_batch_clear(const BatchPairDev* __restrict__ pairs, int n_pairs,
                                                            const uint32_t* __restrict__ stile_pair, uint64_t s_begin,
                                                            uint64_t s_end, const uint32_t* flags,
                                                            const uint32_t* gate) {
  if (entry_skip(gate)) return;
  if (!gate)  // the ungated launch zeroes every pair's count
    for (uint64_t i = uint64_t(blockIdx.x) * BATCH_BLOCK + threadIdx.x; i < uint64_t(n_pairs);
         i += uint64_t(gridDim.x) * BATCH_BLOCK)
      if (pairs[i].count) *pairs[i].count = 0ull;
  for (uint64_t t = s_begin + blockIdx.x; t < s_end; t += gridDim.x) {
    const BatchPairDev& P = pairs[stile_pair[t]];
    if (batch_skip_build(P, flags)) continue;
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
                                                            const uint32_t* __restrict__ ktile_pair, uint64_t k_begin,
                                                            uint64_t k_end, const uint32_t* flags, const uint32_t* gate) {
  if (entry_skip(gate)) return;
  for (uint64_t t = k_begin + blockIdx.x; t < k_end; t += gridDim.x) {
    const BatchPairDev& P = pairs[ktile_pair[t]];
    if (batch_skip_build(P, flags)) continue;
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
                                                           const uint32_t* __restrict__ stile_pair, uint64_t s_begin,
                                                           uint64_t s_end, uint64_t* __restrict__ status, unsigned* ticket,
                                                           const uint32_t* flags, const uint32_t* gate) {
  if (entry_skip(gate)) return;
  constexpr int TILE = BATCH_BLOCK * ITEMS;
  static_assert(TILE == BATCH_STILE, "scan tile");
  __shared__ uint32_t s[TILE + TILE / 32];
  __shared__ uint32_t red[BATCH_BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
  while (true) {
    if (threadIdx.x == 0) s_tile = s_begin + atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t t = s_tile;
    if (t >= s_end) break;
    const BatchPairDev& P = pairs[stile_pair[t]];
    if (batch_skip_build(P, flags)) {
      __syncthreads();  // every thread read s_tile before thread 0 takes the next ticket
      continue;
    }
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
                                                              uint64_t k_begin, uint64_t k_end, const uint32_t* flags,
                                                              const uint32_t* gate) {
  if (entry_skip(gate)) return;
  for (uint64_t t = k_begin + blockIdx.x; t < k_end; t += gridDim.x) {
    const BatchPairDev& P = pairs[ktile_pair[t]];
    if (batch_skip_build(P, flags)) continue;
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
      if (i < P.n && pos >= P.n) record_fault(HG_ERR_DEVICE_STATE);  // offsets past n: write nothing
      else if (i < P.n) {
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
                                                            const uint32_t* __restrict__ qtile_pair, uint64_t q_begin,
                                                            uint64_t q_end, uint64_t* __restrict__ status,
                                                            unsigned* ticket, const uint32_t* flags,
                                                            const uint32_t* gate) {
  if (entry_skip(gate)) return;
  __shared__ uint64_t red[BATCH_BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
  while (true) {
    if (threadIdx.x == 0) s_tile = q_begin + atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t t = s_tile;
    if (t >= q_end) break;
    const BatchPairDev& P = pairs[qtile_pair[t]];
    if (batch_skip_probe(P, flags)) {
      __syncthreads();  // every thread read s_tile before thread 0 takes the next ticket
      continue;
    }
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

// L2 form of a large pair's probe: the pair's table (at most l2_table_bytes
// bytes) was built just before and is read from L2 while the CTAs, which take
// tiles in pair order from a ticket, work on it.  Per thread BATCH_LQPT
// queries side by side (bucket bounds, first entries, the rest of each
// bucket; count and first match in registers); one block scan and ONE atomic
// on the pair's count reserve a tile's output.  A ticket hands out
// BATCH_LCHUNK consecutive tiles of one pair ("chunk"): the pair's descriptor
// is read once for them.
constexpr uint32_t BATCH_LQPT = 2;
constexpr uint32_t BATCH_LTILE = BATCH_BLOCK * BATCH_LQPT;
constexpr uint32_t BATCH_LCHUNK = 4;  // tiles of one pair per ticket: the pair's descriptor is read once for them

template <typename KeyT>
__global__ void __launch_bounds__(BATCH_BLOCK) k_batch_l2probe(const BatchPairDev* __restrict__ pairs,
                                                              const uint32_t* __restrict__ lchunk_pair,
                                                              uint64_t n_lchunks, unsigned* ticket) {
  if (entry_skip(nullptr)) return;
  constexpr int NW = BATCH_BLOCK / 32;
  __shared__ uint64_t red[NW + 1];
  __shared__ unsigned s_t[2];
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  // ticket of iteration i in s_t[i & 1]; the next one is taken during the
  // tile and published by the tile's barriers
  if (threadIdx.x == 0) s_t[0] = atomicAdd(ticket, 1u);
  __syncthreads();
  for (uint32_t it = 0;; it++) {
    const uint64_t c = s_t[it & 1];
    if (c >= n_lchunks) break;
    if (threadIdx.x == 0) s_t[(it + 1) & 1] = atomicAdd(ticket, 1u);
    const BatchPairDev& P = pairs[lchunk_pair[c]];
    const KeyT* q = static_cast<const KeyT*>(P.query);
    const KeyT* a_keys = static_cast<const KeyT*>(P.keys_out);
    const uint32_t* a_off = P.offsets;
    const uint32_t* a_idx = P.idx_out;
    const BucketMap bm = P.bm;
    const uint64_t nq = P.nq;
    uint32_t* pairs_out = P.pairs;
    const uint64_t pair_cap = P.pair_cap;
    unsigned long long* count = P.count;
    const uint64_t t0 = (c - P.ltile0) * BATCH_LCHUNK;
  for (uint32_t k = 0; k < BATCH_LCHUNK; k++) {
    const uint64_t r0 = (t0 + k) * BATCH_LTILE;
    if (r0 >= nq) break;  // the same for the whole CTA
    KeyT key[BATCH_LQPT];
    uint32_t lo[BATCH_LQPT], hi[BATCH_LQPT], cnt[BATCH_LQPT], ref[BATCH_LQPT];
#pragma unroll
    for (uint32_t j = 0; j < BATCH_LQPT; j++) {
      const uint64_t r = r0 + j * BATCH_BLOCK + threadIdx.x;
      key[j] = r < nq ? __ldcs(q + r) : KeyT(0);
    }
#pragma unroll
    for (uint32_t j = 0; j < BATCH_LQPT; j++) {
      const uint64_t r = r0 + j * BATCH_BLOCK + threadIdx.x;
      lo[j] = hi[j] = 0;
      if (r < nq) {
        const uint32_t b = bm.of_key(key[j]);
        lo[j] = a_off[b];
        hi[j] = a_off[b + 1];
      }
    }
    KeyT first[BATCH_LQPT];
#pragma unroll
    for (uint32_t j = 0; j < BATCH_LQPT; j++) first[j] = lo[j] < hi[j] ? a_keys[lo[j]] : KeyT(0);
    uint64_t mine = 0;
#pragma unroll
    for (uint32_t j = 0; j < BATCH_LQPT; j++) {
      cnt[j] = 0;
      ref[j] = 0;
      if (lo[j] < hi[j]) {
        if (first[j] == key[j]) {
          cnt[j] = 1;
          ref[j] = a_idx ? a_idx[lo[j]] : lo[j];
        }
        for (uint32_t x = lo[j] + 1; x < hi[j]; x++) {
          if (a_keys[x] == key[j]) {
            if (cnt[j] == 0) ref[j] = a_idx ? a_idx[x] : x;
            cnt[j]++;
          }
        }
      }
      mine += cnt[j];
    }
    const uint64_t inc = warp_inclusive_scan(mine);
    if (lane == 31) red[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      const uint64_t w = lane < NW ? red[lane] : 0ull;
      const uint64_t wi = warp_inclusive_scan(w);
      const uint64_t tot = __shfl_sync(FULL_MASK, wi, NW - 1);
      uint64_t base = 0;
      if (lane == 0 && tot) {
        base = atomicAdd(count, static_cast<unsigned long long>(tot));
        if (pairs_out && base + tot > pair_cap) record_error(HG_ERR_PAIR_CAPACITY);
      }
      base = __shfl_sync(FULL_MASK, base, 0);
      if (lane < NW) red[lane] = base + wi - w;
    }
    __syncthreads();
    uint64_t pos = red[warp] + inc - mine;
    __syncwarp();  // the warp's lane 31 rewrites red[warp] in the next tile
    if (pairs_out && mine) {
      uint2* out = reinterpret_cast<uint2*>(pairs_out);
#pragma unroll
      for (uint32_t j = 0; j < BATCH_LQPT; j++) {
        if (cnt[j] == 0) continue;
        const uint32_t qref = static_cast<uint32_t>(r0 + j * BATCH_BLOCK + threadIdx.x);
        if (cnt[j] == 1) {
          if (pos < pair_cap) out[pos] = make_uint2(ref[j], qref);
          pos++;
        } else {
          for (uint32_t x = lo[j]; x < hi[j]; x++) {
            if (a_keys[x] == key[j]) {
              if (pos < pair_cap) out[pos] = make_uint2(a_idx ? a_idx[x] : x, qref);
              pos++;
            }
          }
        }
      }
    }
  }
  }
}

// ---------------------------------------------------------------------------
// Partitioned form of large pairs: the pass-1 multisplit of each pair goes
// straight to its fine partitions (at most PASS1_GOOD_PARTS of them: no split
// pass), then the fine build and the fine probe of the single-table path run
// over every pair's partitions at once.  These sources feed those kernels.
// ---------------------------------------------------------------------------
template <typename KeyT, bool QUERIES>
struct BatchSplitTiles {
  const BatchPairDev* pairs;
  const uint32_t* tile_pair;
  uint64_t n_tiles;
  uint32_t shift;        // fine width (log2): partition = bucket >> shift
  uint64_t cap;          // record slots per fine partition
  uint32_t* fcount;
  KeyT* fkeys;
  uint32_t* fidx;
  __device__ __forceinline__ uint64_t ntiles() const { return n_tiles; }
  __device__ __forceinline__ SplitTile<KeyT> at(uint64_t t) const {
    const BatchPairDev& P = pairs[tile_pair[t]];
    const uint64_t base = (t - (QUERIES ? P.mq0 : P.mt0)) * PASS1_TILE;
    const uint64_t n = QUERIES ? P.nq : P.n;
    const uint32_t cnt = base < n ? static_cast<uint32_t>(umin64(PASS1_TILE, n - base)) : 0u;
    const uint64_t f0 = QUERIES ? P.fq0 : P.fb0;
    return SplitTile<KeyT>{static_cast<const KeyT*>(QUERIES ? P.query : P.keys), nullptr, base, cnt, P.bm, shift,
                           QUERIES ? P.nfq : P.nfb, cap, fcount + f0, fkeys + f0 * cap,
                           fidx ? fidx + f0 * cap : nullptr};
  }
};

template <typename KeyT>
struct BatchFine {
  const BatchPairDev* pairs;
  const uint32_t* part_pair;
  uint64_t n_parts;
  const KeyT* fkeys;
  const uint32_t* fidx;
  uint64_t capf;
  const uint32_t* fstart;  // scanned counts over every pair's partitions
  uint32_t fine_log2;
  __device__ __forceinline__ uint64_t count() const { return n_parts; }
  __device__ __forceinline__ uint2 meta(uint64_t f) const {
    const uint32_t s0 = fstart[pairs[part_pair[f]].fb0];  // the pair's first record
    return make_uint2(fstart[f] - s0, fstart[f + 1] - s0);
  }
  __device__ __forceinline__ FinePart<KeyT> at(uint64_t f) const {
    const BatchPairDev& P = pairs[part_pair[f]];
    const uint64_t b0 = (f - P.fb0) << fine_log2;
    const uint32_t nb = static_cast<uint32_t>(umin64(1ull << fine_log2, P.n_buckets - b0));
    return FinePart<KeyT>{fkeys + f * capf, fidx ? fidx + f * capf : nullptr, b0, nb, P.bm, P.offsets,
                          static_cast<KeyT*>(P.keys_out), P.idx_out};
  }
  __device__ __forceinline__ void finish(uint64_t f) const {
    const BatchPairDev& P = pairs[part_pair[f]];
    if (f == P.fb0) P.offsets[P.n_buckets] = static_cast<uint32_t>(P.n);
  }
};

template <typename KeyT>
struct BatchProbe {
  static constexpr bool kOneTable = false;  // one count per pair
  const BatchPairDev* pairs;
  const uint32_t* part_pair;
  uint64_t n_parts;
  const KeyT* qkeys;
  const uint32_t* qidx;
  uint64_t capq;
  const uint32_t* qstart;
  uint32_t fine_log2;
  __device__ __forceinline__ uint64_t count() const { return n_parts; }
  __device__ __forceinline__ uint2 meta(uint64_t f) const { return make_uint2(qstart[f], qstart[f + 1]); }
  __device__ __forceinline__ ProbePart<KeyT> at(uint64_t f) const {
    const BatchPairDev& P = pairs[part_pair[f]];
    const uint64_t b0 = (f - P.fq0) << fine_log2;
    const uint32_t nb = static_cast<uint32_t>(umin64(1ull << fine_log2, P.n_buckets - b0));
    return ProbePart<KeyT>{qkeys + f * capq, qidx + f * capq, b0, nb, P.bm, P.n_buckets, P.offsets,
                           static_cast<const KeyT*>(P.keys_out), P.idx_out, P.n, P.a_bulk != 0, P.pairs,
                           P.pair_cap, P.count};
  }
};

// Host-side batch: the plan, the device workspace and the descriptors.
constexpr uint64_t BATCH_PART_MIN = 1ull << 14;  // default: keys (queries) from which a pair is partitioned
constexpr uint32_t BATCH_FINE_LOG2 = 11;          // fine width of the partitioned build
constexpr uint64_t BATCH_L2_TABLE = uint64_t(24) << 20;  // default: table bytes up to which a large pair's probe reads L2

struct BatchPlan {
  int n_pairs = 0;
  int key_bytes = 8;
  uint64_t n_ktiles = 0, n_stiles = 0, n_qtiles = 0, n_ltiles = 0;
  uint64_t n_kd = 0, n_sd = 0, n_qd = 0;  // tiles of the pairs in the direct form (the ungated launches)
  // partitioned form
  uint64_t n_mt = 0, n_mq = 0;      // pass-1 tiles of the keys / of the queries
  uint64_t n_fb = 0, n_fq = 0;      // fine partitions of the tables / of the queries
  uint64_t capf = 0, capq = 0;      // record slots per fine partition
  uint32_t capa = 0;                // table records a probe CTA stages
  uint32_t lq = 12;                 // probe fine width (log2)
  uint32_t max_pb = 1, max_pq = 1;  // most fine partitions of one pair
  bool wi_b = false, ai_q = false, bulk_b = true, bulk_q = true;
  size_t smem1b = 0, smem1q = 0, smem3b = 0, smem3q = 0;
  size_t off_pairs = 0, off_kmap = 0, off_smap = 0, off_qmap = 0, off_lmap = 0;
  size_t off_mtmap = 0, off_mqmap = 0, off_fbmap = 0, off_fqmap = 0;
  size_t off_fbkeys = 0, off_fbidx = 0, off_fqkeys = 0, off_fqidx = 0;
  size_t off_zero = 0, off_sstat = 0, off_qstat = 0, off_ticket = 0, off_flags = 0;
  size_t off_fbcount = 0, off_fbstat = 0, off_fqcount = 0, off_fqstat = 0, total = 0;
};

}  // namespace hg

struct hg_batch {
  hg::BatchPlan plan;
  int device = 0;
  char* d_mem = nullptr;
};

namespace hg {

static hg_status batch_plan(const hg_batch_pair* pairs, int n_pairs, int key_bytes, const hg_batch_params& prm,
                            BatchPlan* plan,
                            std::vector<BatchPairDev>* dev, std::vector<uint32_t>* kmap,
                            std::vector<uint32_t>* smap, std::vector<uint32_t>* qmap,
                            std::vector<uint32_t>* mtmap, std::vector<uint32_t>* mqmap,
                            std::vector<uint32_t>* fbmap, std::vector<uint32_t>* fqmap,
                            std::vector<uint32_t>* lmap) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_pairs < 0 || (n_pairs > 0 && !pairs)) return HG_ERR_INVALID_ARGUMENT;
  BatchPlan p;
  p.n_pairs = n_pairs;
  p.key_bytes = key_bytes;
  dev->resize(n_pairs);
  for (int i = 0; i < n_pairs; i++) {
    const hg_batch_pair& a = pairs[i];
    if (a.n_buckets == 0 || !a.d_offsets || (a.nq > 0 && !a.d_count))
      return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_batch_create: pair without buckets, offsets or count");
    // d_keys NULL with n > 0: the table is already built in d_offsets /
    // d_keys_out / d_idx_out and is only probed
    if ((a.n > 0 && !a.d_keys_out) || (a.nq > 0 && !a.d_query))
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
    d.prebuilt = (a.n > 0 && !a.d_keys) ? 1u : 0u;
  }
  // Partitioned form: large pairs whose buckets make at most PASS1_GOOD_PARTS
  // fine partitions and whose partitions fit a CTA's shared memory.
  const uint64_t wb = 1ull << BATCH_FINE_LOG2;
  auto aligned = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
  for (int i = 0; i < n_pairs; i++) {
    BatchPairDev& d = (*dev)[i];
    const double per_b = double(d.n) * double(wb) / double(d.n_buckets);
    d.pb = (!d.prebuilt && d.n >= prm.part_min && (d.n_buckets + wb - 1) / wb <= PASS1_GOOD_PARTS && per_b <= 4096.0)
               ? 1u : 0u;
    if (d.pb) {
      p.capf = std::max(p.capf, slack_capacity(per_b, 64));
      p.wi_b = p.wi_b || d.idx_out != nullptr;
      p.bulk_b = p.bulk_b && aligned(d.keys);
    }
    d.a_bulk = (aligned(d.offsets) && aligned(d.keys_out) && (!d.idx_out || aligned(d.idx_out))) ? 1u : 0u;
  }
  const size_t rec_b = key_bytes + (p.wi_b ? 4 : 0);
  p.smem3b = align_up(8 * wb, 16) + p.capf * (2 * rec_b + 6);
  if (p.smem3b > SMEM_BUDGET)
    for (auto& d : *dev) d.pb = 0;
  // the L2 form for large pairs whose whole table fits the L2 budget
  for (auto& d : *dev) {
    const uint64_t table_bytes = 4 * (d.n_buckets + 1) + d.n * (key_bytes + (d.idx_out ? 4 : 0));
    d.pl = (d.nq >= prm.part_min && d.n > 0 && table_bytes <= prm.l2_table_bytes) ? 1u : 0u;
  }
  // the probe's fine width: the widest whose staging fits one CTA
  for (uint32_t lq = 12; lq >= 10; lq--) {
    const uint64_t wq = 1ull << lq;
    uint64_t capq = 0, capa = 0;
    bool ai = false, any = false;
    for (auto& d : *dev) {
      const double per_q = double(d.nq) * double(wq) / double(d.n_buckets);
      const double per_a = double(d.n) * double(wq) / double(d.n_buckets);
      d.pq = (!d.pl && d.nq >= prm.part_min && d.n > 0 && (d.n_buckets + wq - 1) / wq <= PASS1_GOOD_PARTS &&
              per_q <= 8192.0 && per_a <= 8192.0) ? 1u : 0u;
      if (!d.pq) continue;
      any = true;
      capq = std::max(capq, slack_capacity(per_q, 64));
      capa = std::max(capa, slack_capacity(per_a, 64, 4.0));
      ai = ai || d.idx_out != nullptr;
    }
    if (!any) break;
    const size_t smem = fine_probe_smem(lq, static_cast<uint32_t>(capa), capq, key_bytes, ai, true);
    if (smem <= SMEM_BUDGET) {
      p.lq = lq;
      p.capq = capq;
      p.capa = static_cast<uint32_t>(capa);
      p.ai_q = ai;
      p.smem3q = smem;
      break;
    }
    if (lq == 10)
      for (auto& d : *dev) d.pq = 0;
  }
  if (!p.smem3q)
    for (auto& d : *dev) d.pq = 0;
  // Tiles of the direct kernels, numbered pairs in the direct form first, then
  // the partitioned ones: the ungated launches cover [0, n_kd) (keys),
  // [0, n_sd) (scans) and [0, n_qd) (queries); the gated fallback launches
  // the rest, which they redo only when a partitioned pass overflowed.  Pairs
  // probed in the L2 form never need the direct probe (nothing can overflow)
  // and get no query tiles.
  auto assign = [&](bool partitioned_build, bool partitioned_probe) {
    for (int i = 0; i < n_pairs; i++) {
      BatchPairDev& d = (*dev)[i];
      if (!d.prebuilt && (d.pb != 0) == partitioned_build) {
        d.ktile0 = p.n_ktiles;
        d.stile0 = p.n_stiles;
        p.n_ktiles += (d.n + BATCH_KTILE - 1) / BATCH_KTILE;
        p.n_stiles += (d.n_buckets + BATCH_STILE - 1) / BATCH_STILE;
      }
      if (!d.pl && (d.pq != 0) == partitioned_probe) {
        d.qtile0 = p.n_qtiles;
        d.qtiles = (d.nq + BATCH_QTILE - 1) / BATCH_QTILE;
        p.n_qtiles += d.qtiles;
      }
    }
  };
  for (auto& d : *dev) {
    d.qtile0 = 0;
    d.qtiles = 0;
  }
  assign(false, false);
  p.n_kd = p.n_ktiles;
  p.n_sd = p.n_stiles;
  p.n_qd = p.n_qtiles;
  assign(true, true);
  if (p.n_ktiles >= (1ull << 32) || p.n_stiles >= (1ull << 32) || p.n_qtiles >= (1ull << 32))
    return lib_fail(HG_ERR_TOO_LARGE, "hg_batch_create: more than 2^32 tiles");
  kmap->resize(p.n_ktiles);
  smap->resize(p.n_stiles);
  qmap->resize(p.n_qtiles);
  for (int i = 0; i < n_pairs; i++) {
    const BatchPairDev& d = (*dev)[i];
    const uint64_t kt = d.prebuilt ? 0 : (d.n + BATCH_KTILE - 1) / BATCH_KTILE;
    const uint64_t st = d.prebuilt ? 0 : (d.n_buckets + BATCH_STILE - 1) / BATCH_STILE;
    std::fill(kmap->begin() + d.ktile0, kmap->begin() + d.ktile0 + kt, uint32_t(i));
    std::fill(smap->begin() + d.stile0, smap->begin() + d.stile0 + st, uint32_t(i));
    std::fill(qmap->begin() + d.qtile0, qmap->begin() + d.qtile0 + d.qtiles, uint32_t(i));
  }
  // pass-1 tiles and fine partitions of the partitioned pairs
  for (int i = 0; i < n_pairs; i++) {
    BatchPairDev& d = (*dev)[i];
    if (d.pb) {
      d.nfb = static_cast<uint32_t>((d.n_buckets + wb - 1) / wb);
      d.fb0 = p.n_fb;
      d.mt0 = p.n_mt;
      p.n_fb += d.nfb;
      p.n_mt += (d.n + PASS1_TILE - 1) / PASS1_TILE;
      p.max_pb = std::max(p.max_pb, d.nfb);
    }
    if (d.pq) {
      d.nfq = static_cast<uint32_t>((d.n_buckets + (1ull << p.lq) - 1) >> p.lq);
      d.fq0 = p.n_fq;
      d.mq0 = p.n_mq;
      p.n_fq += d.nfq;
      p.n_mq += (d.nq + PASS1_TILE - 1) / PASS1_TILE;
      p.max_pq = std::max(p.max_pq, d.nfq);
      p.bulk_q = p.bulk_q && aligned(d.query);
    }
  }
  for (int i = 0; i < n_pairs; i++) {
    BatchPairDev& d = (*dev)[i];
    d.ltile0 = p.n_ltiles;  // counted in chunks of BATCH_LCHUNK tiles
    d.ltiles = d.pl ? (d.nq + uint64_t(BATCH_LTILE) * BATCH_LCHUNK - 1) / (uint64_t(BATCH_LTILE) * BATCH_LCHUNK) : 0;
    p.n_ltiles += d.ltiles;
  }
  if (p.n_mt >= (1ull << 32) || p.n_mq >= (1ull << 32) || p.n_fb >= (1ull << 32) || p.n_fq >= (1ull << 32) ||
      p.n_ltiles >= (1ull << 32))
    return lib_fail(HG_ERR_TOO_LARGE, "hg_batch_create: more than 2^32 partition tiles");
  lmap->resize(p.n_ltiles);
  for (int i = 0; i < n_pairs; i++) {
    const BatchPairDev& d = (*dev)[i];
    std::fill(lmap->begin() + d.ltile0, lmap->begin() + d.ltile0 + d.ltiles, uint32_t(i));
  }
  p.smem1b = pass1_smem(p.max_pb, key_bytes, PASS1_TILE);
  p.smem1q = pass1_smem(p.max_pq, key_bytes, PASS1_TILE);
  mtmap->resize(p.n_mt);
  mqmap->resize(p.n_mq);
  fbmap->resize(p.n_fb);
  fqmap->resize(p.n_fq);
  for (int i = 0; i < n_pairs; i++) {
    const BatchPairDev& d = (*dev)[i];
    if (d.pb) {
      std::fill(mtmap->begin() + d.mt0, mtmap->begin() + d.mt0 + (d.n + PASS1_TILE - 1) / PASS1_TILE, uint32_t(i));
      std::fill(fbmap->begin() + d.fb0, fbmap->begin() + d.fb0 + d.nfb, uint32_t(i));
    }
    if (d.pq) {
      std::fill(mqmap->begin() + d.mq0, mqmap->begin() + d.mq0 + (d.nq + PASS1_TILE - 1) / PASS1_TILE, uint32_t(i));
      std::fill(fqmap->begin() + d.fq0, fqmap->begin() + d.fq0 + d.nfq, uint32_t(i));
    }
  }
  auto tiles_of = [](uint64_t n) { return std::max<uint64_t>((n + SCAN_TILE - 1) / SCAN_TILE, 1); };
  size_t off = 0;
  p.off_pairs = off;   off = align_up(off + sizeof(BatchPairDev) * std::max(n_pairs, 1));
  p.off_kmap = off;    off = align_up(off + 4 * std::max<uint64_t>(p.n_ktiles, 1));
  p.off_smap = off;    off = align_up(off + 4 * std::max<uint64_t>(p.n_stiles, 1));
  p.off_qmap = off;    off = align_up(off + 4 * std::max<uint64_t>(p.n_qtiles, 1));
  p.off_lmap = off;    off = align_up(off + 4 * std::max<uint64_t>(p.n_ltiles, 1));
  p.off_mtmap = off;   off = align_up(off + 4 * std::max<uint64_t>(p.n_mt, 1));
  p.off_mqmap = off;   off = align_up(off + 4 * std::max<uint64_t>(p.n_mq, 1));
  p.off_fbmap = off;   off = align_up(off + 4 * std::max<uint64_t>(p.n_fb, 1));
  p.off_fqmap = off;   off = align_up(off + 4 * std::max<uint64_t>(p.n_fq, 1));
  p.off_fbkeys = off;  off = align_up(off + p.n_fb * p.capf * key_bytes);
  p.off_fbidx = off;   off = align_up(off + (p.wi_b ? p.n_fb * p.capf * 4 : 0));
  p.off_fqkeys = off;  off = align_up(off + p.n_fq * p.capq * key_bytes);
  p.off_fqidx = off;   off = align_up(off + p.n_fq * p.capq * 4);
  p.off_zero = off;    // zeroed by every run: look-back state, tickets, flags, partition counters
  p.off_sstat = off;   off = align_up(off + 8 * std::max<uint64_t>(p.n_stiles, 1));
  p.off_qstat = off;   off = align_up(off + 8 * std::max<uint64_t>(p.n_qtiles, 1));
  p.off_ticket = off;  off = align_up(off + 8 * sizeof(unsigned));
  p.off_flags = off;   off = align_up(off + 2 * sizeof(uint32_t));
  p.off_fbcount = off; off = align_up(off + 4 * (p.n_fb + 1));
  p.off_fbstat = off;  off = align_up(off + 8 * tiles_of(p.n_fb));
  p.off_fqcount = off; off = align_up(off + 4 * (p.n_fq + 1));
  p.off_fqstat = off;  off = align_up(off + 8 * tiles_of(p.n_fq));
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
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + p.off_flags);
  HG_CUDA(cudaMemsetAsync(ws + p.off_zero, 0, p.total - p.off_zero, s), "hg_batch_run: state memset");
  if (p.n_pairs == 0) return HG_OK;
  const uint64_t resident = uint64_t(device_sm_count()) * 8;  // 256-thread CTAs, 8 per SM
  auto grid_for = [&](uint64_t tiles) { return static_cast<unsigned>(std::max<uint64_t>(1, std::min(tiles, resident))); };
  hg_status st = HG_OK;
  // partitioned pass 1 (keys or queries of the partitioned pairs), then the
  // scan of their fine-partition counts
  auto split_pass = [&](auto src, bool with_idx, bool bulk, size_t smem, uint32_t max_parts, uint32_t* fl,
                        uint32_t* fcount, uint64_t n_f, uint64_t* fstat, unsigned* tk, const char* name,
                        const char* scan_name) {
    using Src = decltype(src);
    auto go = [&](auto kern) {
      const int bps = blocks_per_sm(kern, PASS1_BLOCK, smem);
      if (bps <= 0) {
        st = lib_fail(HG_ERR_CUDA, "batch multisplit kernel cannot be resident");
        return;
      }
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(src.n_tiles, uint64_t(device_sm_count()) * bps));
      Phase ph(s, name);
      count_launch();
      kern<<<std::max(grid, 1u), PASS1_BLOCK, smem, s>>>(src, max_parts, fl);
    };
    if (with_idx) {
      if (bulk) go(k_multisplit<KeyT, true, PASS1_BLOCK, PASS1_KPT, true, Src>);
      else go(k_multisplit<KeyT, true, PASS1_BLOCK, PASS1_KPT, false, Src>);
    } else {
      if (bulk) go(k_multisplit<KeyT, false, PASS1_BLOCK, PASS1_KPT, true, Src>);
      else go(k_multisplit<KeyT, false, PASS1_BLOCK, PASS1_KPT, false, Src>);
    }
    launch_scan(fcount, n_f, fstat, tk, nullptr, fcount + n_f, nullptr, s, scan_name);
  };
  if (p.n_mt) {
    using Src = BatchSplitTiles<KeyT, false>;
    const Src src{pairs, reinterpret_cast<const uint32_t*>(ws + p.off_mtmap), p.n_mt, BATCH_FINE_LOG2, p.capf,
                  reinterpret_cast<uint32_t*>(ws + p.off_fbcount), reinterpret_cast<KeyT*>(ws + p.off_fbkeys),
                  p.wi_b ? reinterpret_cast<uint32_t*>(ws + p.off_fbidx) : nullptr};
    split_pass(src, p.wi_b, p.bulk_b, p.smem1b, p.max_pb, flags, reinterpret_cast<uint32_t*>(ws + p.off_fbcount),
               p.n_fb, reinterpret_cast<uint64_t*>(ws + p.off_fbstat), ticket + 2, "batch_multisplit",
               "batch_part_scan");
    if (st != HG_OK) return st;
    using FSrc = BatchFine<KeyT>;
    const FSrc fsrc{pairs, reinterpret_cast<const uint32_t*>(ws + p.off_fbmap), p.n_fb,
                    reinterpret_cast<const KeyT*>(ws + p.off_fbkeys),
                    p.wi_b ? reinterpret_cast<const uint32_t*>(ws + p.off_fbidx) : nullptr, p.capf,
                    reinterpret_cast<const uint32_t*>(ws + p.off_fbcount), BATCH_FINE_LOG2};
    auto go = [&](auto kern) {
      const int bps = blocks_per_sm(kern, FINE_BLOCK, p.smem3b);
      if (bps <= 0) {
        st = lib_fail(HG_ERR_CUDA, "batch fine-build kernel cannot be resident");
        return;
      }
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(p.n_fb, uint64_t(device_sm_count()) * bps));
      Phase ph(s, "batch_fine_build");
      count_launch();
      kern<<<std::max(grid, 1u), FINE_BLOCK, p.smem3b, s>>>(fsrc, p.capf, BATCH_FINE_LOG2, flags);
    };
    if (p.wi_b) go(k_fine_build<KeyT, true, FINE_BLOCK, FSrc>);
    else go(k_fine_build<KeyT, false, FINE_BLOCK, FSrc>);
    if (st != HG_OK) return st;
  }
  // direct form: every pair not partitioned, and partitioned ones if their
  // pass overflowed (the kernels read the flags)
  // (each kind twice: the pairs in the direct form, then the partitioned
  // pairs gated on the build's overflow flag, which return at once without it)
  {
    Phase ph(s, "batch_clear");
    count_launch(2);
    k_batch_clear<<<grid_for(std::max<uint64_t>(p.n_sd, (p.n_pairs + BATCH_BLOCK - 1) / BATCH_BLOCK)), BATCH_BLOCK, 0, s>>>(
        pairs, p.n_pairs, smap, 0, p.n_sd, flags, nullptr);
    k_batch_clear<<<grid_for(p.n_stiles - p.n_sd), BATCH_BLOCK, 0, s>>>(pairs, p.n_pairs, smap, p.n_sd, p.n_stiles,
                                                                       flags, flags);
  }
  {
    Phase ph(s, "batch_count");
    count_launch(2);
    k_batch_count<KeyT><<<grid_for(p.n_kd), BATCH_BLOCK, 0, s>>>(pairs, kmap, 0, p.n_kd, flags, nullptr);
    k_batch_count<KeyT><<<grid_for(p.n_ktiles - p.n_kd), BATCH_BLOCK, 0, s>>>(pairs, kmap, p.n_kd, p.n_ktiles, flags,
                                                                             flags);
  }
  {
    Phase ph(s, "batch_scan");
    count_launch(2);
    k_batch_scan<SCAN_ITEMS><<<grid_for(p.n_sd), BATCH_BLOCK, 0, s>>>(pairs, smap, 0, p.n_sd, sstat, ticket, flags,
                                                                      nullptr);
    k_batch_scan<SCAN_ITEMS><<<grid_for(p.n_stiles - p.n_sd), BATCH_BLOCK, 0, s>>>(pairs, smap, p.n_sd, p.n_stiles,
                                                                                   sstat, ticket + 5, flags, flags);
  }
  {
    Phase ph(s, "batch_scatter");
    count_launch(2);
    k_batch_scatter<KeyT><<<grid_for(p.n_kd), BATCH_BLOCK, 0, s>>>(pairs, kmap, 0, p.n_kd, flags, nullptr);
    k_batch_scatter<KeyT><<<grid_for(p.n_ktiles - p.n_kd), BATCH_BLOCK, 0, s>>>(pairs, kmap, p.n_kd, p.n_ktiles, flags,
                                                                               flags);
  }
  if (p.n_ltiles) {
    Phase ph(s, "batch_l2_probe");
    count_launch();
    k_batch_l2probe<KeyT><<<grid_for(p.n_ltiles), BATCH_BLOCK, 0, s>>>(
        pairs, reinterpret_cast<const uint32_t*>(ws + p.off_lmap), p.n_ltiles, ticket + 4);
  }
  if (p.n_mq) {
    using Src = BatchSplitTiles<KeyT, true>;
    const Src src{pairs, reinterpret_cast<const uint32_t*>(ws + p.off_mqmap), p.n_mq, p.lq, p.capq,
                  reinterpret_cast<uint32_t*>(ws + p.off_fqcount), reinterpret_cast<KeyT*>(ws + p.off_fqkeys),
                  reinterpret_cast<uint32_t*>(ws + p.off_fqidx)};
    split_pass(src, true, p.bulk_q, p.smem1q, p.max_pq, flags + 1, reinterpret_cast<uint32_t*>(ws + p.off_fqcount),
               p.n_fq, reinterpret_cast<uint64_t*>(ws + p.off_fqstat), ticket + 3, "batch_probe_multisplit",
               "batch_probe_part_scan");
    if (st != HG_OK) return st;
    using PSrc = BatchProbe<KeyT>;
    const PSrc psrc{pairs, reinterpret_cast<const uint32_t*>(ws + p.off_fqmap), p.n_fq,
                    reinterpret_cast<const KeyT*>(ws + p.off_fqkeys), reinterpret_cast<const uint32_t*>(ws + p.off_fqidx),
                    p.capq, reinterpret_cast<const uint32_t*>(ws + p.off_fqcount), p.lq};
    auto go = [&](auto kern) {
      const int bps = blocks_per_sm(kern, FINE_PROBE_BLOCK, p.smem3q);
      if (bps <= 0) {
        st = lib_fail(HG_ERR_CUDA, "batch fine-probe kernel cannot be resident");
        return;
      }
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(p.n_fq, uint64_t(device_sm_count()) * bps));
      Phase ph(s, "batch_fine_probe");
      count_launch();
      kern<<<std::max(grid, 1u), FINE_PROBE_BLOCK, p.smem3q, s>>>(psrc, p.capq, p.lq, p.capa, flags + 1);
    };
    if (p.ai_q) go(k_fine_probe<KeyT, true, true, FINE_PROBE_BLOCK, PSrc>);
    else go(k_fine_probe<KeyT, false, true, FINE_PROBE_BLOCK, PSrc>);
    if (st != HG_OK) return st;
  }
  {
    Phase ph(s, "batch_probe");
    count_launch(2);
    k_batch_probe<KeyT><<<grid_for(p.n_qd), BATCH_BLOCK, 0, s>>>(pairs, qmap, 0, p.n_qd, qstat, ticket + 1, flags,
                                                                 nullptr);
    k_batch_probe<KeyT><<<grid_for(p.n_qtiles - p.n_qd), BATCH_BLOCK, 0, s>>>(pairs, qmap, p.n_qd, p.n_qtiles, qstat,
                                                                             ticket + 6, flags, flags + 1);
  }
  HG_CUDA(cudaPeekAtLastError(), "hg_batch_run: kernel launch");
  return HG_OK;
}

}  // namespace hg

using namespace hg;

extern "C" hg_status hg_batch_params_default(hg_batch_params* params) {
  if (!params) return HG_ERR_INVALID_ARGUMENT;
  params->part_min = BATCH_PART_MIN;
  params->l2_table_bytes = BATCH_L2_TABLE;
  return HG_OK;
}

extern "C" hg_status hg_batch_create_params(const hg_batch_pair* pairs, int n_pairs, int key_bytes,
                                            const hg_batch_params* params, hg_stream_t stream, hg_batch** out) {
  if (!out) return HG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  hg_batch_params prm;
  hg_batch_params_default(&prm);
  if (params) prm = *params;
  if (prm.part_min == 0) return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_batch_create: part_min must be positive");
  BatchPlan plan;
  std::vector<BatchPairDev> dev;
  std::vector<uint32_t> kmap, smap, qmap, mtmap, mqmap, fbmap, fqmap, lmap;
  hg_status st = batch_plan(pairs, n_pairs, key_bytes, prm, &plan, &dev, &kmap, &smap, &qmap, &mtmap, &mqmap, &fbmap,
                            &fqmap, &lmap);
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
      (e = up(plan.off_mtmap, mtmap.data(), mtmap.size() * 4)) != cudaSuccess ||
      (e = up(plan.off_mqmap, mqmap.data(), mqmap.size() * 4)) != cudaSuccess ||
      (e = up(plan.off_fbmap, fbmap.data(), fbmap.size() * 4)) != cudaSuccess ||
      (e = up(plan.off_fqmap, fqmap.data(), fqmap.size() * 4)) != cudaSuccess ||
      (e = up(plan.off_lmap, lmap.data(), lmap.size() * 4)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {  // the host vectors go out of scope
    cudaFreeAsync(b->d_mem, s);
    delete b;
    return cuda_fail(e, "hg_batch_create: descriptor upload");
  }
  *out = b;
  return HG_OK;
}

namespace hg {

// Staged creation, for the serving engine: the descriptors and tile maps are
// packed into the caller's pinned buffer at their device offsets and
// uploaded with ONE asynchronous copy, and the workspace comes from `pool`
// (stream-ordered).  Nothing synchronises: the caller keeps `pinned`
// untouched until the copy has completed (an event recorded after the
// batch's run covers it).  HG_ERR_TOO_LARGE when the descriptors do not fit
// `pinned_cap` bytes.
hg_status batch_create_staged(const hg_batch_pair* pairs, int n_pairs, int key_bytes, const hg_batch_params* params,
                              cudaStream_t s, cudaMemPool_t pool, void* pinned, size_t pinned_cap, hg_batch** out) {
  *out = nullptr;
  hg_batch_params prm;
  hg_batch_params_default(&prm);
  if (params) prm = *params;
  BatchPlan plan;
  std::vector<BatchPairDev> dev;
  std::vector<uint32_t> kmap, smap, qmap, mtmap, mqmap, fbmap, fqmap, lmap;
  hg_status st = batch_plan(pairs, n_pairs, key_bytes, prm, &plan, &dev, &kmap, &smap, &qmap, &mtmap, &mqmap, &fbmap,
                            &fqmap, &lmap);
  if (st != HG_OK) return st;
  const size_t desc_bytes = plan.off_fbkeys;  // the descriptor regions lead the workspace
  if (desc_bytes > pinned_cap) return HG_ERR_TOO_LARGE;
  char* h = static_cast<char*>(pinned);
  auto pack = [&](size_t off, const void* src, size_t bytes) {
    if (bytes) std::memcpy(h + off, src, bytes);
  };
  pack(plan.off_pairs, dev.data(), dev.size() * sizeof(BatchPairDev));
  pack(plan.off_kmap, kmap.data(), kmap.size() * 4);
  pack(plan.off_smap, smap.data(), smap.size() * 4);
  pack(plan.off_qmap, qmap.data(), qmap.size() * 4);
  pack(plan.off_mtmap, mtmap.data(), mtmap.size() * 4);
  pack(plan.off_mqmap, mqmap.data(), mqmap.size() * 4);
  pack(plan.off_fbmap, fbmap.data(), fbmap.size() * 4);
  pack(plan.off_fqmap, fqmap.data(), fqmap.size() * 4);
  pack(plan.off_lmap, lmap.data(), lmap.size() * 4);
  hg_batch* b = new (std::nothrow) hg_batch();
  if (!b) return HG_ERR_OUT_OF_MEMORY;
  b->plan = plan;
  cudaGetDevice(&b->device);
  void* mem = nullptr;
  cudaError_t e = pool ? cudaMallocFromPoolAsync(&mem, plan.total, pool, s) : cudaMallocAsync(&mem, plan.total, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mem, h, desc_bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    if (mem) cudaFreeAsync(mem, s);
    delete b;
    cudaGetLastError();
    return cuda_fail(e, "batch: staged creation");
  }
  b->d_mem = static_cast<char*>(mem);
  *out = b;
  return HG_OK;
}

}  // namespace hg

extern "C" hg_status hg_batch_create(const hg_batch_pair* pairs, int n_pairs, int key_bytes, hg_stream_t stream,
                                     hg_batch** out) {
  return hg_batch_create_params(pairs, n_pairs, key_bytes, nullptr, stream, out);
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

// The size classes of a batch -- direct form below part_min keys, L2 form of
// the probe for tables up to l2_table_bytes, partitioned forms above -- set
// the tile and thread shapes each pair gets.  The autotuner times candidate
// boundaries on the caller's own batch (coordinate search: part_min over
// 2^12 .. 2^16 with the default L2 budget, then the L2 budget over 0, 12, 24
// and 48 MB with the best part_min; each candidate one warm-up run and the
// best of two timed runs) and returns the fastest.  It runs the batch, so the
// outputs hold the last candidate's results (the same results: every form
// computes the same tables and the same pair sets).
extern "C" hg_status hg_batch_autotune(const hg_batch_pair* pairs, int n_pairs, int key_bytes, hg_stream_t stream,
                                       hg_batch_params* best, float* best_ms) {
  if (!best) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  hg_batch_params cur;
  hg_batch_params_default(&cur);
  float cur_ms = -1.f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  HG_CUDA(cudaEventCreate(&e0), "hg_batch_autotune: event");
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_fail(ce, "hg_batch_autotune: event");
  }
  auto time_params = [&](const hg_batch_params& prm, float* ms) -> hg_status {
    hg_batch* b = nullptr;
    hg_status st = hg_batch_create_params(pairs, n_pairs, key_bytes, &prm, stream, &b);
    if (st != HG_OK) return st;
    float bestc = -1.f;
    for (int r = 0; r < 3 && st == HG_OK; r++) {
      cudaEventRecord(e0, s);
      st = hg_batch_run(b, stream);
      cudaEventRecord(e1, s);
      const cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) st = cuda_fail(e, "hg_batch_autotune: run");
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (st == HG_OK && r > 0 && (bestc < 0.f || t < bestc)) bestc = t;  // run 0 warms up
    }
    hg_batch_free(b, stream);
    *ms = bestc;
    return st;
  };
  hg_status st = time_params(cur, &cur_ms);
  const uint64_t part_mins[] = {1ull << 12, 1ull << 13, 1ull << 15, 1ull << 16};
  for (uint64_t pm : part_mins) {
    if (st != HG_OK) break;
    hg_batch_params c = cur;
    c.part_min = pm;
    float t = 0.f;
    st = time_params(c, &t);
    if (st == HG_OK && t < cur_ms) {
      cur = c;
      cur_ms = t;
    }
  }
  const uint64_t l2s[] = {0ull, uint64_t(12) << 20, uint64_t(48) << 20};
  for (uint64_t l2 : l2s) {
    if (st != HG_OK) break;
    hg_batch_params c = cur;
    c.l2_table_bytes = l2;
    float t = 0.f;
    st = time_params(c, &t);
    if (st == HG_OK && t < cur_ms) {
      cur = c;
      cur_ms = t;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != HG_OK) return st;
  *best = cur;
  if (best_ms) *best_ms = cur_ms;
  return HG_OK;
}
