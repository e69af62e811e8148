// hg_probe.cu -- intersect kernels for sm_100a.
//
// The reference intersects two CSR tables built with the same bucket count:
// one thread per bucket runs a nested loop over A's and B's bucket lists,
// counting (pass 1) and then emitting (pass 2) every equal pair, with a
// cub::DeviceReduce::Sum and cub::DeviceScan::ExclusiveSum between the passes
// (include/MultiHashGraphDeviceOperators.cuh:513-543, src/MultiHashGraph.cu:631-740).
//
// Here every query key is hashed to its bucket in A, the bucket range is
// scanned for equal keys, and the matches are counted and emitted in ONE
// pass.  Three forms:
//   direct (k_probe): each tile of queries counts its matches, takes its
//     output offset from the decoupled look-back over tiles, and writes its
//     pairs in query order; the count-only form skips the look-back, first
//     looks keys up in the set of A's long-bucket keys (skew) and sends the
//     rest through a per-warp queue;
//   coarse (k_multisplit over the queries, then k_coarse_probe): the queries
//     grouped by L2-sized bucket ranges of A and probed from L2 -- the
//     default for large probes;
//   partitioned (pass 1, k_split, k_fine_probe): both sides staged in shared
//     memory per fine partition.
// The partitioned forms fall back to a gated direct probe when a query
// partition overflows (heavy duplicates among the queries).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>

#include "hg_bulk.cuh"
#include "hg_device.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"
#include "hg_scan.cuh"

namespace hg {

constexpr int PROBE_BLOCK = 256;
constexpr int PROBE_QPT = 4;
constexpr uint64_t PROBE_TILE = uint64_t(PROBE_BLOCK) * PROBE_QPT;

// ---------------------------------------------------------------------------
// Skew in count-only probes.  A query costs the length of its bucket in A.
// Under heavy duplication (Zipf keys) a few buckets hold tens of millions of
// copies of one key, and every copy of that key among the queries would scan
// its bucket: the product of the two multiplicities, as in the reference's
// nested bucket loop.  A count-only probe therefore first counts the keys of
// A's long buckets (HEAVY_MIN_LEN entries or more) once, into an
// open-addressing set key -> copies:
//   k_heavy_find   S evenly spaced CSR positions of A (a sample by mass) look
//                  for a long bucket; none found, the next steps return;
//   k_heavy_list   lists every long bucket (a pass over the offsets);
//   k_heavy_count  inserts every entry of every listed bucket into the set
//                  and counts it (a warp per bucket; buckets of more than
//                  HEAVY_HUGE entries shared by all CTAs in chunks).
// All copies of a key sit in its bucket, so the counts are exact.  A query
// whose key the set holds takes its count from there without reading its
// bucket bounds; a key the set does not hold whose bucket is long has no copy
// in A.  If a key found no slot (the set is not complete: flagged), counting
// stops and the set is not used: every query scans its bucket.  Buckets of
// COOP_MIN_LEN entries or more are scanned by the whole warp (32 entries per
// step, coalesced), shorter ones by the thread.  The count is exact in every
// case.  Thresholds measured on 2^28 Zipf(1.1) keys over 2^24 (count-only
// probe + set): long buckets from 64 entries and warp scans from 64, 8.07 +
// 1.81 ms; from 32 and 8, 5.82 + 1.78 ms; from 16 and 8 with the set looked
// up before the bounds, 4.90 + 2.05 ms.
// ---------------------------------------------------------------------------
constexpr uint32_t HEAVY_PROBES = 32;          // bound on a set lookup / insertion
constexpr uint32_t HEAVY_MIN_LEN = 16;         // buckets at least this long are counted into the set
constexpr uint32_t COOP_MIN_LEN = 8;           // buckets at least this long are scanned by a warp
constexpr uint32_t HEAVY_HUGE = 1u << 16;      // longer listed buckets are counted by all CTAs
constexpr uint32_t HEAVY_HUGE_MAX = 1u << 16;  // listed huge buckets (n_a < 2^32)
constexpr uint32_t HEAVY_CHUNK = 1u << 14;     // bucket entries per counting work item of a huge bucket
constexpr uint32_t HEAVY_SAMPLES = 1u << 14;   // positions k_heavy_find looks at

// Set slots for a table of n_a keys: n_a / 32 rounded up to a power of two
// in [2^10, 2^22]; the bucket list holds every bucket of HEAVY_MIN_LEN
// entries or more (at most n_a / HEAVY_MIN_LEN of them).
inline uint32_t heavy_slots(uint64_t n_a) {
  uint64_t s = 1024;
  while (s < (n_a >> 5) && s < (1ull << 22)) s <<= 1;
  return static_cast<uint32_t>(s);
}
// A listed bucket of at most HEAVY_HUGE entries is cut into items of at
// most HEAVY_ITEM entries, one warp each, so that no warp walks a long bucket
// alone (at 2^28 Zipf keys the warps' longest buckets set the kernel's time).
constexpr uint32_t HEAVY_ITEM = 1024;
inline uint64_t heavy_list_cap(uint64_t n_a) { return n_a / HEAVY_MIN_LEN + n_a / HEAVY_ITEM + 1; }
inline size_t heavy_bytes(uint64_t n_a) {
  return size_t(heavy_slots(n_a)) * 16 + size_t(heavy_list_cap(n_a)) * 8 + size_t(HEAVY_HUGE_MAX) * 8 + 16;
}

// The set lives in the workspace, zeroed before the probe: a slot holds ~key
// (0 = empty, so the all-ones 64-bit key is kept out of the set) and its count.
struct HeavySet {
  // [slots][2]: ~key, then the key's copies in A -- one 16-byte slot, so a
  // found key's count sits in the sector its key was read from
  unsigned long long* slot;
  uint2* bucket;              // [list_cap] listed items {lo, hi}: pieces of at most HEAVY_ITEM entries of the
                              // buckets of at most HEAVY_HUGE entries
  uint2* huge;                // [HEAVY_HUGE_MAX] listed longer buckets
  unsigned* state;            // [0] listed buckets, [1] listed huge buckets, [2] a long bucket was
                              // sampled, [3] a key found no slot (the set is not complete)
  uint32_t mask;              // slots - 1
  uint32_t list_cap;
  __device__ __forceinline__ unsigned long long* key_at(uint32_t h) const { return slot + 2ull * h; }
  __device__ __forceinline__ unsigned long long* count_at(uint32_t h) const { return slot + 2ull * h + 1; }
};

__device__ __forceinline__ uint32_t heavy_slot(uint64_t key, uint32_t mask) {
  return static_cast<uint32_t>((key * 0x9E3779B97F4A7C15ull) >> 40) & mask;
}

// Slot of `key` in the set, or ~0u when it is not there.
template <typename KeyT>
__device__ __forceinline__ uint32_t heavy_find(const HeavySet& hs, KeyT key) {
  const unsigned long long stored = ~static_cast<unsigned long long>(key);
  if (stored == 0 || hs.slot == nullptr) return ~0u;
  uint32_t h = heavy_slot(static_cast<uint64_t>(key), hs.mask);
  for (uint32_t p = 0; p < HEAVY_PROBES; p++) {
    const unsigned long long v = *hs.key_at(h);
    if (v == stored) return h;
    if (v == 0) return ~0u;
    h = (h + 1) & hs.mask;
  }
  return ~0u;
}

// Slot of `key`, claimed if new; ~0u (and the set marked incomplete) when no
// slot is free within HEAVY_PROBES steps or the key is the all-ones key.
template <typename KeyT>
__device__ __forceinline__ uint32_t heavy_insert(const HeavySet& hs, KeyT key) {
  const unsigned long long stored = ~static_cast<unsigned long long>(key);
  if (stored != 0) {
    uint32_t h = heavy_slot(static_cast<uint64_t>(key), hs.mask);
    for (uint32_t p = 0; p < HEAVY_PROBES; p++) {
      const unsigned long long v = *hs.key_at(h);
      if (v == stored) return h;
      if (v == 0) {
        const unsigned long long prev = atomicCAS(hs.key_at(h), 0ull, stored);
        if (prev == 0 || prev == stored) return h;
      }
      h = (h + 1) & hs.mask;
    }
  }
  atomicOr(hs.state + 3, 1u);
  return ~0u;
}

// Whether the set answers for every key of every long bucket (a key it does
// not hold has no copy in A).
__device__ __forceinline__ bool heavy_complete(const HeavySet& hs) {
  if (hs.slot == nullptr) return false;
  const volatile unsigned* st = hs.state;
  return st[2] != 0 && st[3] == 0;
}

// HEAVY_SAMPLES positions of A: does any sit in a long bucket?
template <typename KeyT>
__global__ void __launch_bounds__(256)
    k_heavy_find(const uint32_t* __restrict__ a_off, const KeyT* __restrict__ a_keys, uint64_t n_a, BucketMap bm,
                 HeavySet hs, const uint32_t* gate) {
  if (entry_skip(gate)) return;
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= HEAVY_SAMPLES || n_a == 0) return;
  const uint64_t pos = (i * n_a + n_a / 2) / HEAVY_SAMPLES;
  const uint32_t b = bm.of_key(a_keys[pos]);
  if (a_off[b + 1] - a_off[b] >= HEAVY_MIN_LEN) atomicOr(hs.state + 2, 1u);
}

// Lists every bucket of HEAVY_MIN_LEN entries or more (when the sample saw
// one): buckets of at most HEAVY_HUGE entries as items of at most HEAVY_ITEM
// entries, longer ones whole.  A CTA takes 2048 consecutive buckets at a time
// (8 per thread); one block scan places its items and one atomic per list
// reserves their slots (an atomic per long bucket on one counter
// serialised: 0.78 ms over 2^28 Zipf buckets).
constexpr int HEAVY_LIST_BLOCK = 256;
constexpr int HEAVY_LIST_BPT = 8;
__global__ void __launch_bounds__(HEAVY_LIST_BLOCK)
    k_heavy_list(const uint32_t* __restrict__ a_off, uint64_t n_buckets, HeavySet hs, const uint32_t* gate) {
  if (entry_skip(gate)) return;
  if (*reinterpret_cast<const volatile unsigned*>(hs.state + 2) == 0) return;
  constexpr uint64_t CHUNK = uint64_t(HEAVY_LIST_BLOCK) * HEAVY_LIST_BPT;
  __shared__ uint32_t red[HEAVY_LIST_BLOCK / 32 + 1];
  __shared__ uint32_t s_base[2];
  for (uint64_t c0 = uint64_t(blockIdx.x) * CHUNK; c0 < n_buckets; c0 += uint64_t(gridDim.x) * CHUNK) {
    const uint64_t b0 = c0 + uint64_t(threadIdx.x) * HEAVY_LIST_BPT;
    uint32_t off[HEAVY_LIST_BPT + 1];
#pragma unroll
    for (int u = 0; u <= HEAVY_LIST_BPT; u++) off[u] = b0 + u <= n_buckets ? a_off[b0 + u] : 0u;
    uint32_t normal = 0, huge = 0, items = 0;  // this thread's long buckets (bit u: bucket b0 + u)
#pragma unroll
    for (int u = 0; u < HEAVY_LIST_BPT; u++) {
      if (b0 + u < n_buckets) {
        const uint32_t len = off[u + 1] - off[u];
        if (len >= HEAVY_MIN_LEN) {
          if (len <= HEAVY_HUGE) {
            normal |= 1u << u;
            items += (len + HEAVY_ITEM - 1) / HEAVY_ITEM;
          } else {
            huge |= 1u << u;
          }
        }
      }
    }
    // both counts in one scan: items in the low 20 bits (at most 2048 * 64),
    // huge buckets in the high 12 (at most 2048)
    uint32_t total;
    const uint32_t excl =
        block_exclusive_scan<HEAVY_LIST_BLOCK>(items | (uint32_t(__popc(huge)) << 20), red, &total);
    if (threadIdx.x == 0) {
      s_base[0] = (total & 0xfffffu) ? atomicAdd(hs.state, total & 0xfffffu) : 0u;
      s_base[1] = (total >> 20) ? atomicAdd(hs.state + 1, total >> 20) : 0u;
    }
    __syncthreads();
    uint32_t cn = s_base[0] + (excl & 0xfffffu), ch = s_base[1] + (excl >> 20);
#pragma unroll
    for (int u = 0; u < HEAVY_LIST_BPT; u++) {
      if ((normal >> u) & 1u) {
        for (uint32_t x = off[u]; x < off[u + 1]; x += HEAVY_ITEM) {
          if (cn < hs.list_cap) hs.bucket[cn] = make_uint2(x, min(off[u + 1], x + HEAVY_ITEM));
          cn++;
        }
      } else if ((huge >> u) & 1u) {
        if (ch < HEAVY_HUGE_MAX) hs.huge[ch] = make_uint2(off[u], off[u + 1]);
        ch++;
      }
    }
    __syncthreads();  // s_base is rewritten by the next chunk
  }
}

// Inserts and counts the entries [first, x1) of A with stride `step`: a
// thread keeps a run (slot, copies) and adds it to the set when the slot
// changes; at the end the warp adds its runs (one add when every lane holds
// the same slot).  Four entries are loaded before any is looked up, and an
// entry equal to the previous one reuses its slot (a long bucket is mostly
// one key), so the loop waits on few dependent reads.  Called by whole warps.
template <typename KeyT>
__device__ __forceinline__ void heavy_count_range(const KeyT* __restrict__ a_keys, const HeavySet& hs, uint32_t first,
                                                  uint32_t x1, uint32_t step) {
  uint32_t run_slot = ~0u;
  unsigned long long run = 0;
  KeyT last_key = 0;
  uint32_t last_slot = ~0u;
  bool have_last = false;
  for (uint32_t x = first; x < x1; x += 4 * step) {
    KeyT k4[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t xu = x + u * step;
      k4[u] = xu < x1 ? a_keys[xu] : KeyT(0);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (x + u * step >= x1) break;
      uint32_t h;
      if (have_last && k4[u] == last_key) {
        h = last_slot;
      } else {
        h = heavy_insert(hs, k4[u]);
        last_key = k4[u];
        last_slot = h;
        have_last = true;
      }
      if (h != run_slot) {
        if (run) atomicAdd(hs.count_at(run_slot), run);
        run_slot = h;
        run = 0;
      }
      run += (h != ~0u);
    }
  }
  const uint32_t lead_slot = __shfl_sync(FULL_MASK, run_slot, 0);
  if (__all_sync(FULL_MASK, run_slot == lead_slot)) {
    run = warp_sum(run);
    if (lane_id() == 0 && run) atomicAdd(hs.count_at(lead_slot), run);
  } else if (run) {
    atomicAdd(hs.count_at(run_slot), run);
  }
}

// Listed items (pieces of the buckets of at most HEAVY_HUGE entries): one warp each.
template <typename KeyT>
__global__ void __launch_bounds__(256) k_heavy_count(const KeyT* __restrict__ a_keys, HeavySet hs,
                                                     const uint32_t* gate) {
  if (entry_skip(gate)) return;
  const uint32_t n_b = min(*reinterpret_cast<volatile unsigned*>(hs.state), hs.list_cap);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < n_b; c += warps) {
    // a set that found no slot for a key is not used: stop counting
    if (__any_sync(FULL_MASK, reinterpret_cast<volatile unsigned*>(hs.state)[3] != 0)) break;
    const uint2 bk = hs.bucket[c];
    heavy_count_range(a_keys, hs, bk.x + lane_id(), bk.y, 32u);
  }
}

// Listed buckets of more than HEAVY_HUGE entries: bucket c is cut into
// HEAVY_CHUNK-entry items, item j goes to CTA (c + j) mod grid, so a bucket of
// tens of millions of entries is shared by all CTAs.
template <typename KeyT, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_heavy_count_huge(const KeyT* __restrict__ a_keys, HeavySet hs,
                                                            const uint32_t* gate) {
  if (entry_skip(gate)) return;
  const uint32_t n_b = min(*reinterpret_cast<volatile unsigned*>(hs.state + 1), HEAVY_HUGE_MAX);
  const uint32_t grid = gridDim.x;
  // the list is read into shared memory BLOCK entries at a time, so the walk
  // over it waits on no global load per bucket
  __shared__ uint2 s_huge[BLOCK];
  bool stop = false;  // a key found no slot: the set is not used (the warp's lanes agree)
  for (uint32_t c0 = 0; c0 < n_b; c0 += BLOCK) {
    const uint32_t nb = min(uint32_t(BLOCK), n_b - c0);
    __syncthreads();  // the previous batch is read
    if (threadIdx.x < nb) s_huge[threadIdx.x] = hs.huge[c0 + threadIdx.x];
    __syncthreads();
    for (uint32_t c = c0; c < c0 + nb; c++) {
      const uint2 bk = s_huge[c - c0];
      const uint32_t chunks = (bk.y - bk.x + HEAVY_CHUNK - 1) / HEAVY_CHUNK;
      for (uint32_t j = (blockIdx.x + grid - c % grid) % grid; j < chunks; j += grid) {
        if (!stop) stop = __any_sync(FULL_MASK, reinterpret_cast<volatile unsigned*>(hs.state)[3] != 0);
        if (stop) continue;
        const uint32_t x0 = bk.x + j * HEAVY_CHUNK;
        heavy_count_range(a_keys, hs, x0 + threadIdx.x, min(bk.y, x0 + HEAVY_CHUNK), uint32_t(BLOCK));
      }
    }
  }
}

// Direct probe.  Persistent: CTAs take tiles of PROBE_TILE queries in ticket
// order (count-only tiles need no order and use the same loop).
template <typename KeyT, bool EMIT, bool A_IDX, bool Q_IDX>
__global__ void __launch_bounds__(PROBE_BLOCK)
    k_probe(const uint32_t* __restrict__ a_off, const KeyT* __restrict__ a_keys, const uint32_t* __restrict__ a_idx,
            BucketMap bm, const KeyT* __restrict__ q, uint64_t nq, const uint32_t* __restrict__ q_idx,
            uint32_t* __restrict__ pairs, uint64_t cap, unsigned long long* d_count, uint64_t* status,
            unsigned* ticket, const uint32_t* gate, HeavySet hs) {
  if (entry_skip(gate)) return;
  __shared__ uint64_t red[PROBE_BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
  __shared__ KeyT s_queue[EMIT ? 1 : PROBE_BLOCK / 32][EMIT ? 1 : 32 * PROBE_QPT];  // count only: per-warp queue
  const uint64_t ntiles = (nq + PROBE_TILE - 1) / PROBE_TILE;
  uint64_t counted = 0;
  while (true) {
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= ntiles) break;
    const uint64_t q0 = tile * PROBE_TILE + uint64_t(threadIdx.x) * PROBE_QPT;
    KeyT key[PROBE_QPT];
    uint32_t lo[PROBE_QPT], hi[PROBE_QPT];
    uint64_t c = 0;
#pragma unroll
    for (int j = 0; j < PROBE_QPT; j++) key[j] = q0 + j < nq ? __ldcs(q + q0 + j) : KeyT(0);
    if constexpr (!EMIT) {
      // count only.  A key a complete heavy-key set holds takes its count
      // from there and reads no bucket bounds.  The warp's other queries go
      // through a queue in shared memory and are then taken 32 at a time,
      // one per lane, so that the bucket work runs once per 32 such queries
      // rather than once per query slot of every lane.  For a key the set
      // does not hold, a long bucket of a complete set has no copy of it;
      // other buckets of COOP_MIN_LEN entries or more are scanned by the
      // whole warp, shorter ones by the lane.
      const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
      const bool complete = heavy_complete(hs);
      KeyT* queue = s_queue[warp];
      uint32_t n_q = 0;
#pragma unroll
      for (int j = 0; j < PROBE_QPT; j++) {
        bool need = q0 + j < nq;
        if (need && complete) {
          const uint32_t h = heavy_find(hs, key[j]);
          if (h != ~0u) {
            c += *hs.count_at(h);
            need = false;
          }
        }
        const unsigned b = __ballot_sync(FULL_MASK, need);
        if (need) queue[n_q + __popc(b & ((1u << lane) - 1u))] = key[j];
        n_q += __popc(b);
      }
      __syncwarp();
      for (uint32_t r = 0; r < n_q; r += 32) {
        const bool act = r + lane < n_q;
        const KeyT kq = act ? queue[r + lane] : KeyT(0);
        uint32_t lo = 0, hi = 0;
        if (act) {
          const uint32_t b = bm.of_key(kq);
          lo = a_off[b];
          hi = a_off[b + 1];
        }
        const uint32_t len = hi - lo;
        const bool absent = len >= HEAVY_MIN_LEN && complete && static_cast<unsigned long long>(kq) != ~0ull;
        const bool pend = !absent && len >= COOP_MIN_LEN;
        if (!absent && !pend)
          for (uint32_t x = lo; x < hi; x++) c += (a_keys[x] == kq);
        unsigned who = __ballot_sync(FULL_MASK, pend);
        while (who) {
          const int leader = __ffs(who) - 1;
          who &= who - 1;
          const KeyT kk = __shfl_sync(FULL_MASK, kq, leader);
          const uint32_t x0 = __shfl_sync(FULL_MASK, lo, leader), x1 = __shfl_sync(FULL_MASK, hi, leader);
          for (uint32_t x = x0 + lane; x < x1; x += 32) c += (a_keys[x] == kk);
        }
      }
      __syncwarp();  // the queue is refilled by the next tile
      counted += c;
      __syncthreads();
    } else {
#pragma unroll
      for (int j = 0; j < PROBE_QPT; j++) {
        lo[j] = hi[j] = 0;
        if (q0 + j < nq) {
          const uint32_t b = bm.of_key(key[j]);
          lo[j] = a_off[b];
          hi[j] = a_off[b + 1];
        }
      }
      // first bucket entries of all the thread's queries are loaded together
      KeyT first[PROBE_QPT];
#pragma unroll
      for (int j = 0; j < PROBE_QPT; j++) first[j] = lo[j] < hi[j] ? a_keys[lo[j]] : KeyT(0);
#pragma unroll
      for (int j = 0; j < PROBE_QPT; j++) {
        if (lo[j] < hi[j]) {
          c += (first[j] == key[j]);
          for (uint32_t x = lo[j] + 1; x < hi[j]; x++) c += (a_keys[x] == key[j]);
        }
      }
      uint64_t tile_total;
      const uint64_t excl = block_exclusive_scan<PROBE_BLOCK>(c, red, &tile_total);
      if (threadIdx.x < 32) {
        const uint64_t p = lookback_exclusive(status, tile, tile_total);
        if (threadIdx.x == 0) s_prefix = p;
      }
      __syncthreads();
      const uint64_t prefix = s_prefix;
      uint64_t pos = prefix + excl;
      if (c) {
#pragma unroll
        for (int j = 0; j < PROBE_QPT; j++) {
          const uint32_t qref = Q_IDX ? (q0 + j < nq ? q_idx[q0 + j] : 0u) : static_cast<uint32_t>(q0 + j);
          for (uint32_t x = lo[j]; x < hi[j]; x++) {
            if (a_keys[x] == key[j]) {
              if (pos < cap) {
                const uint32_t aref = A_IDX ? a_idx[x] : x;
                reinterpret_cast<uint2*>(pairs)[pos] = make_uint2(aref, qref);
              }
              pos++;
            }
          }
        }
      }
      if (threadIdx.x == 0 && tile == ntiles - 1) {
        const uint64_t total = prefix + tile_total;
        *d_count = total;
        if (total > cap) record_error(HG_ERR_PAIR_CAPACITY);
      }
      __syncthreads();
    }
  }
  if constexpr (!EMIT) {
    uint64_t tot;
    block_exclusive_scan<PROBE_BLOCK>(counted, red, &tot);
    if (threadIdx.x == 0 && tot) atomicAdd(d_count, static_cast<unsigned long long>(tot));
  }
}

// Pass 3 of the partitioned probe: one CTA per fine partition of W buckets.
// Both sides of the partition are staged in shared memory by bulk copies --
// A's offsets, keys (and index) for the W buckets, and the partition's
// queries with their positions -- and the next partition's copies are in
// flight while this one is probed.  A's ragged ends that are not 16-byte
// aligned are read with plain loads, so no copy touches memory outside A's
// arrays; an A slice that does not fit ("spill", heavy duplicates) is read
// from global memory instead.
//
// Each thread takes queries r = r0 + j*BLOCK + tid (j < FPROBE_QCH) and keeps,
// per query, its match count and the first match's reference in registers.
// One block scan of the thread totals and ONE atomic on the running pair
// count reserve the round's output range, then every thread writes its pairs
// straight from the registers (a query with several matches rescans its
// bucket).  A round covers FPROBE_QCH*BLOCK queries, so a partition normally
// takes one.
// Dynamic smem: [2] x { off[W+4] | keys[capa + 2*EPK] | idx[capa + 8] | qkeys[capq] | qidx[capq] }
constexpr int FPROBE_QCH = 5;

__host__ __device__ inline size_t fine_probe_buf_bytes(uint32_t fine_log2, uint32_t capa, uint64_t capq,
                                                       int key_bytes, bool a_idx, bool emit) {
  const size_t epk = 16 / key_bytes;
  auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
  return a16(((size_t(1) << fine_log2) + 4) * 4) + a16((capa + 2 * epk) * key_bytes) +
         (a_idx ? a16((size_t(capa) + 8) * 4) : 0) + a16(capq * key_bytes) + (emit ? a16(capq * 4) : 0);
}

// One pass-3 partition of a probe: its query slots, the table it probes and
// where its pairs go.
template <typename KeyT>
struct ProbePart {
  const KeyT* qk;               // the partition's query slots (keys, positions)
  const uint32_t* qi;
  uint64_t b0;                  // first bucket of the partition in the table
  uint32_t nb;                  // buckets of the partition
  BucketMap bm;
  uint64_t n_buckets;           // the table's
  const uint32_t* a_off;        // the table (a_idx may be NULL)
  const KeyT* a_keys;
  const uint32_t* a_idx;
  uint64_t n_a;
  bool a_bulk;                  // the table's arrays are 16-byte aligned
  uint32_t* pairs;
  uint64_t pair_cap;
  unsigned long long* d_count;
};

// Pass-3 partitions of one probe: partition f covers buckets [f*W, (f+1)*W)
// and its queries sit at slot f*capq.
template <typename KeyT>
struct TableProbe {
  static constexpr bool kOneTable = true;  // one count for the whole launch
  const KeyT* qkeys;
  const uint32_t* qidx;
  const uint32_t* qstart;
  uint64_t n_fine, capq;
  uint32_t fine_log2;
  BucketMap bm;
  uint64_t n_buckets;
  const uint32_t* a_off;
  const KeyT* a_keys;
  const uint32_t* a_idx;
  uint64_t n_a;
  bool a_bulk;
  uint32_t* pairs;
  uint64_t pair_cap;
  unsigned long long* d_count;
  __device__ __forceinline__ uint64_t count() const {
    return umin64(n_fine, (n_buckets + (1ull << fine_log2) - 1) >> fine_log2);
  }
  __device__ __forceinline__ uint2 meta(uint64_t f) const { return make_uint2(qstart[f], qstart[f + 1]); }
  __device__ __forceinline__ ProbePart<KeyT> at(uint64_t f) const {
    const uint64_t b0 = f << fine_log2;
    const uint32_t nb = static_cast<uint32_t>(umin64(1ull << fine_log2, n_buckets - b0));
    return ProbePart<KeyT>{qkeys + f * capq, qidx + f * capq, b0, nb, bm, n_buckets, a_off, a_keys, a_idx, n_a,
                           a_bulk, pairs, pair_cap, d_count};
  }
};

template <typename KeyT, bool A_IDX, bool EMIT, int BLOCK, typename Src>
__global__ void __launch_bounds__(BLOCK)
    k_fine_probe(Src src, uint64_t capq, uint32_t fine_log2, uint32_t capa, const uint32_t* flags) {
  if (entry_skip_on_overflow(flags)) return;
  constexpr uint32_t EPK = 16 / sizeof(KeyT);  // keys per 16 bytes
  constexpr uint32_t QCH = FPROBE_QCH;
  constexpr int NW = BLOCK / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t W = 1u << fine_log2;
  const size_t off_bytes = align_up_dev(size_t(W + 4) * 4, 16);
  const size_t key_bytes = align_up_dev(size_t(capa + 2 * EPK) * sizeof(KeyT), 16);
  const size_t idx_bytes = A_IDX ? align_up_dev(size_t(capa + 8) * 4, 16) : 0;
  const size_t qk_bytes = align_up_dev(capq * sizeof(KeyT), 16);
  const size_t buf_bytes = fine_probe_buf_bytes(fine_log2, capa, capq, sizeof(KeyT), A_IDX, EMIT);
  __shared__ uint64_t bar[2];
  // per buffer: A's range [as, ae), where the copied keys / index start
  // (al, ial) and end (ar, iar), plain offset loads still needed, the
  // partition's query count
  __shared__ uint32_t s_as[2], s_ae[2], s_al[2], s_ar[2], s_ial[2], s_iar[2], s_oplain[2], s_qm[2];
  __shared__ uint64_t red[NW + 1];
  const uint64_t n_live = src.count();
  auto buf_off = [&](uint32_t b) { return reinterpret_cast<uint32_t*>(smem_raw + b * buf_bytes); };
  auto buf_keys = [&](uint32_t b) { return reinterpret_cast<KeyT*>(smem_raw + b * buf_bytes + off_bytes); };
  auto buf_idx = [&](uint32_t b) {
    return reinterpret_cast<uint32_t*>(smem_raw + b * buf_bytes + off_bytes + key_bytes);
  };
  auto buf_q = [&](uint32_t b) {
    return reinterpret_cast<KeyT*>(smem_raw + b * buf_bytes + off_bytes + key_bytes + idx_bytes);
  };
  auto buf_qi = [&](uint32_t b) {
    return reinterpret_cast<uint32_t*>(smem_raw + b * buf_bytes + off_bytes + key_bytes + idx_bytes + qk_bytes);
  };
  struct Meta {
    uint32_t as, ae, qb, qe;
  };
  // thread 0: the partition's A range and queries (loaded one iteration early)
  auto load_meta = [&](uint64_t f) -> Meta {
    Meta mt{0, 0, 0, 0};
    if (f < n_live) {
      const ProbePart<KeyT> pp = src.at(f);
      mt.as = pp.a_off[pp.b0];
      mt.ae = pp.a_off[pp.b0 + pp.nb];
      const uint2 q = src.meta(f);
      mt.qb = q.x;
      mt.qe = q.y;
    }
    return mt;
  };
  // thread 0: start the bulk copies of partition f into buffer b.  A's
  // copies are rounded out to 16 bytes where that stays inside A's arrays;
  // only what cannot be covered that way is left to plain loads.  The
  // queries sit at the start of their 16-byte aligned slot (capq is a
  // multiple of 32), so their copies round up inside the slot.
  auto issue = [&](uint64_t f, uint32_t b, const Meta& mt) {
    const ProbePart<KeyT> pp = src.at(f);
    const uint64_t b0 = pp.b0, n_buckets = pp.n_buckets, n_a = pp.n_a;
    const uint32_t nb = pp.nb;
    const uint32_t* a_off = pp.a_off;
    const KeyT* a_keys = pp.a_keys;
    const uint32_t* a_idx = pp.a_idx;
    const uint32_t as = mt.as, ae = mt.ae;
    const bool fits = ae - as + 2 * EPK <= capa;
    uint32_t al = as, ar = as, ial = as, iar = as, ob = 0;
    if (pp.a_bulk) {
      // offsets: entries [0, nb] of the partition, rounded up within B + 1
      const uint64_t oend = umin64((b0 + nb + 1 + 3) & ~3ull, (n_buckets + 1) & ~3ull);
      ob = oend > b0 ? static_cast<uint32_t>((oend - b0) * 4) : 0u;
      if (fits) {
        al = as & ~(EPK - 1);
        ar = static_cast<uint32_t>(umin64((uint64_t(ae) + EPK - 1) & ~uint64_t(EPK - 1), n_a & ~uint64_t(EPK - 1)));
        if (ar < al) ar = al;
        if (A_IDX && a_idx) {
          ial = as & ~3u;
          iar = static_cast<uint32_t>(umin64((uint64_t(ae) + 3) & ~3ull, n_a & ~3ull));
          if (iar < ial) iar = ial;
        }
      }
    }
    uint32_t m = mt.qe - mt.qb;
    if (mt.qe < mt.qb || m > capq) {  // more queries than the partition's slots: bad device state
      record_fault(HG_ERR_DEVICE_STATE);
      m = 0;
    }
    s_as[b] = as;
    s_ae[b] = ae;
    s_al[b] = al;
    s_ar[b] = ar;
    s_ial[b] = ial;
    s_iar[b] = iar;
    s_oplain[b] = ob / 4;
    s_qm[b] = m;
    const uint32_t kb = (ar - al) * uint32_t(sizeof(KeyT));
    const uint32_t ib = (A_IDX && a_idx) ? (iar - ial) * 4u : 0u;
    const uint32_t qkb = (m * uint32_t(sizeof(KeyT)) + 15u) & ~15u;
    const uint32_t qib = EMIT ? ((m * 4u + 15u) & ~15u) : 0u;
    mbar_arrive_expect_tx(&bar[b], ob + kb + ib + qkb + qib);
    if (ob) bulk_g2s(buf_off(b), a_off + b0, ob, &bar[b]);
    if (kb) bulk_g2s(buf_keys(b), a_keys + al, kb, &bar[b]);
    if constexpr (A_IDX) {
      if (ib) bulk_g2s(buf_idx(b), a_idx + ial, ib, &bar[b]);
    }
    if (qkb) bulk_g2s(buf_q(b), pp.qk, qkb, &bar[b]);
    if constexpr (EMIT) {
      if (qib) bulk_g2s(buf_qi(b), pp.qi, qib, &bar[b]);
    }
  };
  Meta next_meta{};  // thread 0: metadata of the partition after the one in flight
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
    if (blockIdx.x < n_live) issue(blockIdx.x, 0, load_meta(blockIdx.x));
    next_meta = load_meta(blockIdx.x + gridDim.x);
  }
  __syncthreads();
  uint64_t counted = 0;
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;

  uint32_t it = 0;
  for (uint64_t f = blockIdx.x; f < n_live; f += gridDim.x, it++) {
    const uint32_t b = it & 1;
    const ProbePart<KeyT> pp = src.at(f);
    const uint64_t b0 = pp.b0;
    const uint32_t nb = pp.nb;
    const BucketMap bm = pp.bm;
    const uint32_t* a_off = pp.a_off;
    const KeyT* a_keys = pp.a_keys;
    const uint32_t* a_idx = pp.a_idx;
    uint32_t* pairs = pp.pairs;
    const uint64_t pair_cap = pp.pair_cap;
    unsigned long long* d_count = pp.d_count;
    if (threadIdx.x == 0) mbar_wait(&bar[b], (it >> 1) & 1);
    // the copy into buffer b landed (published by this barrier), and every
    // thread finished the previous partition, so buffer b ^ 1 is free
    __syncthreads();
    if (threadIdx.x == 0 && f + gridDim.x < n_live) {
      fence_proxy_async_smem();
      issue(f + gridDim.x, b ^ 1u, next_meta);
      next_meta = load_meta(f + 2 * uint64_t(gridDim.x));  // consumed next iteration
    }
    uint32_t* soff = buf_off(b);
    KeyT* sk = buf_keys(b);
    uint32_t* si = buf_idx(b);
    const uint32_t as = s_as[b], ae = s_ae[b], al = s_al[b], ar = s_ar[b];
    const bool spill = ae - as + 2 * EPK > capa;
    // whatever the bulk copies could not cover (the end of A's arrays, or
    // unaligned arrays): plain loads, rare, so the barrier is taken only then
    const uint32_t oplain = s_oplain[b];
    const bool plain = oplain <= nb || (!spill && (ar < ae || (A_IDX && a_idx && s_iar[b] < ae)));
    if (plain) {
      for (uint32_t j = oplain + threadIdx.x; j <= nb; j += BLOCK) soff[j] = a_off[b0 + j];
      if (!spill) {
        for (uint32_t x = ar + threadIdx.x; x < ae; x += BLOCK) sk[x - al] = a_keys[x];
        if (A_IDX && a_idx) {
          const uint32_t ial = s_ial[b], iar = s_iar[b];
          for (uint32_t x = iar + threadIdx.x; x < ae; x += BLOCK) si[x - ial] = a_idx[x];
        }
      }
      __syncthreads();
    }
    const uint32_t m = s_qm[b];
    const KeyT* sq = buf_q(b);
    const uint32_t* sqi = buf_qi(b);
    const uint32_t koff = as - al;  // sk[x + koff] is A's key at global position as + x
    uint32_t ioff = 0;
    if constexpr (A_IDX) ioff = as - s_ial[b];
    // SPILL: A's slice did not fit and is read in place from global memory
    auto probe_partition = [&](auto spill_c) {
      constexpr bool SPILL = decltype(spill_c)::value;
      auto a_key = [&](uint32_t x) -> KeyT {
        if constexpr (SPILL) return a_keys[as + x];
        else return sk[x + koff];
      };
      auto a_ref = [&](uint32_t x) -> uint32_t {
        if constexpr (A_IDX) {
          if (!a_idx) return as + x;  // a table without index: CSR positions
          if constexpr (SPILL) return a_idx[as + x];
          else return si[x + ioff];
        } else {
          return as + x;
        }
      };
      for (uint32_t r0 = 0; r0 < m; r0 += QCH * BLOCK) {
        uint32_t cnt[QCH], ref[QCH], xs[QCH], xe[QCH];
        KeyT kq[QCH];
#pragma unroll
        for (uint32_t j = 0; j < QCH; j++) {
          cnt[j] = ref[j] = xs[j] = xe[j] = 0;
          kq[j] = 0;
          if (r0 + j * BLOCK >= m) continue;  // uniform: chunk j holds no query
          const uint32_t r = r0 + j * BLOCK + threadIdx.x;
          if (r < m) {
            kq[j] = sq[r];
            const uint32_t lb = static_cast<uint32_t>(bm.of_key(kq[j]) - b0);
            xs[j] = soff[lb] - as;
            xe[j] = soff[lb + 1] - as;
          }
        }
        // walk the thread's buckets side by side: the warp runs as many steps
        // as its longest bucket, not the sum of every query's longest
        for (bool more = true; more;) {
          more = false;
#pragma unroll
          for (uint32_t j = 0; j < QCH; j++) {
            if (xs[j] < xe[j]) {
              const uint32_t x = xs[j]++;
              if (a_key(x) == kq[j]) {
                if (cnt[j] == 0) ref[j] = a_ref(x);
                cnt[j]++;
              }
              more |= xs[j] < xe[j];
            }
          }
        }
        uint64_t mine = 0;
#pragma unroll
        for (uint32_t j = 0; j < QCH; j++) mine += cnt[j];
        if constexpr (!EMIT) {
          if constexpr (Src::kOneTable) {
            counted += mine;
          } else {  // partitions of several tables: one count per partition
            uint64_t tot;
            block_exclusive_scan<BLOCK>(mine, red, &tot);
            if (threadIdx.x == 0 && tot) atomicAdd(d_count, static_cast<unsigned long long>(tot));
          }
        } else {
          // block scan of the thread totals; warp 0 reserves the round's range
          const uint64_t inc = warp_inclusive_scan(mine);
          if (lane == 31) red[warp] = inc;
          __syncthreads();
          if (warp == 0) {
            const uint64_t w = lane < NW ? red[lane] : 0ull;
            const uint64_t wi = warp_inclusive_scan(w);
            const uint64_t tot = __shfl_sync(FULL_MASK, wi, NW - 1);
            uint64_t base = 0;
            if (lane == 0 && tot) {
              base = atomicAdd(d_count, static_cast<unsigned long long>(tot));
              if (pairs && base + tot > pair_cap) record_error(HG_ERR_PAIR_CAPACITY);
            }
            base = __shfl_sync(FULL_MASK, base, 0);
            if (lane < NW) red[lane] = base + wi - w;
          }
          __syncthreads();
          uint64_t pos = red[warp] + inc - mine;
          if (mine) {
            uint2* out = reinterpret_cast<uint2*>(pairs);
#pragma unroll
            for (uint32_t j = 0; j < QCH; j++) {
              if (r0 + j * BLOCK >= m) continue;
              const uint32_t r = r0 + j * BLOCK + threadIdx.x;
              if (cnt[j] == 1) {
                if (pos < pair_cap) out[pos] = make_uint2(ref[j], sqi[r]);
                pos++;
              } else if (cnt[j] > 1) {
                const KeyT k = sq[r];
                const uint32_t qref = sqi[r];
                const uint32_t lb = static_cast<uint32_t>(bm.of_key(k) - b0);
                const uint32_t e = soff[lb + 1] - as;
                for (uint32_t x = soff[lb] - as; x < e; x++) {
                  if (a_key(x) == k) {
                    if (pos < pair_cap) out[pos] = make_uint2(a_ref(x), qref);
                    pos++;
                  }
                }
              }
            }
          }
          if (r0 + QCH * BLOCK < m) __syncthreads();  // red is rewritten by the next round
        }
      }
    };
    if (spill) probe_partition(std::true_type{});
    else probe_partition(std::false_type{});
  }
  if constexpr (!EMIT && Src::kOneTable) {
    uint64_t tot;
    block_exclusive_scan<BLOCK>(counted, red, &tot);
    if (threadIdx.x == 0 && tot) atomicAdd(src.d_count, static_cast<unsigned long long>(tot));
  }
}

// The coarse probe: pass 1 has grouped the queries (with their positions) by
// bucket range; CTAs take tiles of CPROBE_BLOCK * QPT queries in range order
// from a ticket, so at any time they all read the table slices of two or
// three ranges, which stay in L2 (each slice comes from HBM once).  Each
// thread probes QPT queries side by side: bucket bounds, then the first
// entries of all its buckets, then the rest of each bucket, keeping the count
// and the first match in registers.  One block scan and ONE atomic on the
// pair count reserve a tile's output; pairs come out grouped by tile (no
// query order).  The kernel waits on L2 reads (bucket bounds and entries,
// about two sectors per query), not on HBM.
constexpr int CPROBE_BLOCK = 128;  // 256 / 512 / 1024 measured slower (3.10, 3.50, 3.75 ms against 3.00 at 2^28)

template <typename KeyT, bool EMIT, bool A_IDX, int QPT>
__global__ void __launch_bounds__(CPROBE_BLOCK)
    k_coarse_probe(const KeyT* __restrict__ pkeys, const uint32_t* __restrict__ pidx,
                   const uint32_t* __restrict__ pcount, uint32_t n_parts, uint64_t part_cap, Div32 tpp,
                   const uint32_t* __restrict__ a_off, const KeyT* __restrict__ a_keys,
                   const uint32_t* __restrict__ a_idx, BucketMap bm, uint32_t* __restrict__ pairs, uint64_t pair_cap,
                   unsigned long long* d_count, unsigned* ticket, const uint32_t* flags) {
  if (entry_skip_on_overflow(flags)) return;
  constexpr int NW = CPROBE_BLOCK / 32;
  constexpr uint32_t TILE = uint32_t(CPROBE_BLOCK) * QPT;
  __shared__ uint64_t red[NW + 1];
  __shared__ unsigned s_vt[3];
  const uint32_t tiles_per_part = tpp.d;
  const uint64_t vtiles = uint64_t(n_parts) * tiles_per_part;  // below 2^32 (the planner keeps it so)
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  auto a_ref = [&](uint32_t x) -> uint32_t {
    if constexpr (A_IDX) return a_idx[x];
    else return x;
  };
  // 128-byte lines of one tile's query keys (and positions, when emitting)
  constexpr uint32_t KEY_LINES = TILE * sizeof(KeyT) / 128, POS_LINES = EMIT ? TILE * 4 / 128 : 0;
  static_assert(KEY_LINES + POS_LINES <= CPROBE_BLOCK, "one prefetch per thread");
  uint64_t counted = 0;
  // tickets are taken a tile ahead: iteration i probes s_vt[i % 3] while its
  // first KEY_LINES + POS_LINES threads prefetch the query lines of the next
  // tile (s_vt[(i + 1) % 3]) into L2, and thread 0 takes the ticket after
  // that; the barrier that closes a tile publishes the ticket taken in it
  if (threadIdx.x == 0) {
    s_vt[0] = atomicAdd(ticket, 1u);
    s_vt[1] = atomicAdd(ticket, 1u);
  }
  __syncthreads();
  uint32_t cur = 0;  // it % 3
  for (uint32_t it = 0;; it++) {
    const uint64_t vt = s_vt[cur];
    if (vt >= vtiles) break;
    const uint32_t nxt = cur == 2 ? 0 : cur + 1;
    if (threadIdx.x == 0) s_vt[nxt == 2 ? 0 : nxt + 1] = atomicAdd(ticket, 1u);
    if (threadIdx.x < KEY_LINES + POS_LINES) {
      const uint32_t vt2 = s_vt[nxt];
      if (vt2 < vtiles) {
        const uint32_t p2 = tpp.div(vt2);
        const uint32_t line = threadIdx.x < KEY_LINES ? threadIdx.x : threadIdx.x - KEY_LINES;
        const uint64_t e = uint64_t(vt2 - p2 * tiles_per_part) * TILE +
                           line * (threadIdx.x < KEY_LINES ? 128 / sizeof(KeyT) : 32);
        if (e < part_cap) {  // a line that starts inside the partition's slots
          const void* a = threadIdx.x < KEY_LINES ? static_cast<const void*>(pkeys + uint64_t(p2) * part_cap + e)
                                                  : static_cast<const void*>(pidx + uint64_t(p2) * part_cap + e);
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
        }
      }
    }
    cur = nxt;
    const uint32_t part32 = tpp.div(static_cast<uint32_t>(vt));
    const uint64_t part = part32;
    const uint32_t r0 = (static_cast<uint32_t>(vt) - part32 * tiles_per_part) * TILE;
    const uint32_t m = pcount[part];
    if (r0 >= m) {  // the same for the whole CTA
      __syncthreads();
      continue;
    }
    const KeyT* qk = pkeys + part * part_cap;
    const uint32_t* qi = pidx + part * part_cap;
    KeyT key[QPT];
    uint32_t lo[QPT], hi[QPT];
#pragma unroll
    for (int j = 0; j < QPT; j++) {
      const uint32_t r = r0 + j * CPROBE_BLOCK + threadIdx.x;
      key[j] = r < m ? __ldcs(qk + r) : KeyT(0);
    }
#pragma unroll
    for (int j = 0; j < QPT; j++) {
      const uint32_t r = r0 + j * CPROBE_BLOCK + threadIdx.x;
      lo[j] = hi[j] = 0;
      if (r < m) {
        const uint32_t b = bm.of_key(key[j]);
        lo[j] = a_off[b];
        hi[j] = a_off[b + 1];
      }
    }
    KeyT first[QPT];
#pragma unroll
    for (int j = 0; j < QPT; j++) first[j] = lo[j] < hi[j] ? a_keys[lo[j]] : KeyT(0);
    uint32_t cnt[QPT], ref[QPT];
    uint64_t mine = 0;
#pragma unroll
    for (int j = 0; j < QPT; j++) {
      cnt[j] = 0;
      ref[j] = 0;
      if (lo[j] < hi[j]) {
        if (first[j] == key[j]) {
          cnt[j] = 1;
          if constexpr (EMIT) ref[j] = a_ref(lo[j]);
        }
        for (uint32_t x = lo[j] + 1; x < hi[j]; x++) {
          if (a_keys[x] == key[j]) {
            if constexpr (EMIT) {
              if (cnt[j] == 0) ref[j] = a_ref(x);
            }
            cnt[j]++;
          }
        }
      }
      mine += cnt[j];
    }
    if constexpr (!EMIT) {
      counted += mine;
      __syncthreads();
    } else {
      const uint64_t inc = warp_inclusive_scan(mine);
      if (lane == 31) red[warp] = inc;
      __syncthreads();
      if (warp == 0) {
        const uint64_t w = lane < NW ? red[lane] : 0ull;
        const uint64_t wi = warp_inclusive_scan(w);
        const uint64_t tot = __shfl_sync(FULL_MASK, wi, NW - 1);
        uint64_t base = 0;
        if (lane == 0 && tot) {
          base = atomicAdd(d_count, static_cast<unsigned long long>(tot));
          if (base + tot > pair_cap) record_error(HG_ERR_PAIR_CAPACITY);
        }
        base = __shfl_sync(FULL_MASK, base, 0);
        if (lane < NW) red[lane] = base + wi - w;
      }
      __syncthreads();
      uint64_t pos = red[warp] + inc - mine;
      __syncwarp();  // the warp's lane 31 rewrites red[warp] in the next tile
      if (mine) {
        uint2* out = reinterpret_cast<uint2*>(pairs);
#pragma unroll
        for (int j = 0; j < QPT; j++) {
          if (cnt[j] == 0) continue;
          const uint32_t qref = qi[r0 + j * CPROBE_BLOCK + threadIdx.x];
          if (cnt[j] == 1) {
            if (pos < pair_cap) out[pos] = make_uint2(ref[j], qref);
            pos++;
          } else {
            for (uint32_t x = lo[j]; x < hi[j]; x++) {
              if (a_keys[x] == key[j]) {
                if (pos < pair_cap) out[pos] = make_uint2(a_ref(x), qref);
                pos++;
              }
            }
          }
        }
      }
    }
  }
  if constexpr (!EMIT) {
    uint64_t tot;
    block_exclusive_scan<CPROBE_BLOCK>(counted, red, &tot);
    if (threadIdx.x == 0 && tot) atomicAdd(d_count, static_cast<unsigned long long>(tot));
  }
}

size_t fine_probe_smem(uint32_t fine_log2, uint32_t capa, uint64_t capq, int key_bytes, bool a_idx, bool emit) {
  return 2 * fine_probe_buf_bytes(fine_log2, capa, capq, key_bytes, a_idx, emit);
}

// Shared-memory budget of one fine-probe CTA (tuning override HG_PROBE_SMEM_KB).
static size_t probe_smem_budget() {
  if (const char* e = std::getenv("HG_PROBE_SMEM_KB")) {
    const int kb = std::atoi(e);
    if (kb >= 16 && kb <= 220) return size_t(kb) * 1024;
  }
  return FINE_PROBE_SMEM_BUDGET;
}

// Bucket ranges of the coarse probe: the widest power of two of buckets whose
// slice of the table (4-byte offsets + records at the table's mean density)
// fits the L2 budget, so the CTAs, which take the ranges in order, find the
// slice they read in L2; at least 16 ranges, so small tables exercise the
// form too.  The budget leaves room in the 126 MB L2 for the two or three
// ranges in flight at once (tuning override HG_L2_SLICE_MB).
static bool plan_coarse(uint64_t nq, uint64_t n_a, size_t a_rec, uint64_t n_buckets, int key_bytes,
                        PartGeometry* out) {
  double budget = double(COARSE_SLICE_BUDGET);
  if (const char* e = std::getenv("HG_L2_SLICE_MB")) {
    const int mb = std::atoi(e);
    if (mb >= 1 && mb <= 120) budget = double(mb) * 1048576.0;
  }
  const double per_bucket = 4.0 + double(a_rec) * double(n_a) / double(n_buckets);
  uint32_t c = 0;
  while (c < 32 && double(1ull << (c + 1)) * per_bucket <= budget) c++;
  while (c > 0 && ((n_buckets + (1ull << c) - 1) >> c) < 16) c--;
  // pass 1 slows down sharply above PASS1_GOOD_PARTS ranges (2^31 buckets of
  // u32 + index: 1024 ranges 14.1 ms, 512 ranges 8.4 ms); wider slices cost
  // the probe little (3 to 48 MB within 4% at 2^28)
  while (c < 32 && ((n_buckets + (1ull << c) - 1) >> c) > PASS1_GOOD_PARTS) c++;
  PartGeometry g;
  g.coarse_log2 = c;
  g.n_parts = (n_buckets + (1ull << c) - 1) >> c;
  if (g.n_parts > PASS1_MAX_PARTS) return false;
  g.part_cap = slack_capacity(double(nq) * double(std::min<uint64_t>(1ull << c, n_buckets)) / double(n_buckets), 256);
  if (g.part_cap >= (1ull << 32)) return false;
  g.tile1 = pass1_tile(key_bytes);
  g.smem1 = pass1_smem(g.n_parts, key_bytes, g.tile1);
  if (g.smem1 > SMEM_BUDGET) return false;
  *out = g;
  return true;
}

hg_status plan_probe(uint64_t n_a, bool a_idx, uint64_t n_buckets, uint64_t nq, int key_bytes, bool emit,
                     ProbePlan* plan, int force_path) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0) return HG_ERR_INVALID_ARGUMENT;
  if (nq >= (1ull << 32) || n_a >= (1ull << 32) || n_buckets > (1ull << 32)) return HG_ERR_TOO_LARGE;
  ProbePlan p;
  p.n_a = n_a;
  p.nq = nq;
  p.n_buckets = n_buckets;
  p.key_bytes = key_bytes;
  p.a_idx = a_idx;
  p.emit = emit;
  p.tiles = (nq + PROBE_TILE - 1) / PROBE_TILE;
  const size_t a_rec = key_bytes + (a_idx ? 4 : 0);
  const size_t q_rec = key_bytes + 4;  // queries travel with their position
  // pass 3 double-buffers A's slice (offsets, keys, index) and the
  // partition's queries (keys, and positions when pairs are emitted)
  bool part_ok = plan_geometry(nq, q_rec, n_a, 2 * a_rec, 8, 2 * (key_bytes + (emit ? 4 : 0)), n_buckets, true,
                               &p.g, probe_smem_budget());
  if (part_ok) {
    p.g.tile1 = pass1_tile(key_bytes);
    p.g.smem1 = pass1_smem(p.g.n_parts, key_bytes, p.g.tile1);
    plan_split(p.g, key_bytes, true);
    p.g.smem3 = fine_probe_smem(p.g.fine_log2, p.g.smem_cap, p.g.fine_cap, key_bytes, a_idx, emit);
    part_ok = p.g.smem1 <= SMEM_BUDGET && p.g.smem2 <= SMEM_BUDGET && p.g.smem3 <= SMEM_BUDGET;
  }
  PartGeometry cg;
  const bool coarse_ok = plan_coarse(nq, n_a, a_rec, n_buckets, key_bytes, &cg);
  const uint64_t a_bytes = n_a * a_rec + 4 * n_buckets;
  int path = force_path;
  if (path < 0) {
    const bool big = a_bytes > (64ull << 20) && nq >= (1ull << 20);
    path = !big ? PROBE_DIRECT : coarse_ok ? PROBE_COARSE : part_ok ? PROBE_PARTITIONED : PROBE_DIRECT;
  }
  // Too few buckets to split the queries finely (everything in a handful of
  // buckets): the direct probe, even when the partitioned one is asked for.
  if (path == PROBE_PARTITIONED && !part_ok) path = PROBE_DIRECT;
  if (path == PROBE_COARSE && !coarse_ok) path = PROBE_DIRECT;
  if (path != PROBE_DIRECT && path != PROBE_PARTITIONED && path != PROBE_COARSE) return HG_ERR_INVALID_ARGUMENT;
  if (path == PROBE_COARSE) p.g = cg;
  p.path = path;
  size_t off = 0;
  p.off_status = off;  off = align_up(off + (emit ? p.tiles * 8 : 0));
  p.off_ticket = off;  off = align_up(off + 4 * sizeof(unsigned));
  p.off_flags = off;   off = align_up(off + sizeof(uint32_t));
  // count only: the heavy-key set of the direct probe (zeroed with the counters)
  p.off_heavy = off;   off = align_up(off + (emit ? 0 : heavy_bytes(n_a)));
  if (path == PROBE_PARTITIONED) {
    const PartGeometry& g = p.g;
    p.off_pcount = off;  off = align_up(off + (g.n_parts + 1) * 4);
    p.off_pstatus = off; off = align_up(off + g.pscan_tiles * 8);
    p.off_fcount = off;  off = align_up(off + (g.n_fine + 1) * 4);
    p.off_fstatus = off; off = align_up(off + g.fscan_tiles * 8);
    p.off_pkeys = off;   off = align_up(off + g.n_parts * g.part_cap * key_bytes);
    p.off_pidx = off;    off = align_up(off + g.n_parts * g.part_cap * 4);
    p.off_fkeys = off;   off = align_up(off + g.n_fine * g.fine_cap * key_bytes);
    p.off_fidx = off;    off = align_up(off + g.n_fine * g.fine_cap * 4);
  } else if (path == PROBE_COARSE) {
    const PartGeometry& g = p.g;
    p.off_pcount = off;  off = align_up(off + (g.n_parts + 1) * 4);
    p.off_pstatus = p.off_fcount = p.off_fstatus = off;
    p.off_pkeys = off;   off = align_up(off + g.n_parts * g.part_cap * key_bytes);
    p.off_pidx = off;    off = align_up(off + g.n_parts * g.part_cap * 4);
    p.off_fkeys = p.off_fidx = off;
  } else {
    p.off_pcount = p.off_pstatus = p.off_fcount = p.off_fstatus = off;
    p.off_pkeys = p.off_pidx = p.off_fkeys = p.off_fidx = off;
  }
  p.total = off;
  *plan = p;
  return HG_OK;
}

static HeavySet heavy_set(const ProbePlan& p, char* ws) {
  HeavySet hs{nullptr, nullptr, nullptr, nullptr, 0u, 0u};
  if (p.emit) return hs;
  const size_t slots = heavy_slots(p.n_a), cap = heavy_list_cap(p.n_a);
  char* h = ws + p.off_heavy;
  hs.slot = reinterpret_cast<unsigned long long*>(h);
  hs.bucket = reinterpret_cast<uint2*>(h + slots * 16);
  hs.huge = reinterpret_cast<uint2*>(h + slots * 16 + cap * 8);
  hs.state = reinterpret_cast<unsigned*>(h + slots * 16 + cap * 8 + size_t(HEAVY_HUGE_MAX) * 8);
  hs.mask = static_cast<uint32_t>(slots - 1);
  hs.list_cap = static_cast<uint32_t>(cap);
  return hs;
}

template <typename KeyT, bool EMIT>
static void launch_probe_direct(const ProbePlan& p, const uint32_t* a_off, const KeyT* a_keys, const uint32_t* a_idx,
                                const KeyT* q, const uint32_t* q_idx, uint32_t* pairs, uint64_t cap,
                                unsigned long long* d_count, uint64_t* status, unsigned* ticket, const uint32_t* gate,
                                HeavySet hs, cudaStream_t s) {
  const BucketMap bm = p.bucket_map();
  if constexpr (!EMIT) {
    // the heavy keys of A (their set was zeroed with the workspace)
    if (p.n_a > 0 && hs.slot != nullptr) {
      Phase ph(s, gate ? "fallback_heavy_keys" : "heavy_keys");
      count_launch();
      k_heavy_find<KeyT><<<HEAVY_SAMPLES / 256, 256, 0, s>>>(a_off, a_keys, p.n_a, bm, hs, gate);
      const unsigned grid = static_cast<unsigned>(device_sm_count()) * 8;  // 8 resident 256-thread CTAs per SM
      count_launch();
      constexpr uint64_t LIST_CHUNK = uint64_t(HEAVY_LIST_BLOCK) * HEAVY_LIST_BPT;
      k_heavy_list<<<static_cast<unsigned>(std::min<uint64_t>((p.n_buckets + LIST_CHUNK - 1) / LIST_CHUNK,
                                                              uint64_t(grid) * 2)),
                     HEAVY_LIST_BLOCK, 0, s>>>(a_off, p.n_buckets, hs, gate);
      count_launch();
      k_heavy_count<KeyT><<<grid, 256, 0, s>>>(a_keys, hs, gate);
      count_launch();
      k_heavy_count_huge<KeyT, 256><<<grid, 256, 0, s>>>(a_keys, hs, gate);
    }
  }
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(p.tiles, uint64_t(device_sm_count()) * 8));
  Phase ph(s, gate ? (EMIT ? "fallback_probe_emit" : "fallback_probe_count") : (EMIT ? "probe_emit" : "probe_count"));
  count_launch();
#define HG_PROBE_LAUNCH(AI, QI)                                                                            \
  k_probe<KeyT, EMIT, AI, QI><<<grid, PROBE_BLOCK, 0, s>>>(a_off, a_keys, a_idx, bm, q, p.nq, q_idx, pairs, \
                                                          cap, d_count, status, ticket, gate, hs)
  if (a_idx) {
    if (q_idx) HG_PROBE_LAUNCH(true, true); else HG_PROBE_LAUNCH(true, false);
  } else {
    if (q_idx) HG_PROBE_LAUNCH(false, true); else HG_PROBE_LAUNCH(false, false);
  }
#undef HG_PROBE_LAUNCH
}

template <typename KeyT, bool EMIT>
static hg_status run_probe_partitioned(const ProbePlan& p, const uint32_t* a_off, const KeyT* a_keys,
                                       const uint32_t* a_idx, const KeyT* q, const uint32_t* q_idx, uint32_t* pairs,
                                       uint64_t cap, unsigned long long* d_count, char* ws, cudaStream_t s) {
  const BucketMap bm = p.bucket_map();
  const PartGeometry& g = p.g;
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + p.off_flags);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  uint64_t* status = reinterpret_cast<uint64_t*>(ws + p.off_status);
  HG_CUDA(cudaMemsetAsync(ws, 0, p.off_pkeys, s), "intersect: workspace memset");
  // queries on a 16-byte boundary are streamed with bulk (TMA) copies
  const bool aligned = (reinterpret_cast<uintptr_t>(q) & 15u) == 0;
  hg_status st = aligned ? run_partition_passes<KeyT, 16 / sizeof(KeyT), true>(
                               g, p.nq, q, q_idx, bm, ws, p.off_flags, p.off_ticket, p.off_pcount, p.off_pstatus,
                               p.off_fcount, p.off_fstatus, p.off_pkeys, p.off_pidx, p.off_fkeys, p.off_fidx, "probe", s)
                         : run_partition_passes<KeyT, 1, true>(g, p.nq, q, q_idx, bm, ws, p.off_flags, p.off_ticket,
                                                               p.off_pcount, p.off_pstatus, p.off_fcount,
                                                               p.off_fstatus, p.off_pkeys, p.off_pidx, p.off_fkeys,
                                                               p.off_fidx, "probe", s);
  if (st != HG_OK) return st;
  {
    const bool a_bulk = ((reinterpret_cast<uintptr_t>(a_off) | reinterpret_cast<uintptr_t>(a_keys) |
                          reinterpret_cast<uintptr_t>(a_idx)) & 15u) == 0;
    using Src = TableProbe<KeyT>;
    const Src src{reinterpret_cast<const KeyT*>(ws + p.off_fkeys), reinterpret_cast<const uint32_t*>(ws + p.off_fidx),
                  reinterpret_cast<const uint32_t*>(ws + p.off_fcount), g.n_fine, g.fine_cap, g.fine_log2, bm,
                  p.n_buckets, a_off, a_keys, a_idx, p.n_a, a_bulk, pairs, cap, d_count};
    auto go = [&](auto kern, unsigned block) {
      const int bps = blocks_per_sm(kern, block, g.smem3);
      if (bps <= 0) {
        st = lib_fail(HG_ERR_CUDA, "fine-probe kernel cannot be resident");
        return;
      }
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(g.n_fine, uint64_t(device_sm_count()) * bps));
      Phase ph(s, EMIT ? "fine_probe_emit" : "fine_probe_count");
      count_launch();
      kern<<<std::max(grid, 1u), block, g.smem3, s>>>(src, g.fine_cap, g.fine_log2, g.smem_cap,
                                                      static_cast<const uint32_t*>(flags));
      const cudaError_t e = cudaPeekAtLastError();
      if (e != cudaSuccess) st = cuda_fail(e, "fine-probe launch");
    };
    // tuning override: HG_PROBE_BLOCK=512 runs the fine probe with 512 threads per CTA
    const char* pb = std::getenv("HG_PROBE_BLOCK");
    if (pb && std::atoi(pb) == 512) {
      if (a_idx) go(k_fine_probe<KeyT, true, EMIT, 512, Src>, 512u);
      else go(k_fine_probe<KeyT, false, EMIT, 512, Src>, 512u);
    } else {
      if (a_idx) go(k_fine_probe<KeyT, true, EMIT, FINE_PROBE_BLOCK, Src>, unsigned(FINE_PROBE_BLOCK));
      else go(k_fine_probe<KeyT, false, EMIT, FINE_PROBE_BLOCK, Src>, unsigned(FINE_PROBE_BLOCK));
    }
    if (st != HG_OK) return st;
  }
  // Fallback when a query partition overflowed (heavy duplicates): the direct
  // probe, gated on the flag.
  launch_probe_direct<KeyT, EMIT>(p, a_off, a_keys, a_idx, q, q_idx, pairs, cap, d_count, status, ticket, flags,
                                  heavy_set(p, ws), s);
  return HG_OK;
}

template <typename KeyT, bool EMIT>
static hg_status run_probe_coarse(const ProbePlan& p, const uint32_t* a_off, const KeyT* a_keys, const uint32_t* a_idx,
                                  const KeyT* q, const uint32_t* q_idx, uint32_t* pairs, uint64_t cap,
                                  unsigned long long* d_count, char* ws, cudaStream_t s) {
  const BucketMap bm = p.bucket_map();
  const PartGeometry& g = p.g;
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + p.off_flags);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  uint64_t* status = reinterpret_cast<uint64_t*>(ws + p.off_status);
  uint32_t* pcount = reinterpret_cast<uint32_t*>(ws + p.off_pcount);
  KeyT* pkeys = reinterpret_cast<KeyT*>(ws + p.off_pkeys);
  uint32_t* pidx = reinterpret_cast<uint32_t*>(ws + p.off_pidx);
  HG_CUDA(cudaMemsetAsync(ws, 0, p.off_pkeys, s), "intersect: workspace memset");
  const bool aligned = (reinterpret_cast<uintptr_t>(q) & 15u) == 0;
  hg_status st = aligned ? launch_pass1<KeyT, 16 / sizeof(KeyT), true>(g, p.nq, q, q_idx, bm, pcount, pkeys, pidx,
                                                                       flags, "probe_multisplit", s)
                         : launch_pass1<KeyT, 1, true>(g, p.nq, q, q_idx, bm, pcount, pkeys, pidx, flags,
                                                       "probe_multisplit", s);
  if (st != HG_OK) return st;
  {
    // queries per thread (tuning override HG_CPROBE_QPT = 1 or 2): fewer
    // queries per thread keep more warps resident, which hides the L2 latency
    // of the bucket reads better (2^28 u64 with pairs: 8 -> 4.94 ms, 4 ->
    // 3.85, 2 -> 3.36, 1 -> 3.84)
    int qpt = 2;
    const int block = CPROBE_BLOCK;
    if (const char* e = std::getenv("HG_CPROBE_QPT")) {
      const int v = std::atoi(e);
      qpt = v == 1 ? 1 : 2;
    }
    const uint32_t tiles_per_part =
        static_cast<uint32_t>((g.part_cap + uint64_t(block) * qpt - 1) / (uint64_t(block) * qpt));
    const uint64_t vtiles = g.n_parts * tiles_per_part;
    auto go = [&](auto kern) {
      const int bps = blocks_per_sm(kern, block, 0);
      if (bps <= 0) {
        st = lib_fail(HG_ERR_CUDA, "coarse-probe kernel cannot be resident");
        return;
      }
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(vtiles, uint64_t(device_sm_count()) * bps));
      Phase ph(s, EMIT ? "coarse_probe_emit" : "coarse_probe_count");
      count_launch();
      kern<<<std::max(grid, 1u), block, 0, s>>>(pkeys, pidx, pcount, static_cast<uint32_t>(g.n_parts),
                                                       g.part_cap, Div32::make(tiles_per_part), a_off, a_keys, a_idx, bm, pairs,
                                                       cap, d_count, ticket + 3, flags);
      const cudaError_t e = cudaPeekAtLastError();
      if (e != cudaSuccess) st = cuda_fail(e, "coarse-probe launch");
    };
    auto pick = [&](auto qpt_c) {
      constexpr int Q = decltype(qpt_c)::value;
      if (a_idx) go(k_coarse_probe<KeyT, EMIT, true, Q>);
      else go(k_coarse_probe<KeyT, EMIT, false, Q>);
    };
    if (qpt == 1) pick(std::integral_constant<int, 1>{});
    else pick(std::integral_constant<int, 2>{});
    if (st != HG_OK) return st;
  }
  // Fallback when a query range overflowed its slots (heavy duplicates): the
  // direct probe, gated on the flag.
  launch_probe_direct<KeyT, EMIT>(p, a_off, a_keys, a_idx, q, q_idx, pairs, cap, d_count, status, ticket, flags,
                                  heavy_set(p, ws), s);
  return HG_OK;
}

hg_status launch_probe(const ProbePlan& p, const uint32_t* a_off, const void* a_keys, const uint32_t* a_idx,
                       const void* q_keys, const uint32_t* q_idx, uint32_t* pairs, uint64_t pair_cap,
                       unsigned long long* d_count, void* d_ws, cudaStream_t s) {
  char* ws = static_cast<char*>(d_ws);
  uint64_t* status = reinterpret_cast<uint64_t*>(ws + p.off_status);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  HG_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s), "intersect: count memset");
  if (p.nq == 0) return HG_OK;
  const bool emit = p.emit && pairs != nullptr;
  hg_status st = HG_OK;
  auto run = [&](auto key_tag) {
    using KeyT = decltype(key_tag);
    auto ak = static_cast<const KeyT*>(a_keys);
    auto qk = static_cast<const KeyT*>(q_keys);
    if (p.path == PROBE_PARTITIONED) {
      st = emit ? run_probe_partitioned<KeyT, true>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, ws, s)
                : run_probe_partitioned<KeyT, false>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, ws, s);
      return;
    }
    if (p.path == PROBE_COARSE) {
      st = emit ? run_probe_coarse<KeyT, true>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, ws, s)
                : run_probe_coarse<KeyT, false>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, ws, s);
      return;
    }
    const cudaError_t e = cudaMemsetAsync(ws, 0, p.total, s);
    if (e != cudaSuccess) { st = cuda_fail(e, "intersect: workspace memset"); return; }
    if (emit)
      launch_probe_direct<KeyT, true>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, status, ticket, nullptr,
                                      heavy_set(p, ws), s);
    else
      launch_probe_direct<KeyT, false>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, status, ticket,
                                       nullptr, heavy_set(p, ws), s);
  };
  if (p.key_bytes == 4) run(uint32_t{});
  else run(uint64_t{});
  if (st != HG_OK) return st;
  HG_CUDA(cudaPeekAtLastError(), "intersect: kernel launch");
  return HG_OK;
}

}  // namespace hg
