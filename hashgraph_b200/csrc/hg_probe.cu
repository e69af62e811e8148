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
// pass: each tile of queries counts its matches, takes its output offset from
// the decoupled look-back over tiles, and writes its pairs in query order.
// The count-only form skips the look-back and adds tile sums atomically.
#include <algorithm>
#include <cmath>

#include "hg_cluster.cuh"
#include "hg_device.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"
#include "hg_scan.cuh"

namespace hg {

constexpr int PROBE_BLOCK = 256;
constexpr int PROBE_QPT = 4;
constexpr uint64_t PROBE_TILE = uint64_t(PROBE_BLOCK) * PROBE_QPT;

// Direct probe.  Persistent: CTAs take tiles of PROBE_TILE queries in ticket
// order (count-only tiles need no order and use the same loop).
template <typename KeyT, bool EMIT, bool A_IDX, bool Q_IDX>
__global__ void __launch_bounds__(PROBE_BLOCK)
    k_probe(const uint32_t* __restrict__ a_off, const KeyT* __restrict__ a_keys, const uint32_t* __restrict__ a_idx,
            BucketMap bm, const KeyT* __restrict__ q, uint64_t nq, const uint32_t* __restrict__ q_idx,
            uint32_t* __restrict__ pairs, uint64_t cap, unsigned long long* d_count, uint64_t* status,
            unsigned* ticket, const uint32_t* gate) {
  if (gated_off(gate)) return;
  __shared__ uint64_t red[PROBE_BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
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
    for (int j = 0; j < PROBE_QPT; j++) {
      const uint64_t i = q0 + j;
      lo[j] = hi[j] = 0;
      key[j] = 0;
      if (i < nq) {
        key[j] = __ldcs(q + i);
        const uint32_t b = bm.of_key(key[j]);
        lo[j] = a_off[b];
        hi[j] = a_off[b + 1];
      }
    }
#pragma unroll
    for (int j = 0; j < PROBE_QPT; j++)
      for (uint32_t x = lo[j]; x < hi[j]; x++) c += (a_keys[x] == key[j]);
    if constexpr (!EMIT) {
      counted += c;
      __syncthreads();
    } else {
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
// The CTA stages table A's offsets for its W buckets and, when they fit, A's
// keys (and index) for those buckets in shared memory with coalesced loads;
// the fine partition's queries then probe shared memory only.  A partition
// whose keys do not fit ("spill", heavy duplicates) reads A from global
// memory instead.  Every query is hashed once: its local bucket is kept in
// shared memory between the counting pass and the emitting pass.  Emission:
// the CTA reserves its partition's output range with one atomic on the running
// pair count, then writes pairs chunk by chunk (block scan per chunk); a
// query with exactly one match writes it from the first pass's result.
// Dynamic smem: soff[W+1] | sak[capa] | sai[capa] | slb[capq] (u16) | sx[capq] (u32, EMIT)
template <typename KeyT, bool A_IDX, bool EMIT, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
    k_fine_probe(const KeyT* __restrict__ qkeys, const uint32_t* __restrict__ qidx, const uint32_t* __restrict__ qstart,
                 uint64_t n_fine, uint64_t capq, uint32_t fine_log2, BucketMap bm, uint64_t n_buckets,
                 const uint32_t* __restrict__ a_off, const KeyT* __restrict__ a_keys, const uint32_t* __restrict__ a_idx,
                 uint32_t capa, uint32_t* __restrict__ pairs, uint64_t pair_cap, unsigned long long* d_count,
                 const uint32_t* flags) {
  if (*reinterpret_cast<const volatile uint32_t*>(flags) & FLAG_OVERFLOW) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t W = 1u << fine_log2;
  uint32_t* soff = reinterpret_cast<uint32_t*>(smem_raw);
  KeyT* sak = reinterpret_cast<KeyT*>(smem_raw + align_up_dev(size_t(W + 1) * 4, 16));
  uint32_t* sai = reinterpret_cast<uint32_t*>(sak + capa);
  uint32_t* sx = A_IDX ? sai + capa : reinterpret_cast<uint32_t*>(sak + capa);  // per query: first match (local)
  uint16_t* slb = reinterpret_cast<uint16_t*>(EMIT ? sx + capq : sx);           // per query: local bucket
  __shared__ uint64_t red[BLOCK / 32 + 1];
  __shared__ uint64_t s_run;
  uint64_t counted = 0;
  for (uint64_t f = blockIdx.x; f < n_fine; f += gridDim.x) {
    const uint64_t b0 = f << fine_log2;
    if (b0 >= n_buckets) break;
    const uint32_t nb = static_cast<uint32_t>(umin64(W, n_buckets - b0));
    const uint32_t a_s = a_off[b0];
    const uint32_t cnt_a = a_off[b0 + nb] - a_s;
    const bool spill = cnt_a > capa;
    for (uint32_t j = threadIdx.x; j <= nb; j += BLOCK) soff[j] = a_off[b0 + j] - a_s;
    if (!spill) {
      for (uint32_t x = threadIdx.x; x < cnt_a; x += BLOCK) {
        sak[x] = a_keys[a_s + x];
        if constexpr (A_IDX) sai[x] = a_idx[a_s + x];
      }
    }
    __syncthreads();
    const uint32_t qb = qstart[f];
    const uint32_t m = qstart[f + 1] - qb;
    const KeyT* src = qkeys + f * capq;
    const uint32_t* srci = qidx + f * capq;

    // matches of key k in local bucket lb: count, first position (local to a_s)
    auto scan_bucket = [&](KeyT k, uint32_t lb, uint32_t& first) -> uint32_t {
      const uint32_t s = soff[lb], e = soff[lb + 1];
      uint32_t c = 0;
      first = 0;
      if (spill) {
        for (uint32_t x = s; x < e; x++)
          if (a_keys[a_s + x] == k) {
            if (c == 0) first = x;
            c++;
          }
      } else {
        for (uint32_t x = s; x < e; x++)
          if (sak[x] == k) {
            if (c == 0) first = x;
            c++;
          }
      }
      return c;
    };
    auto aref_of = [&](uint32_t x) -> uint32_t {
      if constexpr (A_IDX) return spill ? a_idx[a_s + x] : sai[x];
      return a_s + x;
    };

    if constexpr (EMIT) {
      uint64_t mine = 0;
      for (uint32_t r = threadIdx.x; r < m; r += BLOCK) {
        const KeyT k = src[r];
        const uint32_t lb = static_cast<uint32_t>(bm.of_key(k) - b0);
        uint32_t first;
        const uint32_t c = scan_bucket(k, lb, first);
        slb[r] = static_cast<uint16_t>(lb);
        sx[r] = c == 0 ? 0xffffffffu : (c == 1 ? first : 0xfffffffeu);
        mine += c;
      }
      uint64_t tot;
      block_exclusive_scan<BLOCK>(mine, red, &tot);
      if (threadIdx.x == 0) {
        s_run = tot ? atomicAdd(d_count, static_cast<unsigned long long>(tot)) : 0ull;
        if (s_run + tot > pair_cap) record_error(HG_ERR_PAIR_CAPACITY);
      }
      __syncthreads();
      if (tot) {
        uint64_t run = s_run;
        for (uint32_t r0 = 0; r0 < m; r0 += BLOCK) {
          const uint32_t r = r0 + threadIdx.x;
          const uint32_t x = r < m ? sx[r] : 0xffffffffu;
          uint32_t c = 0;
          KeyT k = KeyT(0);
          if (x == 0xfffffffeu) {  // several matches: count them again
            k = src[r];
            uint32_t first;
            c = scan_bucket(k, slb[r], first);
          } else if (x != 0xffffffffu) {
            c = 1;
          }
          uint64_t chunk;
          uint64_t pos = run + block_exclusive_scan<BLOCK>(uint64_t(c), red, &chunk);
          if (c == 1 && x != 0xfffffffeu) {
            if (pos < pair_cap) reinterpret_cast<uint2*>(pairs)[pos] = make_uint2(aref_of(x), srci[r]);
          } else if (c) {
            const uint32_t qref = srci[r];
            const uint32_t lb = slb[r];
            const uint32_t s = soff[lb], e = soff[lb + 1];
            for (uint32_t y = s; y < e; y++) {
              const KeyT a = spill ? a_keys[a_s + y] : sak[y];
              if (a == k) {
                if (pos < pair_cap) reinterpret_cast<uint2*>(pairs)[pos] = make_uint2(aref_of(y), qref);
                pos++;
              }
            }
          }
          run += chunk;
        }
      }
    } else {
      for (uint32_t r = threadIdx.x; r < m; r += BLOCK) {
        const KeyT k = src[r];
        uint32_t first;
        counted += scan_bucket(k, static_cast<uint32_t>(bm.of_key(k) - b0), first);
      }
    }
    __syncthreads();
  }
  if constexpr (!EMIT) {
    uint64_t tot;
    block_exclusive_scan<BLOCK>(counted, red, &tot);
    if (threadIdx.x == 0 && tot) atomicAdd(d_count, static_cast<unsigned long long>(tot));
  }
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
  // pass 3 keeps a 16-bit local bucket and a 32-bit first match per query
  bool part_ok = plan_geometry(nq, q_rec, n_a, a_rec, 4, 6, n_buckets, true, &p.g, FINE_PROBE_SMEM_BUDGET);
  if (part_ok) {
    p.g.smem1 = pass1_smem(p.g.n_parts, key_bytes);
    p.g.smem2 = split_smem(p.g.split_log2, key_bytes, true);
    part_ok = p.g.smem1 <= SMEM_BUDGET && p.g.smem2 <= SMEM_BUDGET;
  }
  const uint64_t a_bytes = n_a * a_rec + 4 * n_buckets;
  int path = force_path;
  if (path < 0) path = (part_ok && a_bytes > (64ull << 20) && nq >= (1ull << 20)) ? PROBE_PARTITIONED : PROBE_DIRECT;
  // Too few buckets to split the queries finely (everything in a handful of
  // buckets): the direct probe, even when the partitioned one is asked for.
  if (path == PROBE_PARTITIONED && !part_ok) path = PROBE_DIRECT;
  p.path = path;
  size_t off = 0;
  p.off_status = off;  off = align_up(off + (emit ? p.tiles * 8 : 0));
  p.off_ticket = off;  off = align_up(off + 4 * sizeof(unsigned));
  p.off_flags = off;   off = align_up(off + sizeof(uint32_t));
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
  } else {
    p.off_pcount = p.off_pstatus = p.off_fcount = p.off_fstatus = off;
    p.off_pkeys = p.off_pidx = p.off_fkeys = p.off_fidx = off;
  }
  p.total = off;
  *plan = p;
  return HG_OK;
}

template <typename KeyT, bool EMIT>
static void launch_probe_direct(const ProbePlan& p, const uint32_t* a_off, const KeyT* a_keys, const uint32_t* a_idx,
                                const KeyT* q, const uint32_t* q_idx, uint32_t* pairs, uint64_t cap,
                                unsigned long long* d_count, uint64_t* status, unsigned* ticket, const uint32_t* gate,
                                cudaStream_t s) {
  const BucketMap bm = BucketMap::make(p.n_buckets);
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(p.tiles, uint64_t(device_sm_count()) * 8));
  Phase ph(s, gate ? (EMIT ? "fallback_probe_emit" : "fallback_probe_count") : (EMIT ? "probe_emit" : "probe_count"));
  count_launch();
#define HG_PROBE_LAUNCH(AI, QI)                                                                            \
  k_probe<KeyT, EMIT, AI, QI><<<grid, PROBE_BLOCK, 0, s>>>(a_off, a_keys, a_idx, bm, q, p.nq, q_idx, pairs, \
                                                          cap, d_count, status, ticket, gate)
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
  const BucketMap bm = BucketMap::make(p.n_buckets);
  const PartGeometry& g = p.g;
  uint32_t* flags = reinterpret_cast<uint32_t*>(ws + p.off_flags);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  uint64_t* status = reinterpret_cast<uint64_t*>(ws + p.off_status);
  HG_CUDA(cudaMemsetAsync(ws, 0, p.off_pkeys, s), "intersect: workspace memset");
  hg_status st = run_partition_passes<KeyT, 1, true>(g, p.nq, q, q_idx, bm, ws, p.off_flags, p.off_ticket,
                                                     p.off_pcount, p.off_pstatus, p.off_fcount, p.off_fstatus,
                                                     p.off_pkeys, p.off_pidx, p.off_fkeys, p.off_fidx, "probe", s);
  if (st != HG_OK) return st;
  {
    auto go = [&](auto kern) {
      const int bps = blocks_per_sm(kern, FINE_BLOCK, g.smem3);
      if (bps <= 0) {
        st = lib_fail(HG_ERR_CUDA, "fine-probe kernel cannot be resident");
        return;
      }
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(g.n_fine, uint64_t(device_sm_count()) * bps));
      Phase ph(s, EMIT ? "fine_probe_emit" : "fine_probe_count");
      count_launch();
      kern<<<std::max(grid, 1u), FINE_BLOCK, g.smem3, s>>>(
          reinterpret_cast<const KeyT*>(ws + p.off_fkeys), reinterpret_cast<const uint32_t*>(ws + p.off_fidx),
          reinterpret_cast<const uint32_t*>(ws + p.off_fcount), g.n_fine, g.fine_cap, g.fine_log2, bm, p.n_buckets,
          a_off, a_keys, a_idx, g.smem_cap, pairs, cap, d_count, static_cast<const uint32_t*>(flags));
      const cudaError_t e = cudaPeekAtLastError();
      if (e != cudaSuccess) st = cuda_fail(e, "fine-probe launch");
    };
    if (a_idx) go(k_fine_probe<KeyT, true, EMIT, FINE_BLOCK>);
    else go(k_fine_probe<KeyT, false, EMIT, FINE_BLOCK>);
    if (st != HG_OK) return st;
  }
  // Fallback when a query partition overflowed (heavy duplicates): the direct
  // probe, gated on the flag.
  launch_probe_direct<KeyT, EMIT>(p, a_off, a_keys, a_idx, q, q_idx, pairs, cap, d_count, status, ticket, flags, s);
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
    const cudaError_t e = cudaMemsetAsync(ws, 0, p.total, s);
    if (e != cudaSuccess) { st = cuda_fail(e, "intersect: workspace memset"); return; }
    if (emit) launch_probe_direct<KeyT, true>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, status, ticket, nullptr, s);
    else launch_probe_direct<KeyT, false>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, status, ticket, nullptr, s);
  };
  if (p.key_bytes == 4) run(uint32_t{});
  else run(uint64_t{});
  if (st != HG_OK) return st;
  HG_CUDA(cudaPeekAtLastError(), "intersect: kernel launch");
  return HG_OK;
}

}  // namespace hg
