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
#include "hg_device.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"
#include "hg_scan.cuh"

namespace hg {

constexpr int PROBE_BLOCK = 256;
constexpr int PROBE_QPT = 4;
constexpr uint64_t PROBE_TILE = uint64_t(PROBE_BLOCK) * PROBE_QPT;

template <typename KeyT, bool EMIT, bool A_IDX, bool Q_IDX>
__global__ void __launch_bounds__(PROBE_BLOCK)
    k_probe(const uint32_t* __restrict__ a_off, const KeyT* __restrict__ a_keys, const uint32_t* __restrict__ a_idx,
            BucketMap bm, const KeyT* __restrict__ q, uint64_t nq, const uint32_t* __restrict__ q_idx,
            uint32_t* __restrict__ pairs, uint64_t cap, unsigned long long* d_count, uint64_t* status,
            unsigned* ticket) {
  __shared__ uint64_t red[PROBE_BLOCK / 32 + 1];
  __shared__ uint64_t s_tile, s_prefix;
  uint64_t tile;
  if constexpr (EMIT) {
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    tile = s_tile;
  } else {
    tile = blockIdx.x;
  }
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

  uint64_t tile_total;
  const uint64_t excl = block_exclusive_scan<PROBE_BLOCK>(c, red, &tile_total);
  if constexpr (!EMIT) {
    if (threadIdx.x == 0 && tile_total) atomicAdd(d_count, static_cast<unsigned long long>(tile_total));
    return;
  } else {
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
    const uint64_t ntiles = (nq + PROBE_TILE - 1) / PROBE_TILE;
    if (threadIdx.x == 0 && tile == ntiles - 1) {
      const uint64_t total = prefix + tile_total;
      *d_count = total;
      if (total > cap) record_error(HG_ERR_PAIR_CAPACITY);
    }
  }
}

hg_status plan_probe(uint64_t n_buckets, uint64_t nq, int key_bytes, bool emit, ProbePlan* plan) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0) return HG_ERR_INVALID_ARGUMENT;
  if (nq >= (1ull << 32) || n_buckets > (1ull << 32)) return HG_ERR_TOO_LARGE;
  ProbePlan p;
  p.nq = nq;
  p.n_buckets = n_buckets;
  p.key_bytes = key_bytes;
  p.emit = emit;
  p.tiles = (nq + PROBE_TILE - 1) / PROBE_TILE;
  size_t off = 0;
  p.off_status = off;
  off = align_up(off + (emit ? p.tiles * 8 : 0));
  p.off_ticket = off;
  off = align_up(off + sizeof(unsigned));
  p.total = off;
  *plan = p;
  return HG_OK;
}

template <typename KeyT, bool EMIT>
static void launch_probe_t(const ProbePlan& p, const uint32_t* a_off, const KeyT* a_keys, const uint32_t* a_idx,
                           const KeyT* q, const uint32_t* q_idx, uint32_t* pairs, uint64_t cap,
                           unsigned long long* d_count, uint64_t* status, unsigned* ticket, cudaStream_t s) {
  const BucketMap bm = BucketMap::make(p.n_buckets);
  const unsigned grid = static_cast<unsigned>(p.tiles);
  Phase ph(s, EMIT ? "probe_emit" : "probe_count");
  count_launch();
#define HG_PROBE_LAUNCH(AI, QI)                                                                            \
  k_probe<KeyT, EMIT, AI, QI><<<grid, PROBE_BLOCK, 0, s>>>(a_off, a_keys, a_idx, bm, q, p.nq, q_idx, pairs, \
                                                          cap, d_count, status, ticket)
  if (a_idx) {
    if (q_idx) HG_PROBE_LAUNCH(true, true); else HG_PROBE_LAUNCH(true, false);
  } else {
    if (q_idx) HG_PROBE_LAUNCH(false, true); else HG_PROBE_LAUNCH(false, false);
  }
#undef HG_PROBE_LAUNCH
}

hg_status launch_probe(const ProbePlan& p, const uint32_t* a_off, const void* a_keys, const uint32_t* a_idx,
                       const void* q_keys, const uint32_t* q_idx, uint32_t* pairs, uint64_t pair_cap,
                       unsigned long long* d_count, void* d_ws, cudaStream_t s) {
  char* ws = static_cast<char*>(d_ws);
  uint64_t* status = reinterpret_cast<uint64_t*>(ws + p.off_status);
  unsigned* ticket = reinterpret_cast<unsigned*>(ws + p.off_ticket);
  if (cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s) != cudaSuccess) return HG_ERR_CUDA;
  if (p.tiles == 0) return HG_OK;
  if (cudaMemsetAsync(ws, 0, p.total, s) != cudaSuccess) return HG_ERR_CUDA;
  const bool emit = p.emit && pairs != nullptr;
  if (p.key_bytes == 4) {
    auto ak = static_cast<const uint32_t*>(a_keys);
    auto qk = static_cast<const uint32_t*>(q_keys);
    if (emit) launch_probe_t<uint32_t, true>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, status, ticket, s);
    else launch_probe_t<uint32_t, false>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, status, ticket, s);
  } else {
    auto ak = static_cast<const uint64_t*>(a_keys);
    auto qk = static_cast<const uint64_t*>(q_keys);
    if (emit) launch_probe_t<uint64_t, true>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, status, ticket, s);
    else launch_probe_t<uint64_t, false>(p, a_off, ak, a_idx, qk, q_idx, pairs, pair_cap, d_count, status, ticket, s);
  }
  return cudaPeekAtLastError() == cudaSuccess ? HG_OK : HG_ERR_CUDA;
}

}  // namespace hg
