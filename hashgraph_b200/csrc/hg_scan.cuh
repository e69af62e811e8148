// hg_scan.cuh -- block scans and the decoupled look-back device-wide scan.
//
// Replaces the reference's cub::DeviceScan::ExclusiveSum over bucket counts
// (src/SingleHashGraph.cu:167-173, src/MultiHashGraph.cu:353-366) and the
// cub::DeviceReduce::Sum + ExclusiveSum pair over intersect counts
// (src/MultiHashGraph.cu:691-715).  One pass: every tile publishes its
// aggregate, then warp 0 walks back over predecessor tiles (32 at a time)
// until it meets an inclusive prefix (Merrill & Garland, "Single-pass
// Parallel Prefix Scan with Decoupled Look-back", 2016).  Tiles are numbered
// by an atomic ticket so every predecessor has started.  The wait is bounded:
// after LOOKBACK_SPIN_LIMIT polls the tile records HG_ERR_DEVICE_TIMEOUT and
// returns instead of hanging.
#pragma once
#include "hg_device.cuh"

namespace hg {

// status word: [63:62] flag, [61:0] value
constexpr uint64_t ST_AGGREGATE = 1ull << 62;
constexpr uint64_t ST_PREFIX = 2ull << 62;
constexpr uint64_t ST_VALUE = (1ull << 62) - 1;
constexpr uint32_t LOOKBACK_SPIN_LIMIT = 1u << 22;
// Polls a look-back makes before it gives up: LOOKBACK_SPIN_LIMIT unless a
// test lowered it (hg_debug_set_wait_limit) to make the wait run out.
__device__ uint32_t g_lookback_limit = LOOKBACK_SPIN_LIMIT;

__device__ __forceinline__ uint64_t ld_acquire(const uint64_t* p) {
  cuda::atomic_ref<const unsigned long long, cuda::thread_scope_device> r(
      *reinterpret_cast<const unsigned long long*>(p));
  return r.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void st_release(uint64_t* p, uint64_t v) {
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(
      *reinterpret_cast<unsigned long long*>(p));
  r.store(v, cuda::memory_order_release);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const unsigned lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(FULL_MASK, v, o);
    if (lane >= static_cast<unsigned>(o)) v += u;
  }
  return v;
}

// Exclusive scan of one value per thread across the block.  `scratch` holds
// at least BLOCK/32 + 1 elements.  Returns the exclusive prefix; *total gets
// the block sum.  Contains __syncthreads().
template <int BLOCK, typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* scratch, T* total) {
  constexpr int NW = BLOCK / 32;
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  T inc = warp_inclusive_scan(v);
  if (lane == 31) scratch[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < NW ? scratch[lane] : T(0);
    T wi = warp_inclusive_scan(w);
    if (lane < NW) scratch[lane] = wi - w;
    if (lane == NW - 1) scratch[NW] = wi;
  }
  __syncthreads();
  T excl = scratch[warp] + inc - v;
  *total = scratch[NW];
  __syncthreads();
  return excl;
}

// Decoupled look-back for `tile` with block aggregate `agg`.  Must be called
// by all 32 lanes of exactly one warp.  Returns the exclusive prefix of the
// tile (the same value in every lane) and publishes the inclusive prefix.
__device__ __forceinline__ uint64_t lookback_exclusive(uint64_t* status, uint64_t tile,
                                                       uint64_t agg) {
  const unsigned lane = lane_id();
  if (tile == 0) {
    if (lane == 0) st_release(status, ST_PREFIX | (agg & ST_VALUE));
    return 0;
  }
  if (lane == 0) st_release(status + tile, ST_AGGREGATE | (agg & ST_VALUE));
  uint64_t excl = 0;
  int64_t pred = static_cast<int64_t>(tile) - 1;
  uint32_t spins = 0;
  const uint32_t limit = *reinterpret_cast<const volatile uint32_t*>(&g_lookback_limit);
  unsigned sleep_ns = 8;
  while (true) {
    const int64_t j = pred - static_cast<int64_t>(lane);
    uint64_t s = j >= 0 ? ld_acquire(status + j) : ST_PREFIX;
    while (__any_sync(FULL_MASK, (s >> 62) == 0)) {
      if (++spins > limit) {
        record_fault(HG_ERR_DEVICE_TIMEOUT);  // later kernels return at entry
        return excl;
      }
      __nanosleep(sleep_ns);
      if (sleep_ns < 256) sleep_ns <<= 1;
      if ((s >> 62) == 0) s = ld_acquire(status + j);
    }
    const unsigned pfx = __ballot_sync(FULL_MASK, (s >> 62) == 2);
    if (pfx) {
      const unsigned first = __ffs(pfx) - 1;
      uint64_t v = lane <= first ? (s & ST_VALUE) : 0;
      excl += warp_sum(v);
      break;
    }
    excl += warp_sum(s & ST_VALUE);
    pred -= 32;
  }
  if (lane == 0) st_release(status + tile, ST_PREFIX | ((excl + agg) & ST_VALUE));
  return excl;
}

// Exclusive scan of ctr[0..nb) in shared memory by a block of BLOCK threads:
// warp w scans the contiguous segment [w*seg, (w+1)*seg) in chunks of 32
// (coalesced), after a block scan of the segment totals.  Replaces ctr[j] by
// base_local + exclusive prefix and calls out(j, global_value) for each j with
// global_value = base_global + exclusive prefix.  Returns the total.
// `wsum` needs BLOCK/32 + 1 entries.  Contains __syncthreads().
template <int BLOCK, typename Out>
__device__ __forceinline__ uint32_t block_scan_segments(uint32_t* ctr, uint32_t nb, uint32_t base_local,
                                                        uint32_t base_global, uint32_t* wsum, Out out) {
  constexpr int NW = BLOCK / 32;
  const unsigned warp = threadIdx.x >> 5, lane = lane_id();
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
    if (lane == NW - 1) wsum[NW] = wi;
  }
  __syncthreads();
  uint32_t run = wsum[warp];
  for (uint32_t j0 = s0; j0 < s1; j0 += 32) {
    const uint32_t j = j0 + lane;
    const uint32_t v = j < s1 ? ctr[j] : 0u;
    const uint32_t inc = warp_inclusive_scan(v);
    if (j < s1) {
      const uint32_t ex = run + inc - v;
      ctr[j] = base_local + ex;
      out(j, base_global + ex);
    }
    run += __shfl_sync(FULL_MASK, inc, 31);
  }
  const uint32_t total = wsum[NW];
  __syncthreads();
  return total;
}

}  // namespace hg
