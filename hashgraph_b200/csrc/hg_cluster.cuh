// hg_cluster.cuh -- thread-block-cluster helpers: launch with a cluster
// dimension, co-resident cluster counts, and the block-level scans the
// cluster kernels share.
#pragma once
#include <cooperative_groups.h>

#include <map>
#include <mutex>
#include <tuple>

#include "hg_device.cuh"
#include "hg_scan.cuh"

namespace hg {

namespace cg = cooperative_groups;

template <typename Kern, typename... Args>
static cudaError_t launch_cluster(Kern kern, unsigned grid, unsigned block, size_t smem, unsigned cl,
                                  cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(block, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

// Prepares `kern` for a cluster launch (dynamic smem, non-portable size when
// cl > 8) and returns how many clusters of `cl` CTAs can be co-resident
// (0 if the shape cannot run).  Cached per (kernel, smem, block, cl, device).
template <typename Kern>
static int cluster_capacity(Kern kern, unsigned block, size_t smem, unsigned cl) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, size_t, unsigned, unsigned, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(reinterpret_cast<const void*>(kern), smem, block, cl, dev);
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  int result = 0;
  // The kernel's dynamic-smem limit is always raised to the device's opt-in
  // maximum, so no later query with a smaller size can lower it under a
  // launch that needs more.
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa = {};
  cudaFuncGetAttributes(&fa, kern);
  const int max_dyn = optin - static_cast<int>(fa.sharedSizeBytes);
  if (max_dyn >= 0 && size_t(max_dyn) >= smem &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn) == cudaSuccess &&
      (cl <= 8 || cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess)) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl, 1, 1);
    cfg.blockDim = dim3(block, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) == cudaSuccess) result = n;
  }
  cudaGetLastError();
  std::lock_guard<std::mutex> g(mu);
  cache[key] = result;
  return result;
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
