// hg_bulk.cuh -- 1-D bulk asynchronous copies (TMA, cp.async.bulk) from global
// to shared memory, completed on an mbarrier.  Used to prefetch the next tile
// of a streaming pass while the current one is processed.
//
// Rules kept here: both addresses 16-byte aligned and the size a multiple of
// 16 (callers round and handle ragged edges with plain loads); every wait is
// bounded -- on expiry the kernel records HG_ERR_DEVICE_TIMEOUT and the caller
// waits (again bounded) for the copy it issued before returning.
#pragma once
#include "hg_device.cuh"

namespace hg {

constexpr uint32_t MBAR_SPIN_LIMIT = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes mbarrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (bulk copy) accesses: issue after a __syncthreads() that
// ends all reads of a buffer the next bulk copy overwrites.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of `bar`.  Returns false (and records the
// fault HG_ERR_DEVICE_TIMEOUT) if it did not complete within MBAR_SPIN_LIMIT
// polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < MBAR_SPIN_LIMIT; i++)
    if (mbar_try_wait(bar, parity)) return true;
  record_fault(HG_ERR_DEVICE_TIMEOUT);
  return false;
}

// Issues a bulk copy of `bytes` (multiple of 16, both ends 16-byte aligned)
// from src to dst completing on `bar`; called by one thread.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  mbar_arrive_expect_tx(bar, bytes);
  if (bytes) bulk_g2s(dst, src, bytes, bar);
}

}  // namespace hg
