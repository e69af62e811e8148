// hg_device.cuh -- device primitives shared by the HashGraph kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>
#include <cuda/atomic>

#include "hashgraph_b200.h"

namespace hg {

constexpr unsigned FULL_MASK = 0xffffffffu;

// murmur3_x86_32 of the key's low 4 bytes, seed 0.  The reference hashes
// len = sizeof(int) bytes starting at &key (include/SingleHashGraphOperators.cuh:31-69,
// include/MultiHashGraphDeviceOperators.cuh:37-73), so a 64-bit key contributes
// only its low 32 bits; with len = 4 the function is one body block, the
// length xor and the fmix32 finaliser.
__host__ __device__ __forceinline__ uint32_t murmur3_low32(uint64_t key) {
  uint32_t k = static_cast<uint32_t>(key);
  k *= 0xcc9e2d51u;
  k = (k << 15) | (k >> 17);
  k *= 0x1b873593u;
  uint32_t h = (k << 13) | (k >> 19);  // (seed 0) ^ k, rotated
  h = h * 5u + 0xe6546b64u;
  h ^= 4u;
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

// Exact `h % d` for 32-bit h and a divisor fixed per launch.  A power-of-two
// d (including d = 2^32, one bucket per hash value) is a mask.  Any other d
// uses the published direct-remainder method of Lemire, Kaser and Kurz
// ("Faster remainder by direct computation", 2019): magic =
// floor((2^64-1)/d) + 1; the remainder is the high 64 bits of
// (magic*h mod 2^64) * d.
struct BucketMap {
  uint64_t magic;
  uint32_t d;
  uint32_t mask;  // d - 1 when d is a power of two (0xffffffff for d = 2^32)
  uint32_t pow2;  // 1 when d is a power of two
  uint32_t base;  // first bucket of a shard's range (fastmod form only)

  static BucketMap make(uint64_t n_buckets) {
    BucketMap m;
    m.pow2 = (n_buckets & (n_buckets - 1)) == 0 ? 1u : 0u;
    m.base = 0;
    if (n_buckets >= (1ull << 32)) {
      m.magic = 0; m.d = 0; m.mask = 0xffffffffu;
    } else {
      m.d = static_cast<uint32_t>(n_buckets);
      m.magic = UINT64_MAX / m.d + 1;
      m.mask = m.pow2 ? m.d - 1 : 0u;
    }
    return m;
  }
  // The shard [lo, lo + local) of a table of `total` buckets: a key's bucket
  // in the shard is (hash % total) - lo, for keys whose bucket lies in the
  // range.  An aligned power-of-two range of a power-of-two table is itself a
  // power-of-two table (the hash's low bits), so it keeps the mask form.
  // total < 2^32 otherwise.
  static BucketMap make_range(uint64_t total, uint64_t lo, uint64_t local) {
    const bool p2 = (total & (total - 1)) == 0 && (local & (local - 1)) == 0;
    if (lo == 0 && local == total) return make(total);
    if (p2 && local > 0 && lo % local == 0) return make(local);
    BucketMap m = make(total);
    m.pow2 = 0;
    m.mask = 0;
    m.base = static_cast<uint32_t>(lo);
    return m;
  }
  // high 64 bits of x * d for a 32-bit d, from 32x32 products: with
  // x = xh*2^32 + xl, x*d = (xh*d + hi32(xl*d))*2^32 + lo32(xl*d), and the
  // low word cannot carry into bit 64, so the result is bits 32.. of
  // xh*d + hi32(xl*d).
  __host__ __device__ __forceinline__ uint32_t of_hash(uint32_t h) const {
    if (pow2) return h & mask;
    const uint64_t x = magic * h;
    const uint32_t xl = static_cast<uint32_t>(x), xh = static_cast<uint32_t>(x >> 32);
#ifdef __CUDA_ARCH__
    const uint32_t c = __umulhi(xl, d);
#else
    const uint32_t c = static_cast<uint32_t>((static_cast<uint64_t>(xl) * d) >> 32);
#endif
    return static_cast<uint32_t>((static_cast<uint64_t>(xh) * d + c) >> 32) - base;
  }
  __host__ __device__ __forceinline__ uint32_t of_key(uint64_t key) const {
    return of_hash(murmur3_low32(key));
  }
};

// ---------------------------------------------------------------------------
// Device-side error word (one per device).  Kernels record the first failure
// (a look-back wait that ran out, a pair buffer that was too small, ...); the
// host reads and clears it with hg_device_error().  Defined here: the library
// is one translation unit (hg_lib.cu).
// ---------------------------------------------------------------------------
__device__ int32_t g_device_error = 0;

// Host-side record of the last CUDA failure inside the library (per thread),
// returned by hg_last_error().
inline char* last_error_buffer() {
  static thread_local char buf[320] = {0};
  return buf;
}
inline hg_status cuda_fail(cudaError_t e, const char* where) {
  std::snprintf(last_error_buffer(), 320, "%s: %s (%d)", where, cudaGetErrorString(e), static_cast<int>(e));
  return e == cudaErrorMemoryAllocation ? HG_ERR_OUT_OF_MEMORY : HG_ERR_CUDA;
}
inline hg_status lib_fail(hg_status st, const char* what) {
  std::snprintf(last_error_buffer(), 320, "%s", what);
  return st;
}
#define HG_CUDA(expr, where)                        \
  do {                                              \
    const cudaError_t hg_e_ = (expr);               \
    if (hg_e_ != cudaSuccess) return ::hg::cuda_fail(hg_e_, where); \
  } while (0)

__device__ __forceinline__ void record_error(int32_t code) {
  atomicCAS(reinterpret_cast<int*>(&g_device_error), 0, code);
}

// Device-side fault word: the first fault (a bounded wait that gave up, or a
// position found outside its output).  The device state that produced it is
// not trusted, so while it is set every kernel of the library returns at
// entry, writing nothing, until the host reads and clears it with
// hg_device_error() -- a fault ends in a clean error status, never in a write
// through bad offsets.
__device__ int32_t g_device_fault = 0;

__device__ __forceinline__ void record_fault(int32_t code) {
  atomicCAS(reinterpret_cast<int*>(&g_device_fault), 0, code);
  record_error(code);
}

__device__ __forceinline__ bool device_faulted() {
  return *reinterpret_cast<const volatile int32_t*>(&g_device_fault) != 0;
}

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__host__ __device__ constexpr size_t align_up_dev(size_t x, size_t a) { return (x + a - 1) / a * a; }

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp-aggregated atomicAdd(ctr + slot, 1): lanes whose `slot` agree elect one
// leader (lowest lane) that adds the group size; every lane gets its own
// position.  Lanes with valid == false take no part.  All 32 lanes of the warp
// must call this together.
template <typename CtrT>
__device__ __forceinline__ CtrT warp_aggregated_inc(CtrT* ctr, uint32_t slot, bool valid) {
  const uint64_t tag = valid ? static_cast<uint64_t>(slot) : (1ull << 40);
  const unsigned peers = __match_any_sync(FULL_MASK, tag);
  const unsigned leader = __ffs(peers) - 1;
  const unsigned rank = __popc(peers & lanemask_lt());
  CtrT base = 0;
  if (valid && lane_id() == leader) base = atomicAdd(ctr + slot, static_cast<CtrT>(__popc(peers)));
  base = __shfl_sync(FULL_MASK, base, leader);
  return base + static_cast<CtrT>(rank);
}

// Warp-aggregated increment without a returned position (counting only).
template <typename CtrT>
__device__ __forceinline__ void warp_aggregated_count(CtrT* ctr, uint32_t slot, bool valid) {
  const uint64_t tag = valid ? static_cast<uint64_t>(slot) : (1ull << 40);
  const unsigned peers = __match_any_sync(FULL_MASK, tag);
  if (valid && lane_id() == static_cast<unsigned>(__ffs(peers) - 1))
    atomicAdd(ctr + slot, static_cast<CtrT>(__popc(peers)));
}

// Quotient of 32-bit v by a fixed 32-bit divisor d >= 1 without a division
// instruction sequence: q = mulhi64(M, v) with M = floor((2^64 - 1) / d) + 1,
// exact for every 32-bit v (Lemire, Kaser, Kurz, "Faster remainder by direct
// computation", 2019, with 64-bit M for 32-bit operands); d = 1 is v itself.
struct Div32 {
  uint64_t magic = 0;
  uint32_t d = 1;
  static Div32 make(uint32_t d) {
    Div32 x;
    x.d = d ? d : 1;
    x.magic = x.d > 1 ? ~0ull / x.d + 1 : 0;
    return x;
  }
  __device__ __forceinline__ uint32_t div(uint32_t v) const {
    return d > 1 ? static_cast<uint32_t>(__umul64hi(magic, v)) : v;
  }
};

// Streaming loads for data touched once.
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }

}  // namespace hg
