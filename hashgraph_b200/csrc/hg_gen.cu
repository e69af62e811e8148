// hg_gen.cu -- seeded workload generators on the device.
//
// The reference's test main feeds sequential keys 0..n-1
// (test/MultiHashGraphTest.cu:105-111) or thrust minstd draws in [0, maxkey]
// (:26-37).  The workloads here need uniform 32/64-bit keys, a controlled
// overlap between two sets and Zipf skew, so keys come from a counter-based
// splitmix64 stream (Steele, Lea, Flood 2014):
//   rand64(seed, stream, i) = mix64(mix64(seed*G + stream + 1) + (i + 1)*G)
// with G = 0x9E3779B97F4A7C15.  32-bit keys take the top 32 bits.
#include <cmath>

#include "hg_device.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"

namespace hg {

constexpr uint64_t GOLDEN = 0x9E3779B97F4A7C15ull;
constexpr uint64_t ZIPF_UNIVERSE_SEED = 0x21BF;  // keys of a Zipf universe: mix64(rank ^ salt)

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t rand64(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed * GOLDEN + stream + 1) + (i + 1) * GOLDEN);
}

// Keyed bijection on [0, n): three odd-multiply / xorshift rounds on the
// enclosing power of two, cycle-walked back into range.
struct Perm {
  uint64_t a[3], c[3], mask, n;
  int s;
  static Perm make(uint64_t n, uint64_t seed) {
    Perm p;
    p.n = n;
    int k = n <= 1 ? 0 : 64 - __builtin_clzll(n - 1);
    p.mask = k == 64 ? ~0ull : ((1ull << k) - 1);
    p.s = k / 2 + 1;
    for (int r = 0; r < 3; r++) {
      p.a[r] = rand64(seed, 100 + r, 0) | 1ull;
      p.c[r] = rand64(seed, 200 + r, 0);
    }
    return p;
  }
  __device__ __forceinline__ uint64_t operator()(uint64_t i) const {
    if (n <= 1) return 0;
    uint64_t x = i;
    do {
#pragma unroll
      for (int r = 0; r < 3; r++) {
        x = (x * a[r] + c[r]) & mask;
        x ^= x >> s;
      }
    } while (x >= n);
    return x;
  }
};

template <typename KeyT>
__global__ void k_gen_uniform(KeyT* out, uint64_t n, uint64_t seed) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t r = rand64(seed, 0, i);
    out[i] = sizeof(KeyT) == 8 ? static_cast<KeyT>(r) : static_cast<KeyT>(r >> 32);
  }
}

template <typename KeyT>
__global__ void k_gen_bounded(KeyT* out, uint64_t n, uint64_t seed, uint64_t bound) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    out[i] = static_cast<KeyT>(rand64(seed, 0, i) % bound);
}

// out[i] = keys[pairs[2i + which]] widened to 64 bits.
template <typename KeyT>
__global__ void k_gather_pair_keys(const KeyT* keys, const uint32_t* pairs, uint64_t count, int which,
                                   int64_t* out) {
  if (entry_skip(nullptr)) return;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += uint64_t(gridDim.x) * blockDim.x)
    out[i] = static_cast<int64_t>(keys[pairs[2 * i + which]]);
}

template <typename KeyT>
__global__ void k_gen_overlap(KeyT* out, uint64_t n, const KeyT* a, uint64_t m, Perm pb, Perm pa, uint64_t seed) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t j = pb(i);
    KeyT v;
    if (j < m) {
      v = a[pa(j)];
    } else {
      const uint64_t r = rand64(seed, 2, j);
      v = sizeof(KeyT) == 8 ? static_cast<KeyT>(r) : static_cast<KeyT>(r >> 32);
    }
    out[i] = v;
  }
}

template <typename KeyT>
__global__ void k_gen_zipf(KeyT* out, uint64_t n, const uint64_t* cdf, uint64_t universe, uint64_t seed,
                           uint64_t salt) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t u = rand64(seed, 3, i);
    uint64_t lo = 0, hi = universe - 1;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (u < cdf[mid]) hi = mid; else lo = mid + 1;
    }
    const uint64_t key = mix64(lo ^ salt);
    out[i] = sizeof(KeyT) == 8 ? static_cast<KeyT>(key) : static_cast<KeyT>(key & 0xffffffffull);
  }
}

static unsigned gen_grid(uint64_t n) {
  const uint64_t want = (n + 255) / 256;
  const uint64_t cap = uint64_t(device_sm_count()) * 16;
  return static_cast<unsigned>(want < cap ? (want ? want : 1) : cap);
}

}  // namespace hg

using namespace hg;

extern "C" hg_status hg_gen_uniform(void* d_out, uint64_t n, int key_bytes, uint64_t seed, hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n == 0) return HG_OK;
  if (!d_out) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (key_bytes == 8) k_gen_uniform<uint64_t><<<gen_grid(n), 256, 0, s>>>(static_cast<uint64_t*>(d_out), n, seed);
  else k_gen_uniform<uint32_t><<<gen_grid(n), 256, 0, s>>>(static_cast<uint32_t*>(d_out), n, seed);
  return cudaPeekAtLastError() == cudaSuccess ? HG_OK : HG_ERR_CUDA;
}

extern "C" hg_status hg_gen_bounded(void* d_out, uint64_t n, int key_bytes, uint64_t seed, uint64_t bound,
                                    hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n == 0) return HG_OK;
  if (!d_out || bound == 0) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  count_launch();
  if (key_bytes == 8) k_gen_bounded<uint64_t><<<gen_grid(n), 256, 0, s>>>(static_cast<uint64_t*>(d_out), n, seed, bound);
  else k_gen_bounded<uint32_t><<<gen_grid(n), 256, 0, s>>>(static_cast<uint32_t*>(d_out), n, seed, bound);
  return cudaPeekAtLastError() == cudaSuccess ? HG_OK : HG_ERR_CUDA;
}

extern "C" hg_status hg_gather_pair_keys(const void* d_keys, int key_bytes, const uint32_t* d_pairs, uint64_t count,
                                         int which, int64_t* d_out, hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (count == 0) return HG_OK;
  if (!d_keys || !d_pairs || !d_out || (which != 0 && which != 1)) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  count_launch();
  if (key_bytes == 8)
    k_gather_pair_keys<uint64_t><<<gen_grid(count), 256, 0, s>>>(static_cast<const uint64_t*>(d_keys), d_pairs, count,
                                                                 which, d_out);
  else
    k_gather_pair_keys<uint32_t><<<gen_grid(count), 256, 0, s>>>(static_cast<const uint32_t*>(d_keys), d_pairs, count,
                                                                 which, d_out);
  return cudaPeekAtLastError() == cudaSuccess ? HG_OK : HG_ERR_CUDA;
}

// Reference-layout export: 16-byte {key, int64 index} records and int64 offsets.
template <typename KeyT>
__global__ void k_export_reference(const KeyT* keys, const uint32_t* idx, uint64_t n, const uint32_t* off,
                                   uint64_t n_buckets, unsigned char* kv16, int64_t* off64) {
  if (entry_skip(nullptr)) return;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += stride) {
    unsigned char* rec = kv16 + 16 * j;
    if (sizeof(KeyT) == 8) {
      *reinterpret_cast<uint64_t*>(rec) = static_cast<uint64_t>(keys[j]);
    } else {
      *reinterpret_cast<uint32_t*>(rec) = static_cast<uint32_t>(keys[j]);
      *reinterpret_cast<uint32_t*>(rec + 4) = 0u;
    }
    *reinterpret_cast<int64_t*>(rec + 8) = idx ? static_cast<int64_t>(idx[j]) : static_cast<int64_t>(j);
  }
  for (uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; b <= n_buckets; b += stride)
    off64[b] = static_cast<int64_t>(off[b]);
}

extern "C" hg_status hg_export_reference_layout(const uint32_t* d_offsets, const void* d_keys, const uint32_t* d_idx,
                                                uint64_t n, uint64_t n_buckets, int key_bytes, void* d_kv16,
                                                int64_t* d_offsets64, hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (!d_offsets || !d_kv16 || !d_offsets64 || (n && !d_keys)) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const uint64_t work = n > n_buckets + 1 ? n : n_buckets + 1;
  count_launch();
  if (key_bytes == 8)
    k_export_reference<uint64_t><<<gen_grid(work), 256, 0, s>>>(static_cast<const uint64_t*>(d_keys), d_idx, n,
                                                                d_offsets, n_buckets,
                                                                static_cast<unsigned char*>(d_kv16), d_offsets64);
  else
    k_export_reference<uint32_t><<<gen_grid(work), 256, 0, s>>>(static_cast<const uint32_t*>(d_keys), d_idx, n,
                                                                d_offsets, n_buckets,
                                                                static_cast<unsigned char*>(d_kv16), d_offsets64);
  return cudaPeekAtLastError() == cudaSuccess ? HG_OK : HG_ERR_CUDA;
}

extern "C" hg_status hg_gen_overlap(void* d_out, uint64_t n, int key_bytes, const void* d_a, uint64_t n_a,
                                    uint64_t n_from_a, uint64_t seed, hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n == 0) return HG_OK;
  if (!d_out || (n_from_a && !d_a) || n_from_a > n || n_from_a > n_a) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const Perm pb = Perm::make(n, seed), pa = Perm::make(n_a, seed + 1);
  if (key_bytes == 8)
    k_gen_overlap<uint64_t><<<gen_grid(n), 256, 0, s>>>(static_cast<uint64_t*>(d_out), n,
                                                        static_cast<const uint64_t*>(d_a), n_from_a, pb, pa, seed);
  else
    k_gen_overlap<uint32_t><<<gen_grid(n), 256, 0, s>>>(static_cast<uint32_t*>(d_out), n,
                                                        static_cast<const uint32_t*>(d_a), n_from_a, pb, pa, seed);
  return cudaPeekAtLastError() == cudaSuccess ? HG_OK : HG_ERR_CUDA;
}

extern "C" hg_status hg_gen_zipf(void* d_out, uint64_t n, int key_bytes, const uint64_t* d_cdf, uint64_t universe,
                                 uint64_t seed, hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n == 0) return HG_OK;
  if (!d_out || !d_cdf || universe == 0) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // The rank -> key map depends on the universe only, so sets drawn with
  // different seeds from one universe share their keys (a join has matches).
  const uint64_t salt = rand64(ZIPF_UNIVERSE_SEED, 4, universe);
  if (key_bytes == 8)
    k_gen_zipf<uint64_t><<<gen_grid(n), 256, 0, s>>>(static_cast<uint64_t*>(d_out), n, d_cdf, universe, seed, salt);
  else
    k_gen_zipf<uint32_t><<<gen_grid(n), 256, 0, s>>>(static_cast<uint32_t*>(d_out), n, d_cdf, universe, seed, salt);
  return cudaPeekAtLastError() == cudaSuccess ? HG_OK : HG_ERR_CUDA;
}

extern "C" hg_status hg_zipf_cdf(uint64_t* cdf, uint64_t universe, double s) {
  if (!cdf || universe == 0) return HG_ERR_INVALID_ARGUMENT;
  long double h = 0.0L;
  for (uint64_t r = 0; r < universe; r++) h += powl(static_cast<long double>(r + 1), -static_cast<long double>(s));
  long double acc = 0.0L;
  const long double two64 = 18446744073709551616.0L;
  for (uint64_t r = 0; r < universe; r++) {
    acc += powl(static_cast<long double>(r + 1), -static_cast<long double>(s));
    const long double v = acc / h * two64;
    cdf[r] = v >= two64 ? UINT64_MAX : static_cast<uint64_t>(v);
  }
  cdf[universe - 1] = UINT64_MAX;
  return HG_OK;
}
