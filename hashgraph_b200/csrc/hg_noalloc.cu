// hg_noalloc.cu -- a build entry point that allocates no device memory.
//
// Who needs it: code that must not call cudaMalloc (or any allocator) at the
// point where it builds a table.  Examples: a serving process whose device
// memory is handed out entirely by its own pool allocator, so an allocation
// from a library would fail or break the pool's accounting; a caller running
// inside another allocator's callback, where allocating again would re-enter
// it; and real-time loops that forbid allocation after start-up because
// cudaMalloc can synchronise the device and has no latency bound.  The
// caller still provides the keys and the output arrays.
//
// What replaces the workspace: the direct build (count, look-back scan,
// scatter) needs only the scan's tile status words and tickets as scratch.
// They live in the file-scope array below, a fixed NOALLOC_SCRATCH_BYTES
// that every GPU loading this library holds until the process exits.  That
// caps n_buckets at NOALLOC_MAX_BUCKETS (2^25); larger tables are refused.
//
// Sharing: every call uses the same array, which keeps the last call's
// contents, so each call clears the words that must start at zero (stream-
// ordered, before its kernels).  Calls whose work overlaps on the GPU (other
// streams, other host threads) race on the array and must be serialised by
// the caller.
//
// Host code sees only a host-side stand-in for g_noalloc_scratch; its device
// address comes from cudaGetSymbolAddress, taken once per device on the
// first call with that device current (so the first call on each device
// should happen before any stream capture).  The address is kept together
// with the id of the CUDA context it was taken in; after a device reset
// (a new primary context, the module loaded again) the next call takes it
// again.
#include <mutex>

#include "hg_device.cuh"
#include "hg_plan.h"

namespace hg {

constexpr uint64_t NOALLOC_MAX_TILES = 8192;                              // look-back status words
constexpr uint64_t NOALLOC_MAX_BUCKETS = NOALLOC_MAX_TILES * SCAN_TILE;   // 2^25
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_MAX_TILES * 8 + 2 * WS_ALIGN;  // + tickets, flags

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Id of the current CUDA context (cuCtxGetCurrent + cuCtxGetId, reached
// through the runtime's driver entry points so the library needs no link to
// the driver library), or 0 when it cannot be read.
static unsigned long long current_context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

// Device address of g_noalloc_scratch on the current device: looked up once
// per device and context (every call when the context id cannot be read).
static hg_status noalloc_scratch(void** out) {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  static unsigned long long ctx_of[64] = {0};
  int dev = 0;
  HG_CUDA(cudaGetDevice(&dev), "hg_build_into_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= 64) return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_build_into_noalloc: device index >= 64");
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev] || ctx == 0 || ctx != ctx_of[dev]) {
    void* p = nullptr;
    HG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch), "hg_build_into_noalloc: cudaGetSymbolAddress");
    addr[dev] = p;
    ctx_of[dev] = current_context_id();  // the lookup makes the device's context current
  }
  *out = addr[dev];
  return HG_OK;
}

}  // namespace hg

using namespace hg;

extern "C" hg_status hg_build_into_noalloc(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                                           uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                                           hg_stream_t stream) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0 || !d_offsets || (n > 0 && (!d_keys || !d_keys_out))) return HG_ERR_INVALID_ARGUMENT;
  if (n >= (1ull << 32)) return lib_fail(HG_ERR_TOO_LARGE, "hg_build_into_noalloc: n must be below 2^32");
  if (n_buckets > NOALLOC_MAX_BUCKETS)
    return lib_fail(HG_ERR_TOO_LARGE,
                    "hg_build_into_noalloc: n_buckets exceeds 33554432 (2^25), the limit of its fixed 64 KiB scratch");
  BuildPlan plan;
  hg_status st = plan_build(n, key_bytes, n_buckets, d_idx_out != nullptr, &plan, BUILD_DIRECT);
  if (st != HG_OK) return st;
  if (plan.path != BUILD_DIRECT || plan.total > NOALLOC_SCRATCH_BYTES)
    return lib_fail(HG_ERR_TOO_LARGE, "hg_build_into_noalloc: plan does not fit the fixed scratch");
  void* scratch = nullptr;
  st = noalloc_scratch(&scratch);
  if (st != HG_OK) return st;
  // launch_build clears the scan status words and tickets in the scratch and
  // the offsets (stream-ordered) before its kernels run.
  return launch_build(plan, d_keys, d_offsets, d_keys_out, d_idx_out, scratch, reinterpret_cast<cudaStream_t>(stream));
}
