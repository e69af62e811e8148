// hg_api.cu -- the C ABI (include/hashgraph_b200.h) over the sm_100a kernels.
#include <cstdio>
#include <cstring>
#include <new>

#include "hg_device.cuh"
#include "hg_plan.h"
#include "hg_prof.cuh"

using namespace hg;

struct hg_table {
  int device = 0;
  uint64_t capacity = 0, n = 0, n_buckets = 0;
  int key_bytes = 8;
  bool with_index = false;
  bool built = false;
  uint32_t* offsets = nullptr;
  void* keys = nullptr;
  uint32_t* idx = nullptr;
  void* ws = nullptr;
  size_t ws_bytes = 0;
};

static hg_status cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return HG_OK;
  if (e == cudaErrorMemoryAllocation) return HG_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return HG_ERR_NO_DEVICE;
  return HG_ERR_CUDA;
}

extern "C" const char* hg_status_str(hg_status s) {
  switch (s) {
    case HG_OK: return "ok";
    case HG_ERR_INVALID_ARGUMENT: return "invalid argument";
    case HG_ERR_CUDA: return "CUDA error";
    case HG_ERR_OUT_OF_MEMORY: return "out of device memory";
    case HG_ERR_PAIR_CAPACITY: return "more matches than pair capacity (count exact, pairs truncated)";
    case HG_ERR_DEVICE_TIMEOUT: return "bounded device-side wait gave up";
    case HG_ERR_TOO_LARGE: return "size out of range (n >= 2^32, n_buckets > 2^32, or workspace too small)";
    case HG_ERR_NO_DEVICE: return "no CUDA device";
    case HG_ERR_KEY_WIDTH: return "key width must be 4 or 8 bytes and match between tables";
    case HG_ERR_BUCKET_MISMATCH: return "tables have different bucket counts";
    case HG_ERR_DEVICE_STATE: return "a kernel found a position outside its output and wrote nothing";
    default: return "unknown status";
  }
}

extern "C" const char* hg_version(void) { return "hashgraph_b200 0.1 sm_100a"; }

extern "C" const char* hg_last_error(void) { return last_error_buffer(); }

extern "C" uint32_t hg_hash(uint64_t key) { return murmur3_low32(key); }

extern "C" hg_status hg_device_error(hg_stream_t stream, hg_status* code) {
  if (!code) return HG_ERR_INVALID_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  hg_status st = cuda_status(cudaStreamSynchronize(s));
  if (st != HG_OK) return st;
  int32_t v = 0, fault = 0;
  st = cuda_status(cudaMemcpyFromSymbol(&v, g_device_error, sizeof(v)));
  if (st == HG_OK) st = cuda_status(cudaMemcpyFromSymbol(&fault, g_device_fault, sizeof(fault)));
  if (st != HG_OK) return st;
  const int32_t zero = 0;
  st = cuda_status(cudaMemcpyToSymbol(g_device_error, &zero, sizeof(zero)));
  if (st == HG_OK) st = cuda_status(cudaMemcpyToSymbol(g_device_fault, &zero, sizeof(zero)));
  if (st != HG_OK) return st;
  *code = fault ? fault : v;
  return HG_OK;
}

extern "C" hg_status hg_debug_set_wait_limit(uint32_t polls, hg_stream_t stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  hg_status st = cuda_status(cudaStreamSynchronize(s));
  if (st != HG_OK) return st;
  const uint32_t v = polls ? polls : LOOKBACK_SPIN_LIMIT;
  return cuda_status(cudaMemcpyToSymbol(g_lookback_limit, &v, sizeof(v)));
}

// ---------------------------------------------------------------------------
// Build
// ---------------------------------------------------------------------------
static hg_status check_build_args(uint64_t n, int key_bytes, uint64_t n_buckets) {
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0) return HG_ERR_INVALID_ARGUMENT;
  if (n >= (1ull << 32) || n_buckets > (1ull << 32)) return HG_ERR_TOO_LARGE;
  return HG_OK;
}

extern "C" hg_status hg_build_workspace_size(uint64_t n, int key_bytes, uint64_t n_buckets, int with_index,
                                             size_t* bytes) {
  if (!bytes) return HG_ERR_INVALID_ARGUMENT;
  hg_status st = check_build_args(n, key_bytes, n_buckets);
  if (st != HG_OK) return st;
  BuildPlan plan;
  st = plan_build(n, key_bytes, n_buckets, with_index != 0, &plan);
  if (st != HG_OK) return st;
  *bytes = plan.total;
  return HG_OK;
}

// Internal: build with an explicit path choice (-1 = planner's choice).
extern "C" hg_status hg_build_into_path(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                                        uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out,
                                        void* d_workspace, size_t workspace_bytes, int path, hg_stream_t stream) {
  hg_status st = check_build_args(n, key_bytes, n_buckets);
  if (st != HG_OK) return st;
  if (!d_offsets || (n > 0 && (!d_keys || !d_keys_out)) || !d_workspace) return HG_ERR_INVALID_ARGUMENT;
  BuildPlan plan;
  st = plan_build(n, key_bytes, n_buckets, d_idx_out != nullptr, &plan, path);
  if (st != HG_OK) return st;
  if (workspace_bytes < plan.total) return HG_ERR_TOO_LARGE;
  return launch_build(plan, d_keys, d_offsets, d_keys_out, d_idx_out, d_workspace,
                      reinterpret_cast<cudaStream_t>(stream));
}

extern "C" hg_status hg_build_workspace_size_path(uint64_t n, int key_bytes, uint64_t n_buckets, int with_index,
                                                  int path, size_t* bytes) {
  if (!bytes) return HG_ERR_INVALID_ARGUMENT;
  BuildPlan plan;
  hg_status st = plan_build(n, key_bytes, n_buckets, with_index != 0, &plan, path);
  if (st != HG_OK) return st;
  *bytes = plan.total;
  return HG_OK;
}

extern "C" hg_status hg_build_into(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets,
                                   uint32_t* d_offsets, void* d_keys_out, uint32_t* d_idx_out, void* d_workspace,
                                   size_t workspace_bytes, hg_stream_t stream) {
  return hg_build_into_path(d_keys, n, key_bytes, n_buckets, d_offsets, d_keys_out, d_idx_out, d_workspace,
                            workspace_bytes, -1, stream);
}

// ---------------------------------------------------------------------------
// Tables
// ---------------------------------------------------------------------------
extern "C" void hg_table_free(hg_table* t) {
  if (!t) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(t->device);
  cudaFree(t->offsets);
  cudaFree(t->keys);
  cudaFree(t->idx);
  cudaFree(t->ws);
  if (prev >= 0) cudaSetDevice(prev);
  delete t;
}

extern "C" hg_status hg_table_create(uint64_t capacity, int key_bytes, uint64_t n_buckets, int with_index,
                                     hg_table** out) {
  if (!out) return HG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  hg_status st = check_build_args(capacity, key_bytes, n_buckets);
  if (st != HG_OK) return st;
  BuildPlan plan;
  st = plan_build(capacity, key_bytes, n_buckets, with_index != 0, &plan);
  if (st != HG_OK) return st;
  hg_table* t = new (std::nothrow) hg_table();
  if (!t) return HG_ERR_OUT_OF_MEMORY;
  cudaGetDevice(&t->device);
  t->capacity = capacity;
  t->n_buckets = n_buckets;
  t->key_bytes = key_bytes;
  t->with_index = with_index != 0;
  t->ws_bytes = plan.total;
  cudaError_t e = cudaMalloc(&t->offsets, (n_buckets + 1) * sizeof(uint32_t));
  if (e == cudaSuccess && capacity) e = cudaMalloc(&t->keys, capacity * key_bytes);
  if (e == cudaSuccess && capacity && with_index) e = cudaMalloc(&t->idx, capacity * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&t->ws, t->ws_bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    hg_table_free(t);
    return cuda_status(e);
  }
  *out = t;
  return HG_OK;
}

extern "C" hg_status hg_table_build(hg_table* t, const void* d_keys, uint64_t n, hg_stream_t stream) {
  if (!t || (n > 0 && !d_keys)) return HG_ERR_INVALID_ARGUMENT;
  if (n > t->capacity) return HG_ERR_TOO_LARGE;
  if (!t->ws) {  // a loaded table gets its build workspace on its first rebuild
    BuildPlan cap_plan;
    hg_status cst = plan_build(t->capacity, t->key_bytes, t->n_buckets, t->with_index, &cap_plan);
    if (cst != HG_OK) return cst;
    const cudaError_t e = cudaMalloc(&t->ws, cap_plan.total);
    if (e != cudaSuccess) {
      cudaGetLastError();
      t->ws = nullptr;
      return cuda_status(e);
    }
    t->ws_bytes = cap_plan.total;
  }
  BuildPlan plan;
  hg_status st = plan_build(n, t->key_bytes, t->n_buckets, t->with_index, &plan);
  if (st != HG_OK) return st;
  if (plan.total > t->ws_bytes) {
    // a smaller n can plan a different path; fall back to the capacity's path
    BuildPlan cap_plan;
    st = plan_build(t->capacity, t->key_bytes, t->n_buckets, t->with_index, &cap_plan);
    if (st != HG_OK) return st;
    st = plan_build(n, t->key_bytes, t->n_buckets, t->with_index, &plan, cap_plan.path);
    if (st != HG_OK) return st;
    if (plan.total > t->ws_bytes) return HG_ERR_TOO_LARGE;
  }
  st = launch_build(plan, d_keys, t->offsets, t->keys, t->idx, t->ws, reinterpret_cast<cudaStream_t>(stream));
  if (st != HG_OK) return st;
  t->n = n;
  t->built = true;
  return HG_OK;
}

extern "C" hg_status hg_build(const void* d_keys, uint64_t n, int key_bytes, uint64_t n_buckets, int with_index,
                              hg_table** out, hg_stream_t stream) {
  hg_table* t = nullptr;
  hg_status st = hg_table_create(n, key_bytes, n_buckets, with_index, &t);
  if (st != HG_OK) return st;
  st = hg_table_build(t, d_keys, n, stream);
  if (st != HG_OK) {
    hg_table_free(t);
    return st;
  }
  *out = t;
  return HG_OK;
}

extern "C" hg_status hg_table_view(const hg_table* t, const uint32_t** d_offsets, const void** d_keys,
                                   const uint32_t** d_idx, uint64_t* n, uint64_t* n_buckets, int* key_bytes) {
  if (!t) return HG_ERR_INVALID_ARGUMENT;
  if (d_offsets) *d_offsets = t->offsets;
  if (d_keys) *d_keys = t->keys;
  if (d_idx) *d_idx = t->idx;
  if (n) *n = t->n;
  if (n_buckets) *n_buckets = t->n_buckets;
  if (key_bytes) *key_bytes = t->key_bytes;
  return HG_OK;
}

extern "C" hg_status hg_table_device_bytes(const hg_table* t, size_t* bytes) {
  if (!t || !bytes) return HG_ERR_INVALID_ARGUMENT;
  *bytes = (t->n_buckets + 1) * 4 + t->capacity * t->key_bytes + (t->with_index ? t->capacity * 4 : 0) + t->ws_bytes;
  return HG_OK;
}

// ---------------------------------------------------------------------------
// Intersect
// ---------------------------------------------------------------------------
extern "C" hg_status hg_intersect_workspace_size(uint64_t n_a, int a_has_index, uint64_t n_buckets, uint64_t nq,
                                                 int key_bytes, int emit_pairs, size_t* bytes) {
  if (!bytes) return HG_ERR_INVALID_ARGUMENT;
  ProbePlan plan;
  hg_status st = plan_probe(n_a, a_has_index != 0, n_buckets, nq, key_bytes, emit_pairs != 0, &plan);
  if (st != HG_OK) return st;
  *bytes = plan.total;
  return HG_OK;
}

extern "C" hg_status hg_intersect_workspace_size_path(uint64_t n_a, int a_has_index, uint64_t n_buckets, uint64_t nq,
                                                      int key_bytes, int emit_pairs, int path, size_t* bytes) {
  if (!bytes) return HG_ERR_INVALID_ARGUMENT;
  ProbePlan plan;
  hg_status st = plan_probe(n_a, a_has_index != 0, n_buckets, nq, key_bytes, emit_pairs != 0, &plan, path);
  if (st != HG_OK) return st;
  *bytes = plan.total;
  return HG_OK;
}

extern "C" hg_status hg_intersect_into_path(const uint32_t* d_a_offsets, const void* d_a_keys, const uint32_t* d_a_idx,
                                            uint64_t n_a, uint64_t n_buckets, int key_bytes, const void* d_query,
                                            uint64_t nq, const uint32_t* d_query_idx, uint32_t* d_pairs,
                                            uint64_t pair_cap, unsigned long long* d_count, void* d_workspace,
                                            size_t workspace_bytes, int path, hg_stream_t stream) {
  if (!d_a_offsets || !d_count || (nq > 0 && !d_query) || (n_a > 0 && !d_a_keys)) return HG_ERR_INVALID_ARGUMENT;
  ProbePlan plan;
  hg_status st = plan_probe(n_a, d_a_idx != nullptr, n_buckets, nq, key_bytes, d_pairs != nullptr, &plan, path);
  if (st != HG_OK) return st;
  if (workspace_bytes < plan.total || (!d_workspace && plan.total)) return HG_ERR_TOO_LARGE;
  return launch_probe(plan, d_a_offsets, d_a_keys, d_a_idx, d_query, d_query_idx, d_pairs, pair_cap, d_count,
                      d_workspace, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" hg_status hg_intersect_into(const uint32_t* d_a_offsets, const void* d_a_keys, const uint32_t* d_a_idx,
                                       uint64_t n_a, uint64_t n_buckets, int key_bytes, const void* d_query,
                                       uint64_t nq, const uint32_t* d_query_idx, uint32_t* d_pairs,
                                       uint64_t pair_cap, unsigned long long* d_count, void* d_workspace,
                                       size_t workspace_bytes, hg_stream_t stream) {
  return hg_intersect_into_path(d_a_offsets, d_a_keys, d_a_idx, n_a, n_buckets, key_bytes, d_query, nq, d_query_idx,
                                d_pairs, pair_cap, d_count, d_workspace, workspace_bytes, -1, stream);
}

extern "C" hg_status hg_intersect(const hg_table* a, const void* d_query, uint64_t nq, const uint32_t* d_query_idx,
                                  uint32_t* d_pairs, uint64_t pair_cap, unsigned long long* d_count,
                                  hg_stream_t stream) {
  if (!a || !a->built) return HG_ERR_INVALID_ARGUMENT;
  size_t bytes = 0;
  hg_status st = hg_intersect_workspace_size(a->n, a->with_index, a->n_buckets, nq, a->key_bytes, d_pairs != nullptr,
                                             &bytes);
  if (st != HG_OK) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  void* ws = nullptr;
  cudaError_t e = cudaMallocAsync(&ws, bytes, s);
  if (e != cudaSuccess) return cuda_status(e);
  st = hg_intersect_into(a->offsets, a->keys, a->idx, a->n, a->n_buckets, a->key_bytes, d_query, nq, d_query_idx,
                         d_pairs, pair_cap, d_count, ws, bytes, stream);
  cudaFreeAsync(ws, s);
  return st;
}

extern "C" hg_status hg_intersect_tables(const hg_table* a, const hg_table* b, uint32_t* d_pairs, uint64_t pair_cap,
                                         unsigned long long* d_count, hg_stream_t stream) {
  if (!a || !b || !a->built || !b->built) return HG_ERR_INVALID_ARGUMENT;
  if (a->key_bytes != b->key_bytes) return HG_ERR_KEY_WIDTH;
  if (a->n_buckets != b->n_buckets) return HG_ERR_BUCKET_MISMATCH;
  return hg_intersect(a, b->keys, b->n, b->idx, d_pairs, pair_cap, d_count, stream);
}

// ---------------------------------------------------------------------------
// Instrumentation
// ---------------------------------------------------------------------------
extern "C" hg_status hg_profile_enable(int on) {
  Profiler& p = profiler();
  std::lock_guard<std::mutex> g(p.mu);
  p.on = on != 0;
  for (auto& r : p.recs) {
    p.pool.push_back(r.a);
    p.pool.push_back(r.b);
  }
  p.recs.clear();
  return HG_OK;
}

extern "C" hg_status hg_profile_read(int cap, int* count, const char** names, float* ms) {
  if (!count || (cap > 0 && (!names || !ms))) return HG_ERR_INVALID_ARGUMENT;
  Profiler& p = profiler();
  std::lock_guard<std::mutex> g(p.mu);
  int k = 0;
  hg_status st = HG_OK;
  for (auto& r : p.recs) {
    if (k < cap) {
      float t = 0.f;
      cudaError_t e = cudaEventSynchronize(r.b);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
      if (e != cudaSuccess) st = HG_ERR_CUDA;
      names[k] = r.name;
      ms[k] = t;
    }
    k++;
    p.pool.push_back(r.a);
    p.pool.push_back(r.b);
  }
  p.recs.clear();
  *count = k;
  return st;
}

extern "C" unsigned long long hg_launch_count(void) { return profiler().launches.load(); }
