// MultiHashGraph.cpp -- reference class API over the C ABI (see the header).
#include "hashgraph_b200/MultiHashGraph.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <mutex>
#include <vector>

namespace {
void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw hg::Error(e == cudaErrorMemoryAllocation ? HG_ERR_OUT_OF_MEMORY : HG_ERR_CUDA, what);
}

template <typename T>
T* dev_alloc(size_t count, const char* what) {
  void* p = nullptr;
  cuda_check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), what);
  return static_cast<T*>(p);
}

void dev_free(void* p) {
  if (p) cudaFree(p);
}

// The barrier the reference takes with `#pragma omp barrier` inside build()
// (include/MultiHashGraphHostOperators.cuh:45-62): every one of the gpuCount
// calling threads waits for the others.  Bounded: a thread that never comes
// turns into an error instead of a hang.
class HostBarrier {
 public:
  explicit HostBarrier(int n) : n_(n) {}
  void wait() {
    std::unique_lock<std::mutex> lk(m_);
    const uint64_t g = gen_;
    if (++waiting_ == n_) {
      waiting_ = 0;
      gen_++;
      cv_.notify_all();
      return;
    }
    if (!cv_.wait_for(lk, std::chrono::seconds(600), [&] { return gen_ != g; }))
      throw hg::Error(HG_ERR_DEVICE_TIMEOUT, "MultiHashGraph: a build thread did not arrive");
  }

 private:
  std::mutex m_;
  std::condition_variable cv_;
  int n_, waiting_ = 0;
  uint64_t gen_ = 0;
};
}  // namespace

// One shard (gpuCount > 1): buckets [lo, hi) on `device`.
struct MultiHashGraph::Shard {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint64_t lo = 0, hi = 0, n = 0;
  uint32_t* off = nullptr;
  hkey_t* keys = nullptr;
  uint32_t* idx = nullptr;
  // build scratch
  std::vector<unsigned long long> bins;
  std::vector<uint64_t> goff;  // routed group boundaries [gpuCount + 1]
  hkey_t* routed = nullptr;
  uint32_t* routed_idx = nullptr;
  hkey_t* recv = nullptr;
  uint32_t* recv_idx = nullptr;
  uint64_t n_recv = 0;
  void release_table() {
    dev_free(off);
    dev_free(keys);
    dev_free(idx);
    off = nullptr;
    keys = nullptr;
    idx = nullptr;
    n = 0;
  }
  void release_scratch() {
    dev_free(routed);
    dev_free(routed_idx);
    dev_free(recv);
    dev_free(recv_idx);
    routed = recv = nullptr;
    routed_idx = recv_idx = nullptr;
  }
};

struct MultiHashGraph::Multi {
  explicit Multi(int g) : barrier(g), shards(g) {}
  HostBarrier barrier;
  std::vector<Shard> shards;
};

MultiHashGraph::MultiHashGraph(inputData* vals, index_t countSize_, index_t maxkey_, index_t tableSize_,
                               index_t binCount_, index_t lrbBins_, index_t gpuCount_)
    : countSize(countSize_), tableSize(tableSize_), gpuCount(gpuCount_), h_dVals(vals), maxkey(maxkey_),
      binCount(binCount_), lrbBins(lrbBins_) {
  if (gpuCount < 1 || gpuCount > HG_MAX_SHARDS)
    throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph: gpuCount must be 1..64");
  if (!vals || countSize < 0 || tableSize < 1)
    throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph: inputData / sizes");
  index_t total = 0;
  for (index_t t = 0; t < gpuCount; t++) total += vals[t].len;
  if (total != countSize) throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph: inputData lengths != countSize");
  const int G = static_cast<int>(gpuCount);
  h_dFinalKeys = new char*[G]();
  h_hashOff = new index_t[G]();
  h_counterOff = new index_t[G]();
  h_offsetOff = new index_t[G]();
  h_edgesOff = new index_t[G]();
  h_lrbOff = new index_t[G]();
  ownSplits = new index_t[G + 1]();
  ownSplits[G] = tableSize;
  h_binSplits = ownSplits;
  h_dBinSplits = new index_t*[G]();
  if (G > 1) {
    multi = new Multi(G);
    int nd = 0;
    cuda_check(cudaGetDeviceCount(&nd), "MultiHashGraph: devices");
    for (int t = 0; t < G; t++) {
      // with fewer devices than gpuCount, shards share devices (t % count)
      multi->shards[t].device = t % nd;
      cuda_check(cudaSetDevice(multi->shards[t].device), "MultiHashGraph: device");
      cuda_check(cudaStreamCreateWithFlags(&multi->shards[t].stream, cudaStreamNonBlocking), "MultiHashGraph: stream");
    }
  }
  for (int t = 0; t < G; t++) {
    if (multi) cuda_check(cudaSetDevice(multi->shards[t].device), "MultiHashGraph: device");
    h_dBinSplits[t] = dev_alloc<index_t>(G + 1, "MultiHashGraph: splits");
    cuda_check(cudaMemcpy(h_dBinSplits[t], h_binSplits, (G + 1) * sizeof(index_t), cudaMemcpyHostToDevice),
               "MultiHashGraph: splits");
  }
  // host copy of the keys in global index order, as the reference keeps for
  // its checks (src/MultiHashGraph.cu:97-98)
  h_vals = new hkey_t[countSize ? countSize : 1]();
  index_t at = 0;
  for (int t = 0; t < G; t++) {
    if (multi) cuda_check(cudaSetDevice(multi->shards[t].device), "MultiHashGraph: device");
    if (vals[t].len)
      cuda_check(cudaMemcpy(h_vals + at, vals[t].d_keys, vals[t].len * sizeof(hkey_t), cudaMemcpyDeviceToHost),
                 "MultiHashGraph: key copy");
    at += vals[t].len;
  }
  if (multi) cuda_check(cudaSetDevice(multi->shards[0].device), "MultiHashGraph: device");
}

MultiHashGraph::~MultiHashGraph() {
  if (tbl) hg_table_free(tbl);
  const int G = static_cast<int>(gpuCount);
  for (int t = 0; t < G; t++) {
    if (multi) cudaSetDevice(multi->shards[t].device);
    if (h_dFinalKeys) dev_free(h_dFinalKeys[t]);
    if (h_dBinSplits) dev_free(h_dBinSplits[t]);
    if (multi) {
      Shard& sh = multi->shards[t];
      sh.release_table();
      sh.release_scratch();
      if (sh.stream) cudaStreamDestroy(sh.stream);
    }
  }
  delete multi;
  delete[] h_dFinalKeys;
  delete[] h_hashOff;
  delete[] h_counterOff;
  delete[] h_offsetOff;
  delete[] h_edgesOff;
  delete[] h_lrbOff;
  delete[] ownSplits;
  delete[] h_dBinSplits;
  delete[] h_vals;
}

void MultiHashGraph::build(bool findSplits, index_t tid) {
  if (tid < 0 || tid >= gpuCount) throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph::build: tid");
  if (multi) {
    buildShard(findSplits, static_cast<int>(tid));
    return;
  }
  // one GPU: the whole table, with the planner's choice of path
  if (!tbl)
    hg::check(hg_table_create(countSize, sizeof(hkey_t), tableSize, /*with_index=*/1, &tbl),
              "MultiHashGraph::build: table");
  hg::check(hg_table_build(tbl, h_dVals[0].d_keys, countSize, nullptr), "MultiHashGraph::build");
  if (exportLayout) {
    const uint32_t* off;
    const void* keys;
    const uint32_t* idx;
    uint64_t n, nb;
    int kb;
    hg::check(hg_table_view(tbl, &off, &keys, &idx, &n, &nb, &kb), "MultiHashGraph: view");
    exportReferenceLayout(0, off, keys, idx, n, nb, nullptr);
  }
}

// gpuCount > 1: the reference's pipeline (src/MultiHashGraph.cu:408-629) on
// the sharding calls -- bin histogram, splits, route, copies to the owning
// devices, shard build -- with this object's barrier where the reference
// takes `omp barrier`.
void MultiHashGraph::buildShard(bool findSplits, int tid) {
  const int G = static_cast<int>(gpuCount);
  Shard& sh = multi->shards[tid];
  cuda_check(cudaSetDevice(sh.device), "build: device");
  cudaStream_t st = sh.stream;
  hg_stream_t hs = reinterpret_cast<hg_stream_t>(st);
  const uint64_t n = static_cast<uint64_t>(h_dVals[tid].len);
  const hkey_t* d_in = h_dVals[tid].d_keys;
  uint64_t index_base = 0;
  for (int t = 0; t < tid; t++) index_base += static_cast<uint64_t>(h_dVals[t].len);
  if (findSplits) {
    const uint32_t nb = static_cast<uint32_t>(std::min<index_t>(std::max<index_t>(binCount, 1), 32768));
    unsigned long long* d_bins = dev_alloc<unsigned long long>(nb, "build: bins");
    cuda_check(cudaMemsetAsync(d_bins, 0, nb * sizeof(unsigned long long), st), "build: bins");
    hg::check(hg_shard_histogram(d_in, n, sizeof(hkey_t), tableSize, nb, d_bins, hs), "build: histogram");
    sh.bins.assign(nb, 0);
    cuda_check(cudaMemcpyAsync(sh.bins.data(), d_bins, nb * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
               "build: bins");
    cuda_check(cudaStreamSynchronize(st), "build: bins");
    dev_free(d_bins);
    multi->barrier.wait();
    if (tid == 0) {
      std::vector<unsigned long long> sum(nb, 0);
      for (int t = 0; t < G; t++)
        for (uint32_t i = 0; i < nb; i++) sum[i] += multi->shards[t].bins[i];
      std::vector<uint64_t> sp(G + 1);
      hg::check(hg_shard_splits(sum.data(), nb, tableSize, G, sp.data()), "build: splits");
      for (int r = 0; r <= G; r++) ownSplits[r] = static_cast<index_t>(sp[r]);
      h_binSplits = ownSplits;
    }
    multi->barrier.wait();
    cuda_check(cudaMemcpyAsync(h_dBinSplits[tid], h_binSplits, (G + 1) * sizeof(index_t), cudaMemcpyHostToDevice, st),
               "build: splits");
  }
  std::vector<uint64_t> splits(G + 1);
  for (int r = 0; r <= G; r++) splits[r] = static_cast<uint64_t>(h_binSplits[r]);
  // route: the keys grouped by owning shard, with their global indices
  size_t ws_bytes = 0;
  hg::check(hg_shard_route_workspace_size(n, G, &ws_bytes), "build: route workspace");
  char* ws = dev_alloc<char>(ws_bytes, "build: route workspace");
  unsigned long long* d_goff = dev_alloc<unsigned long long>(G + 1, "build: groups");
  sh.release_scratch();
  sh.routed = dev_alloc<hkey_t>(n, "build: routed");
  sh.routed_idx = dev_alloc<uint32_t>(n, "build: routed");
  hg::check(hg_shard_route(d_in, n, sizeof(hkey_t), tableSize, splits.data(), G, static_cast<uint32_t>(index_base),
                           sh.routed, sh.routed_idx, d_goff, ws, ws_bytes, hs),
            "build: route");
  std::vector<unsigned long long> goff(G + 1);
  cuda_check(cudaMemcpyAsync(goff.data(), d_goff, (G + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
             "build: groups");
  cuda_check(cudaStreamSynchronize(st), "build: route");
  dev_free(ws);
  dev_free(d_goff);
  sh.goff.assign(goff.begin(), goff.end());
  multi->barrier.wait();
  // receive buffers: every sender's group for this shard, in sender order
  sh.n_recv = 0;
  for (int s = 0; s < G; s++) sh.n_recv += multi->shards[s].goff[tid + 1] - multi->shards[s].goff[tid];
  sh.recv = dev_alloc<hkey_t>(sh.n_recv, "build: receive");
  sh.recv_idx = dev_alloc<uint32_t>(sh.n_recv, "build: receive");
  multi->barrier.wait();
  // send: each group to its owner (the reference's peer copies)
  for (int d = 0; d < G; d++) {
    Shard& dst = multi->shards[d];
    const uint64_t cnt = sh.goff[d + 1] - sh.goff[d];
    if (!cnt) continue;
    uint64_t at = 0;
    for (int s = 0; s < tid; s++) at += multi->shards[s].goff[d + 1] - multi->shards[s].goff[d];
    cuda_check(cudaMemcpyPeerAsync(dst.recv + at, dst.device, sh.routed + sh.goff[d], sh.device, cnt * sizeof(hkey_t),
                                   st),
               "build: send keys");
    cuda_check(cudaMemcpyPeerAsync(dst.recv_idx + at, dst.device, sh.routed_idx + sh.goff[d], sh.device, cnt * 4, st),
               "build: send indices");
  }
  cuda_check(cudaStreamSynchronize(st), "build: send");
  multi->barrier.wait();
  // the shard's table over its bucket range
  sh.release_table();
  sh.lo = splits[tid];
  sh.hi = splits[tid + 1];
  sh.n = sh.n_recv;
  if (sh.hi > sh.lo) {
    size_t bws = 0;
    hg::check(hg_build_workspace_size(sh.n, sizeof(hkey_t), sh.hi - sh.lo, 1, &bws), "build: workspace");
    char* bw = dev_alloc<char>(bws, "build: workspace");
    sh.off = dev_alloc<uint32_t>(sh.hi - sh.lo + 1, "build: offsets");
    sh.keys = dev_alloc<hkey_t>(sh.n, "build: keys");
    sh.idx = dev_alloc<uint32_t>(sh.n, "build: index");
    hg::check(hg_shard_build_into(sh.recv, sh.recv_idx, sh.n, sizeof(hkey_t), tableSize, sh.lo, sh.hi, sh.off,
                                  sh.keys, sh.idx, bw, bws, hs),
              "build: shard");
    cuda_check(cudaStreamSynchronize(st), "build: shard");
    dev_free(bw);
    if (exportLayout) exportReferenceLayout(tid, sh.off, sh.keys, sh.idx, sh.n, sh.hi - sh.lo, hs);
  }
  cuda_check(cudaStreamSynchronize(st), "build");
  multi->barrier.wait();  // every sender's copies into and out of this shard are done
  sh.release_scratch();
}

void MultiHashGraph::exportReferenceLayout(int tid, const uint32_t* off, const void* keys, const uint32_t* idx,
                                           uint64_t n, uint64_t nb, hg_stream_t stream) {
  // compact arena: [edges: n keyval_ind | offsets: nb + 1 int64]
  const size_t edges_bytes = static_cast<size_t>(n) * sizeof(keyval_ind);
  const size_t off_bytes = (static_cast<size_t>(nb) + 1) * sizeof(index_t);
  dev_free(h_dFinalKeys[tid]);
  h_dFinalKeys[tid] = dev_alloc<char>(edges_bytes + off_bytes, "MultiHashGraph: arena");
  h_edgesOff[tid] = 0;
  h_offsetOff[tid] = static_cast<index_t>(edges_bytes);
  h_hashOff[tid] = h_counterOff[tid] = h_lrbOff[tid] = 0;  // not populated: no hash / counter / LRB arrays exist
  hg::check(hg_export_reference_layout(off, keys, idx, n, nb, sizeof(hkey_t), h_dFinalKeys[tid] + h_edgesOff[tid],
                                       reinterpret_cast<int64_t*>(h_dFinalKeys[tid] + h_offsetOff[tid]), stream),
            "MultiHashGraph: export");
  if (stream) cuda_check(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)), "MultiHashGraph: export");
}

void MultiHashGraph::intersect(MultiHashGraph& A, MultiHashGraph& B, index_t* h_Common, keypair** h_dOutput,
                               index_t tid) {
  if (A.gpuCount != B.gpuCount || tid < 0 || tid >= A.gpuCount)
    throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph::intersect: tid / gpuCount");
  if (A.tableSize != B.tableSize)
    throw hg::Error(HG_ERR_BUCKET_MISMATCH, "MultiHashGraph::intersect: table sizes differ");
  if (A.multi) {
    intersectShard(A, B, h_Common, h_dOutput, static_cast<int>(tid));
    return;
  }
  if (!A.tbl || !B.tbl) throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph::intersect: build both first");
  unsigned long long* d_count = dev_alloc<unsigned long long>(1, "intersect: count");
  // pass 1 counts (as the reference's simpleIntersect count pass), pass 2 emits
  hg::check(hg_intersect_tables(A.tbl, B.tbl, nullptr, 0, d_count, nullptr), "intersect: count");
  unsigned long long count = 0;
  cuda_check(cudaMemcpy(&count, d_count, sizeof(count), cudaMemcpyDeviceToHost), "intersect: count");
  h_Common[tid] = static_cast<index_t>(count);
  h_dOutput[tid] = nullptr;
  if (count > 0) {
    uint32_t* d_pairs = dev_alloc<uint32_t>(count * 2, "intersect: pairs");
    h_dOutput[tid] = dev_alloc<keypair>(count, "intersect: output");
    // q_ref is B's input position (B is built with its index); B's key per
    // match is the query key at that position
    hg::check(hg_intersect_tables(A.tbl, B.tbl, d_pairs, count, d_count, nullptr), "intersect: emit");
    hg::check(hg_gather_pair_keys(B.h_dVals[0].d_keys, sizeof(hkey_t), d_pairs, count, 1,
                                  reinterpret_cast<int64_t*>(h_dOutput[tid]), nullptr),
              "intersect: keys");
    cuda_check(cudaDeviceSynchronize(), "intersect");
    cudaFree(d_pairs);
  }
  cudaFree(d_count);
}

// gpuCount > 1: shard tid of A against shard tid of B (B built on A's
// splits, the reference's build(false, tid)); h_Common[tid] and
// h_dOutput[tid] (on shard tid's device) as the reference fills them.
void MultiHashGraph::intersectShard(MultiHashGraph& A, MultiHashGraph& B, index_t* h_Common, keypair** h_dOutput,
                                    int tid) {
  Shard& a = A.multi->shards[tid];
  Shard& b = B.multi->shards[tid];
  if (a.lo != b.lo || a.hi != b.hi)
    throw hg::Error(HG_ERR_BUCKET_MISMATCH, "MultiHashGraph::intersect: B was not built on A's splits");
  h_Common[tid] = 0;
  h_dOutput[tid] = nullptr;
  if (a.hi == a.lo || a.n == 0 || b.n == 0) return;
  cuda_check(cudaSetDevice(a.device), "intersect: device");
  cudaStream_t st = a.stream;
  hg_stream_t hs = reinterpret_cast<hg_stream_t>(st);
  size_t ws_bytes = 0, ws_count = 0;
  hg::check(hg_intersect_workspace_size(a.n, 1, a.hi - a.lo, b.n, sizeof(hkey_t), 1, &ws_bytes), "intersect: ws");
  hg::check(hg_intersect_workspace_size(a.n, 1, a.hi - a.lo, b.n, sizeof(hkey_t), 0, &ws_count), "intersect: ws");
  ws_bytes = std::max(ws_bytes, ws_count);
  char* ws = dev_alloc<char>(ws_bytes, "intersect: workspace");
  unsigned long long* d_count = dev_alloc<unsigned long long>(1, "intersect: count");
  hg::check(hg_shard_intersect_into(a.off, a.keys, a.idx, a.n, A.tableSize, a.lo, a.hi, sizeof(hkey_t), b.keys, b.n,
                                    nullptr, nullptr, 0, d_count, ws, ws_bytes, hs),
            "intersect: count");
  unsigned long long count = 0;
  cuda_check(cudaMemcpyAsync(&count, d_count, sizeof(count), cudaMemcpyDeviceToHost, st), "intersect: count");
  cuda_check(cudaStreamSynchronize(st), "intersect: count");
  h_Common[tid] = static_cast<index_t>(count);
  if (count > 0) {
    uint32_t* d_pairs = dev_alloc<uint32_t>(count * 2, "intersect: pairs");
    h_dOutput[tid] = dev_alloc<keypair>(count, "intersect: output");
    // q_ref = position in B's shard (no query index given): B's key per match
    hg::check(hg_shard_intersect_into(a.off, a.keys, a.idx, a.n, A.tableSize, a.lo, a.hi, sizeof(hkey_t), b.keys, b.n,
                                      nullptr, d_pairs, count, d_count, ws, ws_bytes, hs),
              "intersect: emit");
    hg::check(hg_gather_pair_keys(b.keys, sizeof(hkey_t), d_pairs, count, 1,
                                  reinterpret_cast<int64_t*>(h_dOutput[tid]), hs),
              "intersect: keys");
    cuda_check(cudaStreamSynchronize(st), "intersect");
    dev_free(d_pairs);
  }
  dev_free(ws);
  dev_free(d_count);
}

void MultiHashGraph::buildSingle() {
  // The reference rebuilds the table with the plain single-table path and
  // compares degrees and sorted bucket contents (src/MultiHashGraph.cu:742-862);
  // with several shards, each shard's range of the single table.
  const size_t n = static_cast<size_t>(countSize), B = static_cast<size_t>(tableSize);
  const int G = static_cast<int>(gpuCount);
  const int dev0 = multi ? multi->shards[0].device : 0;
  cuda_check(cudaSetDevice(dev0), "buildSingle");
  hkey_t* d_all = dev_alloc<hkey_t>(n, "buildSingle");
  if (n) cuda_check(cudaMemcpy(d_all, h_vals, n * sizeof(hkey_t), cudaMemcpyHostToDevice), "buildSingle");
  uint32_t* d_off = dev_alloc<uint32_t>(B + 1, "buildSingle");
  hkey_t* d_keys = dev_alloc<hkey_t>(n, "buildSingle");
  size_t ws = 0;
  hg::check(hg_build_workspace_size_path(n, sizeof(hkey_t), B, 0, 0, &ws), "buildSingle");
  char* d_ws = dev_alloc<char>(ws, "buildSingle");
  hg::check(hg_build_into_path(d_all, n, sizeof(hkey_t), B, d_off, d_keys, nullptr, d_ws, ws, 0, nullptr),
            "buildSingle");
  std::vector<uint32_t> so(B + 1);
  std::vector<hkey_t> sk(n);
  cuda_check(cudaMemcpy(so.data(), d_off, (B + 1) * 4, cudaMemcpyDeviceToHost), "buildSingle");
  if (n) cuda_check(cudaMemcpy(sk.data(), d_keys, n * sizeof(hkey_t), cudaMemcpyDeviceToHost), "buildSingle");
  dev_free(d_all);
  dev_free(d_off);
  dev_free(d_keys);
  dev_free(d_ws);
  for (int t = 0; t < G; t++) {
    // shard t as the reference's public fields expose it (or the native arrays)
    const uint64_t lo = multi ? multi->shards[t].lo : 0, hi = multi ? multi->shards[t].hi : B;
    const uint64_t nb = hi - lo;
    if (nb == 0) continue;
    std::vector<uint32_t> mo(nb + 1);
    std::vector<hkey_t> mk;
    if (multi) cuda_check(cudaSetDevice(multi->shards[t].device), "buildSingle");
    if (exportLayout && h_dFinalKeys[t]) {
      std::vector<index_t> o64(nb + 1);
      cuda_check(cudaMemcpy(o64.data(), h_dFinalKeys[t] + h_offsetOff[t], (nb + 1) * sizeof(index_t),
                            cudaMemcpyDeviceToHost), "buildSingle");
      const size_t m = static_cast<size_t>(o64[nb]);
      std::vector<keyval_ind> kv(m);
      if (m) cuda_check(cudaMemcpy(kv.data(), h_dFinalKeys[t] + h_edgesOff[t], m * sizeof(keyval_ind),
                                   cudaMemcpyDeviceToHost), "buildSingle");
      for (uint64_t b = 0; b <= nb; b++) mo[b] = static_cast<uint32_t>(o64[b]);
      mk.resize(m);
      for (size_t j = 0; j < m; j++) {
        mk[j] = kv[j].key;
        if (kv[j].ind < 0 || static_cast<size_t>(kv[j].ind) >= n || h_vals[kv[j].ind] != kv[j].key)
          std::fprintf(stderr, "Index error edge: %zu\n", j);
      }
    } else if (multi) {
      const Shard& sh = multi->shards[t];
      mk.resize(sh.n);
      cuda_check(cudaMemcpy(mo.data(), sh.off, (nb + 1) * 4, cudaMemcpyDeviceToHost), "buildSingle");
      if (sh.n) cuda_check(cudaMemcpy(mk.data(), sh.keys, sh.n * sizeof(hkey_t), cudaMemcpyDeviceToHost), "buildSingle");
    } else {
      const uint32_t* off;
      const void* keys;
      uint64_t tn, tb;
      int kb;
      hg::check(hg_table_view(tbl, &off, &keys, nullptr, &tn, &tb, &kb), "buildSingle");
      mk.resize(n);
      cuda_check(cudaMemcpy(mo.data(), off, (B + 1) * 4, cudaMemcpyDeviceToHost), "buildSingle");
      if (n) cuda_check(cudaMemcpy(mk.data(), keys, n * sizeof(hkey_t), cudaMemcpyDeviceToHost), "buildSingle");
    }
    for (uint64_t b = 0; b < nb; b++) {
      const uint64_t g = lo + b;
      const int64_t md = int64_t(mo[b + 1]) - mo[b], sd = int64_t(so[g + 1]) - so[g];
      if (md != sd) {
        std::fprintf(stderr, "Degree error hash: %llu multi: %lld single: %lld\n", (unsigned long long)g,
                     (long long)md, (long long)sd);
        continue;
      }
      std::vector<hkey_t> x(mk.begin() + mo[b], mk.begin() + mo[b + 1]), y(sk.begin() + so[g], sk.begin() + so[g + 1]);
      std::sort(x.begin(), x.end());
      std::sort(y.begin(), y.end());
      if (x != y) std::fprintf(stderr, "List error\n");
    }
  }
  if (multi) cuda_check(cudaSetDevice(dev0), "buildSingle");
}

void MultiHashGraph::destroyMulti() {}
