// MultiHashGraph.cpp -- reference class API over the C ABI (see the header).
#include "hashgraph_b200/MultiHashGraph.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

namespace {
void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw hg::Error(e == cudaErrorMemoryAllocation ? HG_ERR_OUT_OF_MEMORY : HG_ERR_CUDA, what);
}
}  // namespace

MultiHashGraph::MultiHashGraph(inputData* vals, index_t countSize_, index_t maxkey_, index_t tableSize_,
                               index_t binCount_, index_t lrbBins_, index_t gpuCount_)
    : countSize(countSize_), tableSize(tableSize_), gpuCount(gpuCount_), h_dVals(vals), maxkey(maxkey_),
      binCount(binCount_), lrbBins(lrbBins_) {
  if (gpuCount != 1)
    throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph: this build covers one GPU (gpuCount must be 1)");
  if (!vals || countSize < 0 || tableSize < 1 || vals[0].len != countSize)
    throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph: inputData / sizes");
  h_dFinalKeys = new char*[1]();
  h_hashOff = new index_t[1]();
  h_counterOff = new index_t[1]();
  h_offsetOff = new index_t[1]();
  h_edgesOff = new index_t[1]();
  h_lrbOff = new index_t[1]();
  h_binSplits = new index_t[2]{0, tableSize};
  h_dBinSplits = new index_t*[1]();
  cuda_check(cudaMalloc(&h_dBinSplits[0], 2 * sizeof(index_t)), "MultiHashGraph: splits");
  cuda_check(cudaMemcpy(h_dBinSplits[0], h_binSplits, 2 * sizeof(index_t), cudaMemcpyHostToDevice),
             "MultiHashGraph: splits");
  // host copy of the keys, as the reference keeps for its checks (src/MultiHashGraph.cu:97-98)
  h_vals = new hkey_t[countSize ? countSize : 1]();
  if (countSize)
    cuda_check(cudaMemcpy(h_vals, vals[0].d_keys, countSize * sizeof(hkey_t), cudaMemcpyDeviceToHost),
               "MultiHashGraph: key copy");
}

MultiHashGraph::~MultiHashGraph() {
  if (tbl) hg_table_free(tbl);
  if (h_dFinalKeys) cudaFree(h_dFinalKeys[0]);
  if (h_dBinSplits) cudaFree(h_dBinSplits[0]);
  delete[] h_dFinalKeys;
  delete[] h_hashOff;
  delete[] h_counterOff;
  delete[] h_offsetOff;
  delete[] h_edgesOff;
  delete[] h_lrbOff;
  delete[] h_binSplits;
  delete[] h_dBinSplits;
  delete[] h_vals;
}

void MultiHashGraph::build(bool /*findSplits*/, index_t tid) {
  if (tid != 0) throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph::build: tid must be 0 (one GPU)");
  if (!tbl)
    hg::check(hg_table_create(countSize, sizeof(hkey_t), tableSize, /*with_index=*/1, &tbl),
              "MultiHashGraph::build: table");
  hg::check(hg_table_build(tbl, h_dVals[0].d_keys, countSize, nullptr), "MultiHashGraph::build");
  if (exportLayout) exportReferenceLayout();
}

void MultiHashGraph::exportReferenceLayout() {
  // compact arena: [edges: countSize keyval_ind | offsets: tableSize+1 int64]
  const size_t edges_bytes = static_cast<size_t>(countSize) * sizeof(keyval_ind);
  const size_t off_bytes = (static_cast<size_t>(tableSize) + 1) * sizeof(index_t);
  if (!h_dFinalKeys[0])
    cuda_check(cudaMalloc(&h_dFinalKeys[0], edges_bytes + off_bytes), "MultiHashGraph: arena");
  h_edgesOff[0] = 0;
  h_offsetOff[0] = static_cast<index_t>(edges_bytes);
  h_hashOff[0] = h_counterOff[0] = h_lrbOff[0] = 0;  // not populated: no hash / counter / LRB arrays exist
  const uint32_t* off;
  const void* keys;
  const uint32_t* idx;
  uint64_t n, nb;
  int kb;
  hg::check(hg_table_view(tbl, &off, &keys, &idx, &n, &nb, &kb), "MultiHashGraph: view");
  hg::check(hg_export_reference_layout(off, keys, idx, n, nb, kb, h_dFinalKeys[0] + h_edgesOff[0],
                                       reinterpret_cast<int64_t*>(h_dFinalKeys[0] + h_offsetOff[0]), nullptr),
            "MultiHashGraph: export");
}

void MultiHashGraph::intersect(MultiHashGraph& A, MultiHashGraph& B, index_t* h_Common, keypair** h_dOutput,
                               index_t tid) {
  if (tid != 0) throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph::intersect: tid must be 0 (one GPU)");
  if (!A.tbl || !B.tbl) throw hg::Error(HG_ERR_INVALID_ARGUMENT, "MultiHashGraph::intersect: build both first");
  if (A.tableSize != B.tableSize)
    throw hg::Error(HG_ERR_BUCKET_MISMATCH, "MultiHashGraph::intersect: table sizes differ");
  unsigned long long* d_count = nullptr;
  cuda_check(cudaMalloc(&d_count, sizeof(unsigned long long)), "intersect: count");
  // pass 1 counts (as the reference's simpleIntersect count pass), pass 2 emits
  hg::check(hg_intersect_tables(A.tbl, B.tbl, nullptr, 0, d_count, nullptr), "intersect: count");
  unsigned long long count = 0;
  cuda_check(cudaMemcpy(&count, d_count, sizeof(count), cudaMemcpyDeviceToHost), "intersect: count");
  h_Common[tid] = static_cast<index_t>(count);
  h_dOutput[tid] = nullptr;
  if (count > 0) {
    uint32_t* d_pairs = nullptr;
    cuda_check(cudaMalloc(&d_pairs, count * 2 * sizeof(uint32_t)), "intersect: pairs");
    cuda_check(cudaMalloc(&h_dOutput[tid], count * sizeof(keypair)), "intersect: output");
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

void MultiHashGraph::buildSingle() {
  // The reference rebuilds the table with the plain single-table path and
  // compares degrees and sorted bucket contents (src/MultiHashGraph.cu:742-862).
  const size_t n = static_cast<size_t>(countSize), B = static_cast<size_t>(tableSize);
  uint32_t* d_off = nullptr;
  hkey_t* d_keys = nullptr;
  void* d_ws = nullptr;
  size_t ws = 0;
  hg::check(hg_build_workspace_size_path(n, sizeof(hkey_t), B, 0, 0, &ws), "buildSingle");
  cuda_check(cudaMalloc(&d_off, (B + 1) * sizeof(uint32_t)), "buildSingle");
  cuda_check(cudaMalloc(&d_keys, (n ? n : 1) * sizeof(hkey_t)), "buildSingle");
  cuda_check(cudaMalloc(&d_ws, ws), "buildSingle");
  hg::check(hg_build_into_path(h_dVals[0].d_keys, n, sizeof(hkey_t), B, d_off, d_keys, nullptr, d_ws, ws, 0, nullptr),
            "buildSingle");
  std::vector<uint32_t> so(B + 1), mo(B + 1);
  std::vector<hkey_t> sk(n), mk(n);
  cuda_check(cudaMemcpy(so.data(), d_off, (B + 1) * 4, cudaMemcpyDeviceToHost), "buildSingle");
  if (n) cuda_check(cudaMemcpy(sk.data(), d_keys, n * sizeof(hkey_t), cudaMemcpyDeviceToHost), "buildSingle");
  if (exportLayout && h_dFinalKeys[0]) {
    // the table as the reference's public fields expose it
    std::vector<index_t> o64(B + 1);
    std::vector<keyval_ind> kv(n);
    cuda_check(cudaMemcpy(o64.data(), h_dFinalKeys[0] + h_offsetOff[0], (B + 1) * sizeof(index_t),
                          cudaMemcpyDeviceToHost), "buildSingle");
    if (n) cuda_check(cudaMemcpy(kv.data(), h_dFinalKeys[0] + h_edgesOff[0], n * sizeof(keyval_ind),
                                 cudaMemcpyDeviceToHost), "buildSingle");
    for (size_t b = 0; b <= B; b++) mo[b] = static_cast<uint32_t>(o64[b]);
    for (size_t j = 0; j < n; j++) {
      mk[j] = kv[j].key;
      if (kv[j].ind < 0 || static_cast<size_t>(kv[j].ind) >= n || h_vals[kv[j].ind] != kv[j].key)
        std::fprintf(stderr, "Index error edge: %zu\n", j);
    }
  } else {
    const uint32_t* off;
    const void* keys;
    uint64_t tn, tb;
    int kb;
    hg::check(hg_table_view(tbl, &off, &keys, nullptr, &tn, &tb, &kb), "buildSingle");
    cuda_check(cudaMemcpy(mo.data(), off, (B + 1) * 4, cudaMemcpyDeviceToHost), "buildSingle");
    if (n) cuda_check(cudaMemcpy(mk.data(), keys, n * sizeof(hkey_t), cudaMemcpyDeviceToHost), "buildSingle");
  }
  for (size_t b = 0; b < B; b++) {
    const int64_t md = int64_t(mo[b + 1]) - mo[b], sd = int64_t(so[b + 1]) - so[b];
    if (md != sd) std::fprintf(stderr, "Degree error hash: %zu multi: %lld single: %lld\n", b, (long long)md, (long long)sd);
    std::vector<hkey_t> x(mk.begin() + mo[b], mk.begin() + mo[b + 1]), y(sk.begin() + so[b], sk.begin() + so[b + 1]);
    std::sort(x.begin(), x.end());
    std::sort(y.begin(), y.end());
    if (x != y) std::fprintf(stderr, "List error\n");
  }
  cudaFree(d_off);
  cudaFree(d_keys);
  cudaFree(d_ws);
}

void MultiHashGraph::destroyMulti() {}
