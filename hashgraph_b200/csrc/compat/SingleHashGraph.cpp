// SingleHashGraph.cpp -- reference class API over the C ABI (see the header).
#include "hashgraph_b200/SingleHashGraph.h"

#include <cuda_runtime.h>

namespace {
void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw hg::Error(e == cudaErrorMemoryAllocation ? HG_ERR_OUT_OF_MEMORY : HG_ERR_CUDA, what);
}
constexpr uint64_t SINGLE_KEY_SEED = 0;  // the reference seeds its generator with 0 (src/SingleHashGraph.cu:116)
}  // namespace

SingleHashGraph::SingleHashGraph(int64_t countSize_, int64_t maxkey, int64_t tableSize_, int64_t lrbBins_)
    : countSize(countSize_), tableSize(tableSize_), lrbBins(lrbBins_) {
  if (countSize < 0 || tableSize < 1 || maxkey < 0) throw hg::Error(HG_ERR_INVALID_ARGUMENT, "SingleHashGraph");
  const size_t n = static_cast<size_t>(countSize);
  cuda_check(cudaMalloc(&d_vals, (n ? n : 1) * sizeof(hkey_t)), "SingleHashGraph: keys");
  cuda_check(cudaMalloc(&d_offset, (static_cast<size_t>(tableSize) + 1) * sizeof(uint32_t)), "SingleHashGraph: offsets");
  cuda_check(cudaMalloc(&d_edges, (n ? n : 1) * sizeof(hkey_t)), "SingleHashGraph: edges");
  hg::check(hg_build_workspace_size(n, sizeof(hkey_t), tableSize, 0, &ws_bytes), "SingleHashGraph: workspace size");
  cuda_check(cudaMalloc(&d_ws, ws_bytes), "SingleHashGraph: workspace");
  // keys uniform in [0, maxkey], generated on the device as the reference does
  hg::check(hg_gen_bounded(d_vals, n, sizeof(hkey_t), SINGLE_KEY_SEED, static_cast<uint64_t>(maxkey) + 1, nullptr),
            "SingleHashGraph: key generation");
}

SingleHashGraph::~SingleHashGraph() {
  cudaFree(d_vals);
  cudaFree(d_offset);
  cudaFree(d_edges);
  cudaFree(d_ws);
}

void SingleHashGraph::build(int64_t n, int64_t nbuckets) {
  if (n < 0 || n > countSize || nbuckets != tableSize)
    throw hg::Error(HG_ERR_INVALID_ARGUMENT, "SingleHashGraph::build: sizes differ from the constructor's");
  hg::check(hg_build_into(d_vals, static_cast<uint64_t>(n), sizeof(hkey_t), static_cast<uint64_t>(nbuckets), d_offset,
                          d_edges, nullptr, d_ws, ws_bytes, nullptr),
            "SingleHashGraph::build");
}
