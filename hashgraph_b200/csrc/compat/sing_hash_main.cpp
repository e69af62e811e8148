// sing_hash_main.cpp -- the reference's SingleHashGraph test main
// (alokpathy/hashgraph test/SingleHashGraphTest.cu:18-60) over the drop-in
// class: arguments `countSize maxkey lrbBins`, tableSize = maxkey, one timed
// build, "single buildTable() time: <s>".
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "hashgraph_b200/SingleHashGraph.h"

int main(int argc, char** argv) {
  int64_t countSize = 1L << 24, maxkey = 1L << 26, lrbBins = 16000;
  if (argc >= 3 && argc < 4) {
    std::fprintf(stderr, "Please specify all arguments.\n");
    return 1;
  }
  if (argc >= 4) {
    countSize = std::atoll(argv[1]);
    maxkey = std::atoll(argv[2]);
    lrbBins = std::atoll(argv[3]);
  }
  const int64_t tableSize = maxkey;
  try {
    SingleHashGraph shg(countSize, maxkey, tableSize, lrbBins);
    cudaEvent_t start, stop;
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
    cudaEventRecord(start);
    shg.build(countSize, tableSize);
    cudaEventRecord(stop);
    cudaEventSynchronize(stop);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, start, stop);
    std::printf("single buildTable() time: %g\n", ms / 1000.0);
  } catch (const hg::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  return 0;
}
