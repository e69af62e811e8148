// multi_hash_main.cpp -- the reference's MultiHashGraph test main
// (alokpathy/hashgraph test/MultiHashGraphTest.cu:130-427) rewritten over the
// drop-in classes: same positional arguments
//   multi-hash size maxkey binCount gpuCount lrbBins check|nocheck countSizeB build|intersect
// same inputs (sequential keys A = 0..size-1, B = 0..countSizeB-1), same
// timed regions (CUDA events around build, and around build A + build B +
// intersect) and the same "multi ... time:" lines.  With `check` the build is
// cross-checked by buildSingle() and the intersect output against a CPU
// multiset join; unlike the reference, a mismatch exits with status 1.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "hashgraph_b200/MultiHashGraph.h"

static void generate_input(inputData* d, index_t count) {
  std::vector<hkey_t> h(static_cast<size_t>(count));
  for (index_t j = 0; j < count; j++) h[j] = static_cast<hkey_t>(j);
  cudaMalloc(&d->d_keys, (count ? count : 1) * sizeof(hkey_t));
  cudaMalloc(&d->d_hash, (count ? count : 1) * sizeof(HashKey));
  cudaMemcpy(d->d_keys, h.data(), count * sizeof(hkey_t), cudaMemcpyHostToDevice);
  d->len = count;
}

int main(int argc, char** argv) {
  index_t countSizeA = 1L << 24, maxkey = 1L << 26, countSizeB = 1L << 22;
  index_t binCount = 16000, gpuCount = 1, lrbBins = 16000;
  bool check = false, buildTest = false;
  if (argc >= 2 && argc < 9) {
    std::fprintf(stderr, "Please specify all arguments.\n");
    return 1;
  }
  if (argc >= 9) {
    countSizeA = std::strtoll(argv[1], nullptr, 0);
    maxkey = std::strtoll(argv[2], nullptr, 0);
    binCount = std::atoi(argv[3]);
    gpuCount = std::atoi(argv[4]);
    lrbBins = std::strtoll(argv[5], nullptr, 0);
    check = !std::strcmp(argv[6], "check");
    countSizeB = std::strtoll(argv[7], nullptr, 0);
    buildTest = !std::strcmp(argv[8], "build");
  }
  const index_t tableSize = maxkey;
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  float ms = 0.f;
  try {
    if (buildTest) {
      inputData in[1];
      generate_input(in, countSizeA);
      MultiHashGraph mhg(in, countSizeA, maxkey, tableSize, binCount, lrbBins, gpuCount);
      cudaEventRecord(start);
      mhg.build(true, 0);
      cudaEventRecord(stop);
      cudaEventSynchronize(stop);
      cudaEventElapsedTime(&ms, start, stop);
      std::printf("multi buildTable() time: %g\n", ms / 1000.0);
      if (check) mhg.buildSingle();
      return 0;
    }
    inputData inA[1], inB[1];
    generate_input(inA, countSizeA);
    generate_input(inB, countSizeB);
    MultiHashGraph mhgA(inA, countSizeA, maxkey, tableSize, binCount, lrbBins, gpuCount);
    MultiHashGraph mhgB(inB, countSizeB, maxkey, tableSize, binCount, lrbBins, gpuCount);
    keypair* h_dOutput[1] = {nullptr};
    index_t h_Common[1] = {0};
    cudaEventRecord(start);
    mhgA.build(true, 0);
    mhgB.build(false, 0);
    MultiHashGraph::intersect(mhgA, mhgB, h_Common, h_dOutput, 0);
    cudaEventRecord(stop);
    cudaEventSynchronize(stop);
    cudaEventElapsedTime(&ms, start, stop);
    std::printf("multi intersect() time: %g\n", ms / 1000.0);
    if (check) {
      mhgA.buildSingle();
      mhgB.buildSingle();
      std::vector<keypair> out(static_cast<size_t>(h_Common[0]));
      if (h_Common[0]) cudaMemcpy(out.data(), h_dOutput[0], out.size() * sizeof(keypair), cudaMemcpyDeviceToHost);
      std::vector<hkey_t> result;
      for (const keypair& p : out) result.push_back(static_cast<hkey_t>(p.right));
      std::vector<hkey_t> a(mhgA.h_vals, mhgA.h_vals + countSizeA), b(mhgB.h_vals, mhgB.h_vals + countSizeB);
      std::sort(a.begin(), a.end());
      std::sort(b.begin(), b.end());
      std::vector<hkey_t> ans;  // multiset join by merging the sorted sets
      size_t i = 0, j = 0;
      while (i < a.size() && j < b.size()) {
        if (a[i] < b[j]) { i++; continue; }
        if (b[j] < a[i]) { j++; continue; }
        size_t i2 = i, j2 = j;
        while (i2 < a.size() && a[i2] == a[i]) i2++;
        while (j2 < b.size() && b[j2] == a[i]) j2++;
        for (size_t c = 0; c < (i2 - i) * (j2 - j); c++) ans.push_back(a[i]);
        i = i2;
        j = j2;
      }
      std::sort(result.begin(), result.end());
      if (result.size() != ans.size()) {
        std::fprintf(stderr, "ERROR: INTERSECT OUTPUT HAS INCORRECT SIZE\nansSize: %zu outputSize: %zu\n", ans.size(),
                     result.size());
        return 1;
      }
      if (result != ans) {
        std::fprintf(stderr, "ERROR: INTERSECT OUTPUT HAS INCORRECT CONTENT\n");
        return 1;
      }
      std::printf("intersect check ok: %lld matches\n", static_cast<long long>(h_Common[0]));
    }
    cudaFree(h_dOutput[0]);
  } catch (const hg::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  return 0;
}
