// multi_hash_main.cpp -- the reference's MultiHashGraph test main
// (alokpathy/hashgraph test/MultiHashGraphTest.cu:130-427) rewritten over the
// drop-in classes: same positional arguments
//   multi-hash size maxkey binCount gpuCount lrbBins check|nocheck countSizeB build|intersect
// same inputs (sequential keys A = 0..size-1, B = 0..countSizeB-1, each cut
// into gpuCount contiguous chunks of ceil(size / gpuCount), chunk t on GPU t),
// the same OpenMP team of gpuCount threads calling build(true, tid), B's
// build(false, tid) on A's splits and intersect(..., tid), the same timed
// regions (CUDA events around build, and around build A + build B +
// intersect) and the same "multi ... time:" lines.  With `check` the build is
// cross-checked by buildSingle() and the intersect output (every GPU's)
// against a CPU multiset join; unlike the reference, a mismatch exits with
// status 1.  With fewer devices than gpuCount, GPU t is device t % count.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "hashgraph_b200/MultiHashGraph.h"

static int device_of(index_t t) {
  int nd = 1;
  cudaGetDeviceCount(&nd);
  return static_cast<int>(t % nd);
}

// keys 0..count-1, chunk t = [ceil(count/G) * t, ...) on GPU t
static void generate_input(inputData* d, index_t count, index_t gpuCount) {
  const index_t avg = (count + gpuCount - 1) / gpuCount;
  for (index_t t = 0; t < gpuCount; t++) {
    const index_t lo = std::min(avg * t, count), hi = std::min(avg * (t + 1), count);
    std::vector<hkey_t> h(static_cast<size_t>(hi - lo));
    for (index_t j = lo; j < hi; j++) h[j - lo] = static_cast<hkey_t>(j);
    cudaSetDevice(device_of(t));
    cudaMalloc(&d[t].d_keys, (hi > lo ? hi - lo : 1) * sizeof(hkey_t));
    cudaMalloc(&d[t].d_hash, (hi > lo ? hi - lo : 1) * sizeof(HashKey));
    cudaMemcpy(d[t].d_keys, h.data(), (hi - lo) * sizeof(hkey_t), cudaMemcpyHostToDevice);
    d[t].len = hi - lo;
  }
  cudaSetDevice(0);
}

static void free_input(inputData* d, index_t gpuCount) {
  for (index_t t = 0; t < gpuCount; t++) {
    cudaSetDevice(device_of(t));
    cudaFree(d[t].d_keys);
    cudaFree(d[t].d_hash);
  }
  cudaSetDevice(0);
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
  if (gpuCount < 1 || gpuCount > HG_MAX_SHARDS) {
    std::fprintf(stderr, "gpuCount must be 1..64\n");
    return 1;
  }
  try {
    if (buildTest) {
      std::vector<inputData> in(gpuCount);
      generate_input(in.data(), countSizeA, gpuCount);
      MultiHashGraph mhg(in.data(), countSizeA, maxkey, tableSize, binCount, lrbBins, gpuCount);
      cudaEventRecord(start);
#pragma omp parallel num_threads(gpuCount)
      {
        const index_t tid = omp_get_thread_num();
        mhg.build(true, tid);
      }
      cudaSetDevice(0);
      cudaEventRecord(stop);
      cudaEventSynchronize(stop);
      cudaEventElapsedTime(&ms, start, stop);
      std::printf("multi buildTable() time: %g\n", ms / 1000.0);
      if (check) mhg.buildSingle();
      free_input(in.data(), gpuCount);
      return 0;
    }
    std::vector<inputData> inA(gpuCount), inB(gpuCount);
    generate_input(inA.data(), countSizeA, gpuCount);
    generate_input(inB.data(), countSizeB, gpuCount);
    MultiHashGraph mhgA(inA.data(), countSizeA, maxkey, tableSize, binCount, lrbBins, gpuCount);
    MultiHashGraph mhgB(inB.data(), countSizeB, maxkey, tableSize, binCount, lrbBins, gpuCount);
    std::vector<keypair*> h_dOutput(gpuCount, nullptr);
    std::vector<index_t> h_Common(gpuCount, 0);
    cudaEventRecord(start);
#pragma omp parallel num_threads(gpuCount)
    {
      const index_t tid = omp_get_thread_num();
      mhgA.build(true, tid);
#pragma omp master
      mhgB.h_binSplits = mhgA.h_binSplits;  // B on A's splits
#pragma omp barrier
      mhgB.build(false, tid);
#pragma omp barrier
      MultiHashGraph::intersect(mhgA, mhgB, h_Common.data(), h_dOutput.data(), tid);
    }
    cudaSetDevice(0);
    cudaEventRecord(stop);
    cudaEventSynchronize(stop);
    cudaEventElapsedTime(&ms, start, stop);
    std::printf("multi intersect() time: %g\n", ms / 1000.0);
    if (check) {
      mhgA.buildSingle();
      mhgB.buildSingle();
      std::vector<hkey_t> result;
      index_t total = 0;
      for (index_t t = 0; t < gpuCount; t++) {
        std::vector<keypair> out(static_cast<size_t>(h_Common[t]));
        cudaSetDevice(device_of(t));
        if (h_Common[t]) cudaMemcpy(out.data(), h_dOutput[t], out.size() * sizeof(keypair), cudaMemcpyDeviceToHost);
        for (const keypair& p : out) result.push_back(static_cast<hkey_t>(p.right));
        total += h_Common[t];
      }
      cudaSetDevice(0);
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
      std::printf("intersect check ok: %lld matches\n", static_cast<long long>(total));
    }
    for (index_t t = 0; t < gpuCount; t++) {
      cudaSetDevice(device_of(t));
      cudaFree(h_dOutput[t]);
    }
    cudaSetDevice(0);
    free_input(inA.data(), gpuCount);
    free_input(inB.data(), gpuCount);
  } catch (const hg::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  return 0;
}
