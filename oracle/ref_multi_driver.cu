// ref_multi_driver.cu -- TEST INFRASTRUCTURE ONLY.
//
// Runs the UNMODIFIED reference MultiHashGraph (src/MultiHashGraph.cu, linked
// from its own source by oracle/Makefile) with gpuCount = 1 on keys read from
// files, through its public API exactly as test/MultiHashGraphTest.cu:257-325
// drives it: construct A and B, build A with split finding, hand A's splits to
// B, build B, then MultiHashGraph::intersect.  Times build and the whole
// sequence with CUDA events (as the reference's test main does) and dumps the
// results so tests can compare them with the oracle and with this library.
//
// usage: ref_multi <keysA> <nA> <keysB|-> <nB> <tableSize> <outdir|-> [warmup] [repeats]
//   keys files hold raw hkey_t (int64, or uint32 when built with -DB32).
//   With repeats > 1 the whole sequence (construct, build A, build B,
//   intersect) runs that many times on the same inputs; one JSON line per run.
//   Outputs in outdir: A_offsets.i64 (hashRange+1 int64), A_edges.kv
//   (keyval records), common.i64, pairs.key (hkey_t per match, B's key).
#include "MultiHashGraph.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static std::vector<hkey_t> read_keys(const char* path, index_t n) {
  std::vector<hkey_t> v((size_t)n);
  std::FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), sizeof(hkey_t), (size_t)n, f) != (size_t)n) {
    std::fprintf(stderr, "cannot read %lld keys from %s\n", (long long)n, path);
    std::exit(3);
  }
  std::fclose(f);
  return v;
}

static void to_device(inputData* d, const std::vector<hkey_t>& keys) {
  cudaMalloc(&d->d_keys, keys.size() * sizeof(hkey_t));
  cudaMalloc(&d->d_hash, keys.size() * sizeof(HashKey));
  cudaMemcpy(d->d_keys, keys.data(), keys.size() * sizeof(hkey_t), cudaMemcpyHostToDevice);
  d->len = (index_t)keys.size();
}

template <typename T>
static void dump(const std::string& path, const T* dptr, size_t count) {
  std::vector<T> h(count);
  if (count) cudaMemcpy(h.data(), dptr, count * sizeof(T), cudaMemcpyDeviceToHost);
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) { std::fprintf(stderr, "cannot write %s\n", path.c_str()); std::exit(4); }
  if (count) std::fwrite(h.data(), sizeof(T), count, f);
  std::fclose(f);
}

struct RunTimes { float build_a_ms, build_b_ms, intersect_ms, total_ms; };

static RunTimes run(const std::vector<hkey_t>& a, const std::vector<hkey_t>& b, index_t tableSize,
                    const char* outdir) {
  const index_t binCount = 16000, lrbBins = 16000, gpuCount = 1;
  const bool do_intersect = !b.empty();
  inputData* hA = new inputData[1]();
  inputData* hB = new inputData[1]();
  to_device(hA, a);
  if (do_intersect) to_device(hB, b);
  cudaDeviceSynchronize();

  MultiHashGraph mA(hA, (index_t)a.size(), tableSize, tableSize, binCount, lrbBins, gpuCount);
  MultiHashGraph* mB = nullptr;
  if (do_intersect)
    mB = new MultiHashGraph(hB, (index_t)b.size(), tableSize, tableSize, binCount, lrbBins, gpuCount);

  keypair** h_dOutput = new keypair*[gpuCount]();
  index_t* h_Common = new index_t[gpuCount]();
  cudaEvent_t e0, e1, e2, e3;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
  omp_set_num_threads(gpuCount);
  cudaSetDevice(0);
  cudaEventRecord(e0);
  #pragma omp parallel
  {
    index_t tid = omp_get_thread_num();
    mA.build(true, tid);
    cudaSetDevice(0);
    cudaEventRecord(e1);
    if (do_intersect) {
      #pragma omp master
      {
        mB->h_binSplits = mA.h_binSplits;
        mB->h_dBinSplits = mA.h_dBinSplits;
      }
      #pragma omp barrier
      mB->build(false, tid);
      cudaSetDevice(0);
      cudaEventRecord(e2);
      #pragma omp barrier
      MultiHashGraph::intersect(mA, *mB, h_Common, h_dOutput, tid);
    }
  }
  cudaSetDevice(0);
  cudaEventRecord(e3);
  cudaEventSynchronize(e3);
  RunTimes t{0, 0, 0, 0};
  cudaEventElapsedTime(&t.build_a_ms, e0, e1);
  if (do_intersect) {
    cudaEventElapsedTime(&t.build_b_ms, e1, e2);
    cudaEventElapsedTime(&t.intersect_ms, e2, e3);
  }
  cudaEventElapsedTime(&t.total_ms, e0, e3);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    std::fprintf(stderr, "cuda error %s\n", cudaGetErrorString(err));
    std::exit(5);
  }

  if (outdir && std::strcmp(outdir, "-") != 0) {
    std::string od(outdir);
    index_t range = mA.h_binSplits[1] - mA.h_binSplits[0];
    dump(od + "/A_offsets.i64", (index_t*)(mA.h_dFinalKeys[0] + mA.h_offsetOff[0]), (size_t)range + 1);
    dump(od + "/A_edges.kv", (keyval*)(mA.h_dFinalKeys[0] + mA.h_edgesOff[0]), a.size());
    if (do_intersect) {
      std::FILE* f = std::fopen((od + "/common.i64").c_str(), "wb");
      std::fwrite(h_Common, sizeof(index_t), 1, f);
      std::fclose(f);
      std::vector<hkey_t> right((size_t)h_Common[0]);
      std::vector<keypair> kp((size_t)h_Common[0]);
      if (h_Common[0] > 0)
        cudaMemcpy(kp.data(), h_dOutput[0], kp.size() * sizeof(keypair), cudaMemcpyDeviceToHost);
      for (size_t i = 0; i < kp.size(); i++) right[i] = (hkey_t)kp[i].right;
      std::FILE* g = std::fopen((od + "/pairs.key").c_str(), "wb");
      if (!right.empty()) std::fwrite(right.data(), sizeof(hkey_t), right.size(), g);
      std::fclose(g);
    }
  }
  return t;
}

int main(int argc, char** argv) {
  if (argc < 7) {
    std::fprintf(stderr, "usage: %s keysA nA keysB|- nB tableSize outdir|- [warmup]\n", argv[0]);
    return 2;
  }
  index_t nA = (index_t)std::strtoll(argv[2], nullptr, 0);
  index_t nB = (index_t)std::strtoll(argv[4], nullptr, 0);
  index_t tableSize = (index_t)std::strtoll(argv[5], nullptr, 0);
  int warmup = argc > 7 ? std::atoi(argv[7]) : 1;
  std::vector<hkey_t> a = read_keys(argv[1], nA);
  std::vector<hkey_t> b;
  if (std::strcmp(argv[3], "-") != 0 && nB > 0) b = read_keys(argv[3], nB);
  if (warmup) {
    // Module load and context set-up on a tiny input, outside the timed run.
    std::vector<hkey_t> wa(a.begin(), a.begin() + std::min<size_t>(a.size(), 4096));
    std::vector<hkey_t> wb(b.begin(), b.begin() + std::min<size_t>(b.size(), 4096));
    run(wa, wb, std::min<index_t>(tableSize, 4096), "-");
  }
  const int repeats = argc > 8 ? std::max(1, std::atoi(argv[8])) : 1;
  for (int r = 0; r < repeats; r++) {
    // results are dumped from the last run only
    RunTimes t = run(a, b, tableSize, r + 1 == repeats ? argv[6] : "-");
    std::printf("{\"n_a\": %lld, \"n_b\": %lld, \"table_size\": %lld, \"run\": %d, \"build_a_s\": %.9f, "
                "\"build_b_s\": %.9f, \"intersect_s\": %.9f, \"total_s\": %.9f}\n",
                (long long)nA, (long long)nB, (long long)tableSize, r, t.build_a_ms / 1e3,
                t.build_b_ms / 1e3, t.intersect_ms / 1e3, t.total_ms / 1e3);
    std::fflush(stdout);
  }
  return 0;
}
