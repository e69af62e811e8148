// MultiHashGraph.h -- the reference's class API for the hash-range
// partitioned table (alokpathy/hashgraph include/MultiHashGraph.cuh:150-293,
// src/MultiHashGraph.cu:61-862) on top of the hashgraph_b200 C ABI.
//
// Kept: constructor arguments and their meaning, build(findSplits, tid) and
// static intersect(A, B, h_Common, h_dOutput, tid) called from gpuCount host
// threads (tid = 0..gpuCount-1, e.g. an OpenMP team as in the reference's
// test/MultiHashGraphTest.cu:288-338), with their outputs (h_Common[tid] =
// matches found on GPU tid, h_dOutput[tid] = device array of keypair{B's key}
// on that GPU, owned by the caller), buildSingle() (cross-check against the
// plain single-table build, mismatches printed to stderr), destroyMulti(),
// and the public result fields: h_binSplits[0..gpuCount] (GPU tid holds
// buckets [h_binSplits[tid], h_binSplits[tid+1]); a second table is put on
// the first one's splits by assigning h_binSplits and building with
// findSplits = false, as the reference's test does), h_dFinalKeys[tid] holds
// GPU tid's table in the reference layout -- keyval_ind edges at
// h_edgesOff[tid] and int64 offsets of its range at h_offsetOff[tid].
// gpuCount = 1 builds the whole table on device 0 with the planner's path;
// gpuCount > 1 follows the reference's pipeline on the sharding calls
// (hg_shard_histogram / hg_shard_splits / hg_shard_route, copies to the owning
// devices, hg_shard_build_into), GPU tid on device tid (tid % device count
// when there are fewer devices).  build() waits for the other threads where
// the reference takes `omp barrier` (bounded: a missing thread is an error).
// Not kept: the reference frees the caller's inputData buffers in build() and
// exits on errors; here nothing of the caller's is freed and errors throw
// hg::Error.  Edge indices are global input positions (the reference's are
// positions on the source GPU).  lrbBins has no meaning (geometry is planned
// from the sizes); binCount is the histogram's bin count (at most 32768).
#pragma once
#include <cstdint>
#include <vector>

#include "hg_types.h"

class MultiHashGraph {
 public:
  MultiHashGraph(inputData* h_dVals, index_t countSize, index_t maxkey, index_t tableSize, index_t binCount,
                 index_t lrbBins, index_t gpuCount);
  ~MultiHashGraph();
  MultiHashGraph(const MultiHashGraph&) = delete;
  MultiHashGraph& operator=(const MultiHashGraph&) = delete;

  void build(bool findSplits, index_t tid);
  void buildSingle();
  static void intersect(MultiHashGraph& mgA, MultiHashGraph& mgB, index_t* h_Common, keypair** h_dOutput,
                        index_t tid);
  void destroyMulti();

  // Whether build() also writes the reference layout into h_dFinalKeys
  // (on by default; intersect never needs it).
  void setExportReferenceLayout(bool on) { exportLayout = on; }
  // The native table (C ABI handle) after build() with gpuCount = 1.
  hg_table* table() const { return tbl; }

  // Public fields of the reference class, same meaning.
  char** h_dFinalKeys = nullptr;
  index_t* h_hashOff = nullptr;
  index_t* h_counterOff = nullptr;
  index_t* h_offsetOff = nullptr;
  index_t* h_edgesOff = nullptr;
  index_t* h_lrbOff = nullptr;
  index_t* h_binSplits = nullptr;
  index_t** h_dBinSplits = nullptr;
  index_t countSize = 0;
  index_t tableSize = 0;
  index_t gpuCount = 1;
  hkey_t* h_vals = nullptr;  // host copy of the input keys (for checks)

 private:
  inputData* h_dVals = nullptr;
  index_t maxkey = 0, binCount = 0, lrbBins = 0;
  hg_table* tbl = nullptr;
  bool exportLayout = true;
  index_t* ownSplits = nullptr;  // the splits this table found (h_binSplits may point elsewhere)
  struct Shard;
  struct Multi;
  Multi* multi = nullptr;  // gpuCount > 1
  void buildShard(bool findSplits, int tid);
  static void intersectShard(MultiHashGraph& A, MultiHashGraph& B, index_t* h_Common, keypair** h_dOutput, int tid);
  void exportReferenceLayout(int tid, const uint32_t* off, const void* keys, const uint32_t* idx, uint64_t n,
                             uint64_t nb, hg_stream_t stream);
};
