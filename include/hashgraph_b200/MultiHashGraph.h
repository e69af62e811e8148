// MultiHashGraph.h -- the reference's class API for the hash-range
// partitioned table (alokpathy/hashgraph include/MultiHashGraph.cuh:150-293,
// src/MultiHashGraph.cu:61-862) on top of the hashgraph_b200 C ABI, for one
// GPU (gpuCount = 1: the single-device hot path; other counts throw).
//
// Kept: constructor arguments and their meaning, build(findSplits, tid),
// static intersect(A, B, h_Common, h_dOutput, tid) with its outputs
// (h_Common[tid] = number of matches, h_dOutput[tid] = device array of
// keypair{B's key} that the caller owns), buildSingle() (cross-check against
// the plain single-table build, mismatches printed to stderr), destroyMulti(),
// and the public result fields: h_dFinalKeys[tid] holds the table in the
// reference layout -- keyval_ind edges at h_edgesOff[tid] and int64 offsets
// at h_offsetOff[tid] -- and h_binSplits = {0, tableSize}.
// Not kept: the reference frees the caller's inputData buffers in build() and
// exits on errors; here nothing of the caller's is freed and errors throw
// hg::Error.  binCount and lrbBins have no meaning (geometry is planned from
// the sizes).
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
  // The native table (C ABI handle) after build().
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
  void exportReferenceLayout();
};
