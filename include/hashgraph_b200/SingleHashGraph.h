// SingleHashGraph.h -- the reference's single-GPU class API
// (alokpathy/hashgraph include/SingleHashGraph.cuh:89-116,
// src/SingleHashGraph.cu:79-232) on top of the hashgraph_b200 C ABI.
//
// As in the reference, the constructor allocates the table and generates
// countSize keys uniform in [0, maxkey] on the device; build() builds the CSR
// of those keys into tableSize buckets.  The keys come from the library's
// seeded generator (the reference uses thrust minstd draws), and lrbBins has
// no meaning here: the partition geometry is planned from the sizes.  Errors
// throw hg::Error instead of exiting.
#pragma once
#include <cstdint>

#include "hg_types.h"

class SingleHashGraph {
 public:
  SingleHashGraph(int64_t countSize, int64_t maxkey, int64_t tableSize, int64_t lrbBins);
  ~SingleHashGraph();
  SingleHashGraph(const SingleHashGraph&) = delete;
  SingleHashGraph& operator=(const SingleHashGraph&) = delete;

  // Builds the CSR of the first countSize generated keys into tableSize
  // buckets (stream-ordered on the legacy default stream, like the reference).
  void build(int64_t countSize, int64_t tableSize);

  // Views of the built table (device pointers; offsets are uint32).
  const uint32_t* offsets() const { return d_offset; }
  const hkey_t* edges() const { return reinterpret_cast<const hkey_t*>(d_edges); }
  const hkey_t* keys() const { return d_vals; }
  int64_t size() const { return countSize; }

 private:
  int64_t countSize = 0, tableSize = 0, lrbBins = 0;
  hkey_t* d_vals = nullptr;
  uint32_t* d_offset = nullptr;
  hkey_t* d_edges = nullptr;
  void* d_ws = nullptr;
  size_t ws_bytes = 0;
};
