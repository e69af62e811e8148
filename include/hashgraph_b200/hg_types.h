// hg_types.h -- the reference's key/index types and records, kept for the
// C++ classes (alokpathy/hashgraph include/MultiHashGraph.cuh:66-106): 64-bit
// keys by default, 32-bit keys when B32 is defined; int64 indices.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>

#include "hashgraph_b200.h"

#ifdef B32
using hkey_t = uint32_t;
using index_t = int64_t;
using HashKey = uint32_t;
#else
using hkey_t = int64_t;
using index_t = int64_t;
using HashKey = int64_t;
#endif

// Edge record of the exported reference layout (include/MultiHashGraph.cuh:82-87,
// the INDEX_TRACK form the reference builds with).
struct keyval_ind {
  hkey_t key;
  index_t ind;
};
using keyval = keyval_ind;

// Intersect output record: B's key per match (include/MultiHashGraph.cuh:89-93).
struct keypair {
  index_t right;
};

// Per-GPU input (include/MultiHashGraph.cuh:95-100).
struct inputData {
  hkey_t* d_keys;
  HashKey* d_hash;
  index_t len;
};

namespace hg {
// Errors are thrown (the reference prints and calls exit(0)).
class Error : public std::runtime_error {
 public:
  Error(hg_status status, const std::string& what)
      : std::runtime_error(what + ": " + hg_status_str(status) + " " + hg_last_error()), status_(status) {}
  hg_status status() const { return status_; }

 private:
  hg_status status_;
};
inline void check(hg_status st, const char* what) {
  if (st != HG_OK) throw Error(st, what);
}
}  // namespace hg
