// ref_hash_driver.cu -- TEST INFRASTRUCTURE ONLY.
//
// Host-side driver around the reference's own hash function, used to pin the
// oracle's murmur restatement.  oracle/Makefile compiles it against the
// reference headers where they lie (never copied):
//   -DREF_SINGLE: include/SingleHashGraph.cuh + SingleHashGraphOperators.cuh
//                 (HashKey = uint32_t; keys reach hash_murmur through the
//                 int64 -> uint32 conversion of hashValuesD, :71-79)
//   -DREF_MULTI:  include/MultiHashGraph.cuh + MultiHashGraphDeviceOperators.cuh
//                 (64-bit build: HashKey = int64_t, hash reads its first 4 bytes)
// Reads little-endian u64 keys from argv[1], writes u32 hashes to argv[2].
#include <cstdio>
#include <cstdint>
#include <vector>

#if defined(REF_SINGLE)
#include "SingleHashGraph.cuh"
#include "SingleHashGraphOperators.cuh"
static uint32_t ref_hash(uint64_t k) {
  hkey_t v = (hkey_t)k;
  return hash_murmur(v);  // hkey_t -> const HashKey& as in hashValuesD
}
#elif defined(REF_MULTI)
#include "MultiHashGraph.cuh"
#include "MultiHashGraphDeviceOperators.cuh"
static uint32_t ref_hash(uint64_t k) {
  HashKey v = (HashKey)k;
  return hash_murmur(v);
}
#else
#error "define REF_SINGLE or REF_MULTI"
#endif

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s keys.u64 hashes.u32\n", argv[0]);
    return 2;
  }
  std::FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  std::vector<uint64_t> keys;
  uint64_t k;
  while (std::fread(&k, sizeof(k), 1, f) == 1) keys.push_back(k);
  std::fclose(f);
  std::vector<uint32_t> out(keys.size());
  for (size_t i = 0; i < keys.size(); i++) out[i] = ref_hash(keys[i]);
  std::FILE* g = std::fopen(argv[2], "wb");
  if (!g) return 4;
  if (!out.empty() && std::fwrite(out.data(), sizeof(uint32_t), out.size(), g) != out.size()) return 5;
  std::fclose(g);
  return 0;
}
