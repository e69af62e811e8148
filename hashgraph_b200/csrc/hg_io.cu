// hg_io.cu -- table files: save a built table to disk and load it back onto a
// device, so a table is built once and reused across processes.  The
// reference has no serialisation (its tables live and die with the process).
//
// File layout (little-endian):
//   header, 64 bytes:
//     char     magic[8]      "HGB2TBL" + NUL
//     uint32   version       1
//     uint32   key_bytes     4 or 8
//     uint32   with_index    0 or 1
//     uint32   hash          1 = murmur3_x86_32 of the key's low 32 bits, seed
//                            0, bucket = hash % n_buckets
//     uint64   n             keys
//     uint64   n_buckets
//     uint64   checksum      FNV-1a 64 of every payload byte in file order
//     uint64   reserved[2]   0
//   payload: offsets[n_buckets + 1] (uint32), keys[n] (key_bytes each),
//            idx[n] (uint32, only with_index)
// The arrays move between device and file through a pinned staging buffer in
// chunks, on the caller's stream.
#include <cstdio>
#include <cstring>

#include "hg_device.cuh"

namespace hg {

constexpr char TABLE_MAGIC[8] = {'H', 'G', 'B', '2', 'T', 'B', 'L', '\0'};
constexpr uint32_t TABLE_VERSION = 1;
constexpr uint32_t TABLE_HASH_MURMUR3_LOW32 = 1;
constexpr size_t IO_CHUNK = size_t(64) << 20;

struct TableHeader {
  char magic[8];
  uint32_t version, key_bytes, with_index, hash;
  uint64_t n, n_buckets, checksum, reserved[2];
};
static_assert(sizeof(TableHeader) == 64, "table header is 64 bytes");

inline uint64_t fnv1a(uint64_t h, const unsigned char* p, size_t len) {
  for (size_t i = 0; i < len; i++) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}
constexpr uint64_t FNV_BASIS = 0xcbf29ce484222325ull;

struct HostFile {
  FILE* f = nullptr;
  ~HostFile() {
    if (f) fclose(f);
  }
};

struct Pinned {
  void* p = nullptr;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

static hg_status read_header(FILE* f, const char* path, TableHeader* h) {
  if (fread(h, sizeof(*h), 1, f) != 1) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: short header");
  if (std::memcmp(h->magic, TABLE_MAGIC, 8) != 0) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: bad magic");
  if (h->version != TABLE_VERSION) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: unknown version");
  if (h->key_bytes != 4 && h->key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (h->with_index > 1 || h->hash != TABLE_HASH_MURMUR3_LOW32)
    return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: unknown index flag or hash");
  if (h->n_buckets == 0 || h->n_buckets > (1ull << 32) || h->n >= (1ull << 32))
    return lib_fail(HG_ERR_TOO_LARGE, "table file: sizes out of range");
  // the payload must be exactly what the header announces
  const uint64_t want = sizeof(TableHeader) + 4 * (h->n_buckets + 1) + h->n * h->key_bytes + (h->with_index ? 4 * h->n : 0);
  if (fseek(f, 0, SEEK_END) != 0) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: cannot seek");
  const long long size = ftell(f);
  if (size < 0 || uint64_t(size) != want) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: size does not match its header");
  if (fseek(f, sizeof(TableHeader), SEEK_SET) != 0) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: cannot seek");
  (void)path;
  return HG_OK;
}

// Device -> file, `bytes` from `d_src`, through the staging buffer.
static hg_status save_array(FILE* f, const void* d_src, uint64_t bytes, void* stage, cudaStream_t s, uint64_t* sum) {
  const char* src = static_cast<const char*>(d_src);
  for (uint64_t off = 0; off < bytes; off += IO_CHUNK) {
    const size_t len = static_cast<size_t>(std::min<uint64_t>(IO_CHUNK, bytes - off));
    HG_CUDA(cudaMemcpyAsync(stage, src + off, len, cudaMemcpyDeviceToHost, s), "hg_table_save: copy");
    HG_CUDA(cudaStreamSynchronize(s), "hg_table_save: copy");
    *sum = fnv1a(*sum, static_cast<const unsigned char*>(stage), len);
    if (fwrite(stage, 1, len, f) != len) return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_table_save: write failed");
  }
  return HG_OK;
}

// File -> device; `check` sees each chunk on the host.
template <typename Check>
static hg_status load_array(FILE* f, void* d_dst, uint64_t bytes, void* stage, cudaStream_t s, uint64_t* sum,
                            Check check) {
  char* dst = static_cast<char*>(d_dst);
  for (uint64_t off = 0; off < bytes; off += IO_CHUNK) {
    const size_t len = static_cast<size_t>(std::min<uint64_t>(IO_CHUNK, bytes - off));
    HG_CUDA(cudaStreamSynchronize(s), "hg_table_load: copy");  // the previous chunk left the staging buffer
    if (fread(stage, 1, len, f) != len) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: short read");
    *sum = fnv1a(*sum, static_cast<const unsigned char*>(stage), len);
    hg_status st = check(off, static_cast<const unsigned char*>(stage), len);
    if (st != HG_OK) return st;
    HG_CUDA(cudaMemcpyAsync(dst + off, stage, len, cudaMemcpyHostToDevice, s), "hg_table_load: copy");
  }
  return HG_OK;
}

}  // namespace hg

using namespace hg;

extern "C" hg_status hg_table_save_arrays(const char* path, const uint32_t* d_offsets, const void* d_keys,
                                          const uint32_t* d_idx, uint64_t n, uint64_t n_buckets, int key_bytes,
                                          hg_stream_t stream) {
  if (!path || !d_offsets || (n > 0 && !d_keys)) return HG_ERR_INVALID_ARGUMENT;
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (n_buckets == 0 || n_buckets > (1ull << 32) || n >= (1ull << 32)) return HG_ERR_TOO_LARGE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  HostFile hf;
  hf.f = fopen(path, "wb");
  if (!hf.f) return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_table_save: cannot open the file for writing");
  TableHeader h{};
  std::memcpy(h.magic, TABLE_MAGIC, 8);
  h.version = TABLE_VERSION;
  h.key_bytes = static_cast<uint32_t>(key_bytes);
  h.with_index = d_idx ? 1u : 0u;
  h.hash = TABLE_HASH_MURMUR3_LOW32;
  h.n = n;
  h.n_buckets = n_buckets;
  if (fwrite(&h, sizeof(h), 1, hf.f) != 1) return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_table_save: write failed");
  Pinned stage;
  HG_CUDA(cudaMallocHost(&stage.p, IO_CHUNK), "hg_table_save: staging buffer");
  uint64_t sum = FNV_BASIS;
  hg_status st = save_array(hf.f, d_offsets, 4 * (n_buckets + 1), stage.p, s, &sum);
  if (st == HG_OK && n) st = save_array(hf.f, d_keys, n * uint64_t(key_bytes), stage.p, s, &sum);
  if (st == HG_OK && n && d_idx) st = save_array(hf.f, d_idx, 4 * n, stage.p, s, &sum);
  if (st != HG_OK) return st;
  h.checksum = sum;
  if (fseek(hf.f, 0, SEEK_SET) != 0 || fwrite(&h, sizeof(h), 1, hf.f) != 1 || fflush(hf.f) != 0)
    return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_table_save: write failed");
  return HG_OK;
}

extern "C" hg_status hg_table_file_info(const char* path, uint64_t* n, uint64_t* n_buckets, int* key_bytes,
                                        int* with_index) {
  if (!path) return HG_ERR_INVALID_ARGUMENT;
  HostFile hf;
  hf.f = fopen(path, "rb");
  if (!hf.f) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: cannot open");
  TableHeader h;
  hg_status st = read_header(hf.f, path, &h);
  if (st != HG_OK) return st;
  if (n) *n = h.n;
  if (n_buckets) *n_buckets = h.n_buckets;
  if (key_bytes) *key_bytes = static_cast<int>(h.key_bytes);
  if (with_index) *with_index = static_cast<int>(h.with_index);
  return HG_OK;
}

extern "C" hg_status hg_table_load_arrays(const char* path, uint32_t* d_offsets, void* d_keys, uint32_t* d_idx,
                                          uint64_t n, uint64_t n_buckets, int key_bytes, hg_stream_t stream) {
  if (!path || !d_offsets) return HG_ERR_INVALID_ARGUMENT;
  HostFile hf;
  hf.f = fopen(path, "rb");
  if (!hf.f) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: cannot open");
  TableHeader h;
  hg_status st = read_header(hf.f, path, &h);
  if (st != HG_OK) return st;
  if (h.n != n || h.n_buckets != n_buckets || int(h.key_bytes) != key_bytes)
    return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_table_load_arrays: sizes differ from the file's");
  if ((h.n > 0 && !d_keys) || (h.with_index && h.n > 0 && !d_idx))
    return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_table_load_arrays: missing destination array");
  if (!h.with_index && d_idx)
    return lib_fail(HG_ERR_INVALID_ARGUMENT,
                    "hg_table_load_arrays: the file holds no input positions, but d_idx was given");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Pinned stage;
  HG_CUDA(cudaMallocHost(&stage.p, IO_CHUNK), "hg_table_load: staging buffer");
  uint64_t sum = FNV_BASIS;
  const uint64_t off_bytes = 4 * (n_buckets + 1);
  // offsets[0] must be 0, offsets[n_buckets] must be n, and the offsets must
  // not decrease (checked chunk by chunk on the host, before each chunk is
  // copied, carrying the last value across chunks): the probes read
  // keys[offsets[b] .. offsets[b+1]) without further checks.
  uint32_t prev = 0;
  st = load_array(hf.f, d_offsets, off_bytes, stage.p, s, &sum,
                  [&](uint64_t off, const unsigned char* p, size_t len) -> hg_status {
                    uint32_t v;
                    if (off == 0) {
                      std::memcpy(&v, p, 4);
                      if (v != 0) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: offsets[0] is not 0");
                    }
                    for (size_t x = 0; x + 4 <= len; x += 4) {
                      std::memcpy(&v, p + x, 4);
                      if (v < prev || v > h.n)
                        return lib_fail(HG_ERR_INVALID_ARGUMENT,
                                        "table file: offsets decrease or exceed n");
                      prev = v;
                    }
                    if (off + len == off_bytes) {
                      std::memcpy(&v, p + len - 4, 4);
                      if (v != h.n) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: offsets[n_buckets] is not n");
                    }
                    return HG_OK;
                  });
  auto none = [](uint64_t, const unsigned char*, size_t) -> hg_status { return HG_OK; };
  if (st == HG_OK && h.n) st = load_array(hf.f, d_keys, h.n * h.key_bytes, stage.p, s, &sum, none);
  if (st == HG_OK && h.n && h.with_index) st = load_array(hf.f, d_idx, 4 * h.n, stage.p, s, &sum, none);
  HG_CUDA(cudaStreamSynchronize(s), "hg_table_load: copy");  // the staging buffer is freed on return
  if (st != HG_OK) return st;
  if (sum != h.checksum) return lib_fail(HG_ERR_INVALID_ARGUMENT, "table file: checksum mismatch");
  return HG_OK;
}

extern "C" hg_status hg_table_save(const hg_table* t, const char* path, hg_stream_t stream) {
  if (!t || !t->built) return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_table_save: table not built");
  return hg_table_save_arrays(path, t->offsets, t->keys, t->idx, t->n, t->n_buckets, t->key_bytes, stream);
}

extern "C" hg_status hg_table_load(const char* path, hg_table** out, hg_stream_t stream) {
  if (!out) return HG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  uint64_t n = 0, nb = 0;
  int kb = 0, wi = 0;
  hg_status st = hg_table_file_info(path, &n, &nb, &kb, &wi);
  if (st != HG_OK) return st;
  hg_table* t = new (std::nothrow) hg_table();
  if (!t) return HG_ERR_OUT_OF_MEMORY;
  cudaGetDevice(&t->device);
  t->capacity = n;
  t->n = n;
  t->n_buckets = nb;
  t->key_bytes = kb;
  t->with_index = wi != 0;
  // no build workspace: hg_table_build allocates one if the table is rebuilt
  cudaError_t e = cudaMalloc(&t->offsets, (nb + 1) * sizeof(uint32_t));
  if (e == cudaSuccess && n) e = cudaMalloc(&t->keys, n * kb);
  if (e == cudaSuccess && n && wi) e = cudaMalloc(&t->idx, n * sizeof(uint32_t));
  if (e != cudaSuccess) {
    cudaGetLastError();
    hg_table_free(t);
    return cuda_fail(e, "hg_table_load: allocation");
  }
  st = hg_table_load_arrays(path, t->offsets, t->keys, t->idx, n, nb, kb, stream);
  if (st != HG_OK) {
    hg_table_free(t);
    return st;
  }
  t->built = true;
  *out = t;
  return HG_OK;
}
