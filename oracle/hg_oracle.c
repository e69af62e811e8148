/*
 * hg_oracle.c -- CPU oracle for the HashGraph build + intersect path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Plain-C restatement of the
 * reference's algorithm; only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it.  The product library never does.
 *
 * Reference citations are paths inside alokpathy/hashgraph.
 */
#include "hg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

/* ---------------------------------------------------------------------------
 * Hash.  murmur3_x86_32 (Appleby, public domain) over len = sizeof(int) = 4
 * bytes starting at &key, seed h1 = 0: include/SingleHashGraphOperators.cuh:31-69
 * (identical copy in include/MultiHashGraphDeviceOperators.cuh:37-73).  Only the
 * low 32 bits of a 64-bit key reach the hash (little-endian first 4 bytes).
 * With len = 4 there is exactly one body block and no tail.
 * ------------------------------------------------------------------------- */
static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

uint32_t or_murmur3_low32(uint64_t key) {
  uint32_t k = (uint32_t)key;
  k *= 0xcc9e2d51u;              /* c1, SingleHashGraphOperators.cuh:37 */
  k = rotl32(k, 15);
  k *= 0x1b873593u;              /* c2, :38 */
  uint32_t h = 0u ^ k;           /* seed 0, :36 */
  h = rotl32(h, 13);
  h = h * 5u + 0xe6546b64u;      /* :51 */
  h ^= 4u;                       /* h1 ^= len, :66 */
  h ^= h >> 16;                  /* fmix32, :22-29 */
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

/* `% tableSize`: u32 % u32 in Single (SingleHashGraphOperators.cuh:76), and
 * u32 promoted to int64 % int64 in Multi (MultiHashGraphDeviceOperators.cuh:81);
 * both equal the unsigned remainder below for tableSize >= 1. */
uint64_t or_bucket(uint64_t key, uint64_t n_buckets) {
  return (uint64_t)or_murmur3_low32(key) % n_buckets;
}

static inline uint64_t load_key(const void* keys, uint64_t i, int kb) {
  return kb == 8 ? ((const uint64_t*)keys)[i] : (uint64_t)((const uint32_t*)keys)[i];
}
static inline void store_key(void* keys, uint64_t i, int kb, uint64_t v) {
  if (kb == 8) ((uint64_t*)keys)[i] = v; else ((uint32_t*)keys)[i] = (uint32_t)v;
}

void or_buckets(const void* keys, uint64_t n, int kb, uint64_t n_buckets, uint64_t* out) {
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) out[i] = or_bucket(load_key(keys, (uint64_t)i, kb), n_buckets);
}

/* Lemire, Kaser, Kurz, "Faster remainder by direct computation" (2019):
 * M = floor((2^64-1)/d) + 1, a % d = hi64((M * a mod 2^64) * d) for 32-bit a, d. */
uint64_t or_fastmod_magic(uint32_t d) { return UINT64_MAX / d + 1; }
uint32_t or_fastmod(uint32_t a, uint64_t magic, uint32_t d) {
  uint64_t low = magic * a;
  return (uint32_t)(((__uint128_t)low * d) >> 64);
}

/* ---------------------------------------------------------------------------
 * Workload generators.  The reference generates sequential keys
 * (test/MultiHashGraphTest.cu:105-111) or thrust minstd draws in [0, maxkey]
 * (:26-37); the workloads here need uniform 32/64-bit keys, controlled
 * overlap and Zipf skew, so they use a counter-based splitmix64 stream
 * (Steele, Lea, Flood 2014).  The device generator in the library states the
 * same definitions; tests check both agree bit for bit.
 * ------------------------------------------------------------------------- */
#define GOLDEN 0x9E3779B97F4A7C15ull

uint64_t or_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t or_rand64(uint64_t seed, uint64_t stream, uint64_t i) {
  uint64_t base = or_mix64(seed * GOLDEN + stream + 1);
  return or_mix64(base + (i + 1) * GOLDEN);
}

/* Keyed bijection on [0, n): three odd-multiply / xorshift rounds on the
 * enclosing power of two, then cycle-walking back into [0, n). */
uint64_t or_perm(uint64_t i, uint64_t n, uint64_t seed) {
  if (n <= 1) return 0;
  int k = 64 - __builtin_clzll(n - 1);
  uint64_t mask = (k == 64) ? ~0ull : ((1ull << k) - 1);
  int s = k / 2 + 1;
  uint64_t a[3], c[3];
  for (int r = 0; r < 3; r++) {
    a[r] = or_rand64(seed, 100 + r, 0) | 1ull;
    c[r] = or_rand64(seed, 200 + r, 0);
  }
  uint64_t x = i;
  do {
    for (int r = 0; r < 3; r++) {
      x = (x * a[r] + c[r]) & mask;
      x ^= x >> s;
    }
  } while (x >= n);
  return x;
}

void or_gen_uniform(void* out, uint64_t n, int kb, uint64_t seed) {
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint64_t r = or_rand64(seed, 0, (uint64_t)i);
    store_key(out, (uint64_t)i, kb, kb == 8 ? r : (r >> 32));
  }
}

/* Set B of n keys: round(frac*n) of them (capped at n_a) are distinct draws
 * from A, the rest are fresh uniform keys, and the whole set is shuffled. */
void or_gen_overlap(void* out, uint64_t n, int kb, const void* a_keys, uint64_t n_a,
                    double frac, uint64_t seed) {
  uint64_t m = (uint64_t)llround(frac * (double)n);
  if (m > n) m = n;
  if (m > n_a) m = n_a;
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint64_t j = or_perm((uint64_t)i, n, seed);
    uint64_t v;
    if (j < m) {
      v = load_key(a_keys, or_perm(j, n_a, seed + 1), kb);
    } else {
      uint64_t r = or_rand64(seed, 2, j);
      v = kb == 8 ? r : (r >> 32);
    }
    store_key(out, (uint64_t)i, kb, v);
  }
}

/* Zipf(s) over ranks 0..U-1 with weight (r+1)^-s; cdf is u64 fixed point,
 * cdf[U-1] = 2^64-1. */
int or_zipf_cdf(uint64_t* cdf, uint64_t U, double s) {
  if (U == 0) return -1;
  long double h = 0.0L;
  for (uint64_t r = 0; r < U; r++) h += powl((long double)(r + 1), -(long double)s);
  long double acc = 0.0L;
  const long double two64 = 18446744073709551616.0L;
  for (uint64_t r = 0; r < U; r++) {
    acc += powl((long double)(r + 1), -(long double)s);
    long double v = acc / h * two64;
    cdf[r] = (v >= two64) ? UINT64_MAX : (uint64_t)v;
  }
  cdf[U - 1] = UINT64_MAX;
  return 0;
}

void or_gen_zipf(void* out, uint64_t n, int kb, const uint64_t* cdf, uint64_t U, uint64_t seed) {
  /* rank -> key depends on the universe only: sets drawn with different
   * seeds share keys */
  uint64_t salt = or_rand64(0x21BF, 4, U);
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint64_t u = or_rand64(seed, 3, (uint64_t)i);
    uint64_t lo = 0, hi = U - 1;
    while (lo < hi) {
      uint64_t mid = (lo + hi) >> 1;
      if (u < cdf[mid]) hi = mid; else lo = mid + 1;
    }
    uint64_t key = or_mix64(lo ^ salt);
    store_key(out, (uint64_t)i, kb, kb == 8 ? key : (key & 0xffffffffull));
  }
}

/* ---------------------------------------------------------------------------
 * CSR build.  Reference: hash (hashValuesD / basicHashD), per-bucket count
 * (countHashD, SingleHashGraphOperators.cuh:81-87), exclusive scan with
 * offsets[tableSize] = n (src/SingleHashGraph.cu:199-207), then scatter via a
 * second per-bucket cursor (copyToGraphD, :89-100).  The oracle uses a stable
 * counting sort, so keys inside a bucket keep input order; the reference's
 * in-bucket order is nondeterministic, so parity compares canonical
 * (sorted) buckets.
 * ------------------------------------------------------------------------- */
int or_build(const void* keys, uint64_t n, int kb, uint64_t B, uint32_t* offsets,
             void* keys_out, uint32_t* idx_out) {
  if (B == 0 || n >= (1ull << 32)) return -1;
  uint32_t* cursor = (uint32_t*)calloc(B + 1, sizeof(uint32_t));
  if (!cursor) return -2;
  for (uint64_t i = 0; i < n; i++) cursor[or_bucket(load_key(keys, i, kb), B)]++;
  uint32_t run = 0;
  for (uint64_t b = 0; b < B; b++) {
    uint32_t c = cursor[b];
    offsets[b] = run;
    cursor[b] = run;
    run += c;
  }
  offsets[B] = (uint32_t)n;
  for (uint64_t i = 0; i < n; i++) {
    uint64_t k = load_key(keys, i, kb);
    uint32_t pos = cursor[or_bucket(k, B)]++;
    store_key(keys_out, pos, kb, k);
    if (idx_out) idx_out[pos] = (uint32_t)i;
  }
  free(cursor);
  return 0;
}

/* Multithreaded form of the same stable build (the CPU baseline): per-thread
 * partition histograms over bucket ranges, a scan, a stable scatter into
 * partition order, then an independent counting sort per bucket range. */
int or_build_mt(const void* keys, uint64_t n, int kb, uint64_t B, uint32_t* offsets,
                void* keys_out, uint32_t* idx_out, int threads) {
  if (B == 0 || n >= (1ull << 32)) return -1;
  if (threads <= 0) threads = omp_get_max_threads();
  uint64_t W = 1;
  while ((B + W - 1) / W > 4096) W <<= 1;
  uint64_t P = (B + W - 1) / W;
  uint64_t* hist = (uint64_t*)calloc((size_t)threads * P, sizeof(uint64_t));
  uint64_t* tmp_k = (uint64_t*)malloc((size_t)(n ? n : 1) * 8);
  uint32_t* tmp_i = (uint32_t*)malloc((size_t)(n ? n : 1) * 4);
  uint64_t* pstart = (uint64_t*)malloc((P + 1) * sizeof(uint64_t));
  if (!hist || !tmp_k || !tmp_i || !pstart) {
    free(hist); free(tmp_k); free(tmp_i); free(pstart);
    return -2;
  }
  #pragma omp parallel num_threads(threads)
  {
    int t = omp_get_thread_num();
    int nt = omp_get_num_threads();
    uint64_t lo = n * (uint64_t)t / (uint64_t)nt, hi = n * (uint64_t)(t + 1) / (uint64_t)nt;
    uint64_t* h = hist + (size_t)t * P;
    for (uint64_t i = lo; i < hi; i++) h[or_bucket(load_key(keys, i, kb), B) / W]++;
    #pragma omp barrier
    #pragma omp single
    {
      uint64_t run = 0;
      for (uint64_t p = 0; p < P; p++) {
        pstart[p] = run;
        for (int u = 0; u < nt; u++) {
          uint64_t c = hist[(size_t)u * P + p];
          hist[(size_t)u * P + p] = run;
          run += c;
        }
      }
      pstart[P] = run;
    }
    for (uint64_t i = lo; i < hi; i++) {
      uint64_t k = load_key(keys, i, kb);
      uint64_t pos = h[or_bucket(k, B) / W]++;
      tmp_k[pos] = k;
      tmp_i[pos] = (uint32_t)i;
    }
    #pragma omp barrier
    uint32_t* cnt = (uint32_t*)malloc((size_t)W * sizeof(uint32_t));
    #pragma omp for schedule(dynamic, 4)
    for (int64_t p = 0; p < (int64_t)P; p++) {
      uint64_t b0 = (uint64_t)p * W, b1 = b0 + W < B ? b0 + W : B;
      memset(cnt, 0, (size_t)W * sizeof(uint32_t));
      for (uint64_t j = pstart[p]; j < pstart[p + 1]; j++) cnt[or_bucket(tmp_k[j], B) - b0]++;
      uint32_t run = (uint32_t)pstart[p];
      for (uint64_t b = b0; b < b1; b++) {
        uint32_t c = cnt[b - b0];
        offsets[b] = run;
        cnt[b - b0] = run;
        run += c;
      }
      for (uint64_t j = pstart[p]; j < pstart[p + 1]; j++) {
        uint64_t k = tmp_k[j];
        uint32_t pos = cnt[or_bucket(k, B) - b0]++;
        store_key(keys_out, pos, kb, k);
        if (idx_out) idx_out[pos] = tmp_i[j];
      }
    }
    free(cnt);
  }
  offsets[B] = (uint32_t)n;
  free(hist); free(tmp_k); free(tmp_i); free(pstart);
  return 0;
}

/* Canonical bucket order: ascending (key, idx).  Short buckets take an
 * insertion sort; long ones (heavy duplicates, hot buckets) a qsort of
 * (key, idx) records, so a bucket of millions of entries stays O(L log L). */
typedef struct { uint64_t key; uint32_t idx; } or_rec;

static int or_rec_cmp(const void* x, const void* y) {
  const or_rec* a = (const or_rec*)x;
  const or_rec* b = (const or_rec*)y;
  if (a->key != b->key) return a->key < b->key ? -1 : 1;
  return (a->idx > b->idx) - (a->idx < b->idx);
}

void or_canonicalize(const uint32_t* offsets, uint64_t B, void* keys, int kb, uint32_t* idx) {
  #pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t b = 0; b < (int64_t)B; b++) {
    uint32_t s = offsets[b], e = offsets[b + 1];
    if (e - s > 32) {
      or_rec* r = (or_rec*)malloc((size_t)(e - s) * sizeof(or_rec));
      if (r) {
        for (uint32_t j = s; j < e; j++) {
          r[j - s].key = load_key(keys, j, kb);
          r[j - s].idx = idx ? idx[j] : 0;
        }
        qsort(r, e - s, sizeof(or_rec), or_rec_cmp);
        for (uint32_t j = s; j < e; j++) {
          store_key(keys, j, kb, r[j - s].key);
          if (idx) idx[j] = r[j - s].idx;
        }
        free(r);
        continue;
      }
    }
    for (uint32_t j = s + 1; j < e; j++) {
      uint64_t k = load_key(keys, j, kb);
      uint32_t x = idx ? idx[j] : 0;
      uint32_t m = j;
      while (m > s) {
        uint64_t pk = load_key(keys, m - 1, kb);
        uint32_t px = idx ? idx[m - 1] : 0;
        if (pk < k || (pk == k && px <= x)) break;
        store_key(keys, m, kb, pk);
        if (idx) idx[m] = px;
        m--;
      }
      store_key(keys, m, kb, k);
      if (idx) idx[m] = x;
    }
  }
}

/* ---------------------------------------------------------------------------
 * Intersect.  The reference joins two CSRs bucket by bucket and, for every
 * equal (aKey, bKey) pair in the same bucket, counts or emits one match
 * (simpleIntersect, include/MultiHashGraphDeviceOperators.cuh:513-543):
 * multiset-join semantics.  Probing each query's bucket in A gives the same
 * multiset of matches.
 * ------------------------------------------------------------------------- */
static inline uint64_t probe_one(const uint32_t* off, uint64_t B, const void* a_keys,
                                 const uint32_t* a_idx, int kb, uint64_t q, uint32_t q_ref,
                                 uint32_t* pairs, uint64_t pos, uint64_t cap) {
  uint64_t b = or_bucket(q, B);
  uint64_t c = 0;
  for (uint32_t j = off[b]; j < off[b + 1]; j++) {
    if (load_key(a_keys, j, kb) == q) {
      if (pairs && pos + c < cap) {
        pairs[2 * (pos + c)] = a_idx ? a_idx[j] : j;
        pairs[2 * (pos + c) + 1] = q_ref;
      }
      c++;
    }
  }
  return c;
}

uint64_t or_intersect(const uint32_t* off, uint64_t B, const void* a_keys, const uint32_t* a_idx,
                      int kb, const void* q_keys, uint64_t nq, const uint32_t* q_idx,
                      uint32_t* pairs, uint64_t cap) {
  uint64_t total = 0;
  for (uint64_t i = 0; i < nq; i++)
    total += probe_one(off, B, a_keys, a_idx, kb, load_key(q_keys, i, kb),
                       q_idx ? q_idx[i] : (uint32_t)i, pairs, total, cap);
  return total;
}

uint64_t or_intersect_mt(const uint32_t* off, uint64_t B, const void* a_keys, const uint32_t* a_idx,
                         int kb, const void* q_keys, uint64_t nq, uint32_t* pairs, uint64_t cap,
                         int threads) {
  if (threads <= 0) threads = omp_get_max_threads();
  uint64_t* part = (uint64_t*)calloc((size_t)threads + 1, sizeof(uint64_t));
  uint64_t total = 0;
  #pragma omp parallel num_threads(threads)
  {
    int t = omp_get_thread_num();
    int nt = omp_get_num_threads();
    uint64_t lo = nq * (uint64_t)t / (uint64_t)nt, hi = nq * (uint64_t)(t + 1) / (uint64_t)nt;
    uint64_t c = 0;
    for (uint64_t i = lo; i < hi; i++)
      c += probe_one(off, B, a_keys, a_idx, kb, load_key(q_keys, i, kb), (uint32_t)i, NULL, 0, 0);
    part[t + 1] = c;
    #pragma omp barrier
    #pragma omp single
    {
      for (int u = 0; u < nt; u++) part[u + 1] += part[u];
      total = part[nt];
    }
    if (pairs) {
      uint64_t pos = part[t];
      for (uint64_t i = lo; i < hi; i++)
        pos += probe_one(off, B, a_keys, a_idx, kb, load_key(q_keys, i, kb), (uint32_t)i,
                         pairs, pos, cap);
    }
  }
  free(part);
  return total;
}

uint64_t or_join_count_sorted(const void* a, uint64_t na, const void* b, uint64_t nb, int kb) {
  uint64_t i = 0, j = 0, total = 0;
  while (i < na && j < nb) {
    uint64_t x = load_key(a, i, kb), y = load_key(b, j, kb);
    if (x < y) { i++; continue; }
    if (y < x) { j++; continue; }
    uint64_t ci = 0, cj = 0;
    while (i < na && load_key(a, i, kb) == x) { i++; ci++; }
    while (j < nb && load_key(b, j, kb) == x) { j++; cj++; }
    total += ci * cj;
  }
  return total;
}

/* The same count, sum over keys of multA(k) * multB(k), through a hash map of
 * A's distinct keys and their multiplicities (open addressing, CAS inserts);
 * linear in na + nb, so it also checks heavily skewed inputs at full size,
 * where probing every query's bucket costs the product of the multiplicities.
 * Returns UINT64_MAX when the map cannot be allocated. */
#define OR_EMPTY_SLOT 0xFFFFFFFFFFFFFFFFull
uint64_t or_join_count_hashed(const void* a, uint64_t na, const void* b, uint64_t nb, int kb,
                              uint64_t max_distinct, int threads) {
  if (threads <= 0) threads = omp_get_max_threads();
  uint64_t cap = 1024;
  uint64_t want = max_distinct < na ? max_distinct : na;
  while (cap < 2 * want) cap <<= 1;
  uint64_t* slot_key = (uint64_t*)malloc((size_t)cap * sizeof(uint64_t));
  uint64_t* slot_cnt = (uint64_t*)calloc((size_t)cap, sizeof(uint64_t));
  if (!slot_key || !slot_cnt) { free(slot_key); free(slot_cnt); return UINT64_MAX; }
  for (uint64_t i = 0; i < cap; i++) slot_key[i] = OR_EMPTY_SLOT;
  uint64_t empty_key_count = 0, full = 0;  /* the key equal to the empty marker */
  const uint64_t mask = cap - 1;
  #pragma omp parallel for num_threads(threads) schedule(static) reduction(+ : empty_key_count)
  for (int64_t i = 0; i < (int64_t)na; i++) {
    uint64_t k = load_key(a, (uint64_t)i, kb);
    if (k == OR_EMPTY_SLOT) { empty_key_count++; continue; }
    uint64_t h = or_mix64(k) & mask, probes = 0;
    for (;;) {
      uint64_t cur = __atomic_load_n(&slot_key[h], __ATOMIC_ACQUIRE);
      if (cur == k) { __atomic_fetch_add(&slot_cnt[h], 1, __ATOMIC_RELAXED); break; }
      if (cur == OR_EMPTY_SLOT) {
        uint64_t expect = OR_EMPTY_SLOT;
        if (__atomic_compare_exchange_n(&slot_key[h], &expect, k, 0, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE) ||
            expect == k) {
          __atomic_fetch_add(&slot_cnt[h], 1, __ATOMIC_RELAXED);
          break;
        }
        continue;  /* another key took the slot: look at it again */
      }
      h = (h + 1) & mask;
      if (++probes > cap) { __atomic_store_n(&full, 1, __ATOMIC_RELAXED); break; }
    }
  }
  uint64_t total = 0;
  if (!full) {
    #pragma omp parallel for num_threads(threads) schedule(static) reduction(+ : total)
    for (int64_t i = 0; i < (int64_t)nb; i++) {
      uint64_t k = load_key(b, (uint64_t)i, kb);
      if (k == OR_EMPTY_SLOT) { total += empty_key_count; continue; }
      uint64_t h = or_mix64(k) & mask;
      for (;;) {
        uint64_t cur = slot_key[h];
        if (cur == k) { total += slot_cnt[h]; break; }
        if (cur == OR_EMPTY_SLOT) break;
        h = (h + 1) & mask;
      }
    }
  }
  free(slot_key);
  free(slot_cnt);
  return full ? UINT64_MAX : total;
}

int or_max_threads(void) { return omp_get_max_threads(); }
