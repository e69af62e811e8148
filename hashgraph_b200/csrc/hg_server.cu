// hg_server.cu -- a native serving engine: resident tables under a device
// memory budget with least-recently-used eviction, build and intersect
// requests spread over a pool of CUDA streams, and per-request latency.
//
// The reference has no serving component (its tables are built and
// intersected once per process, test/MultiHashGraphTest.cu:288-338).  A
// request costs one library call here, a few microseconds of host time, so
// the host keeps up with tens of thousands of requests per second.
//
// Ordering between streams:
//   * an intersect waits (cudaStreamWaitEvent) for its table's build;
//   * a table's memory is freed stream-ordered on the stream that built it,
//     after that stream has waited for everything already queued on every
//     stream, so no kernel still reading an evicted table loses its memory.
// Tables come from the server's own stream-ordered memory pool, whose
// release threshold is the budget: memory freed by an eviction is reused by
// the next build instead of being unmapped at the next synchronisation.
// Latency = arrival time (the caller's CLOCK_MONOTONIC stamp) to the device
// completion of the request's last operation, mapped onto the host clock by
// a reference event (re-taken every REF_MAX_AGE_S).
//
// Continuous batching: a request of at most `batch_small` keys is not
// launched on its own.  It joins a queue, and the queue is flushed as ONE
// batched launch sequence (hg_batch: build-only pairs for the queued builds,
// probe-only pairs for the queued intersects, against resident tables or
// tables built in the same batch) when it holds `batch_max` requests, when
// its oldest request has waited `batch_wait` seconds (checked at every poll),
// before any request that is launched on its own (so requests keep their
// order), and when the caller blocks for completions.  A flush is cut into
// segments in submission order; a batch builds all its tables before it
// probes, so that every intersect sees the tables the requests before it
// left, a build starts a new segment when the segment already builds that
// table or one of its intersects reads it (any other build joins, and the
// tables the segment's intersects read are kept from eviction).  Each
// segment takes one stream, waits for the builds (on other streams) of the
// tables it probes, and uploads its descriptors from a pinned ring buffer
// without synchronising.
#include <time.h>

#include <algorithm>
#include <deque>
#include <list>
#include <unordered_map>
#include <vector>

#include "hg_device.cuh"
#include "hg_plan.h"

namespace hg {

struct ServerTable {
  uint64_t n = 0, n_buckets = 0;
  bool with_index = false;
  uint32_t* offsets = nullptr;
  void* keys = nullptr;
  uint32_t* idx = nullptr;
  size_t bytes = 0;
  int stream = 0;             // the stream that built it (its memory is freed there)
  cudaEvent_t ready = nullptr;
  std::list<uint64_t>::iterator lru;
};

struct ServerReq {
  uint64_t ticket;
  int kind;                   // 0 build, 1 intersect
  int missed;
  double arrival;
  cudaEvent_t done;
  uint32_t slot;              // count slot (intersect)
};

// A request waiting in the batching queue.
struct QueuedReq {
  int kind;                   // 0 build, 1 intersect
  uint64_t table_id;
  const void* data;           // keys (build) or queries (intersect)
  uint64_t n, n_buckets;
  int with_index;
  uint32_t* d_pairs;
  uint64_t pair_cap;
  double arrival;
  uint64_t ticket;
};

constexpr size_t STAGE_BYTES = size_t(4) << 20;  // pinned descriptor buffer of one batch
constexpr size_t BATCH_MIN_REQUESTS = 4;          // smaller segments are launched request by request
constexpr int STAGE_RING = 8;

static double monotonic_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return double(ts.tv_sec) + 1e-9 * double(ts.tv_nsec);
}

}  // namespace hg

struct hg_server {
  int device = 0, key_bytes = 8, max_tables = 0;
  size_t budget = 0, bytes = 0, ws_bytes = 0;
  uint64_t max_keys = 0, evictions = 0, next_ticket = 1;
  std::vector<cudaStream_t> streams;
  std::vector<void*> ws;
  std::vector<uint32_t*> pair_buf;
  std::vector<double> busy_until;
  std::unordered_map<uint64_t, hg::ServerTable> tables;
  std::list<uint64_t> lru;    // least recently used first
  std::deque<hg::ServerReq> inflight;
  unsigned long long* d_counts = nullptr;
  unsigned long long* h_counts = nullptr;  // pinned
  uint32_t n_slots = 0, next_slot = 0;
  std::vector<uint8_t> slot_busy;
  std::vector<cudaEvent_t> free_events;
  std::unordered_map<cudaEvent_t, uint32_t> event_refs;  // requests sharing one completion event (a batch)
  cudaMemPool_t pool = nullptr;
  cudaStream_t clock_stream = nullptr;  // carries only `ref`, so `ref` completes at once
  cudaEvent_t ref = nullptr;
  double ref_host = 0;
  // continuous batching
  bool batching = true;
  uint64_t batch_small = 1ull << 16;
  uint32_t batch_max = 256;
  double batch_wait = 100e-6;
  std::vector<hg::QueuedReq> queue;
  double queued_since = 0;
  std::vector<void*> stage;             // pinned descriptor buffers (a ring)
  std::vector<cudaEvent_t> stage_done;  // recorded after the batch that used the buffer
  std::vector<uint8_t> stage_used;
  size_t stage_next = 0;
  uint64_t batches = 0, batched_requests = 0;
};

namespace hg {

static cudaEvent_t take_event(hg_server* s) {
  if (!s->free_events.empty()) {
    cudaEvent_t e = s->free_events.back();
    s->free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Frees a table's memory stream-ordered after everything queued so far.
static void release_table(hg_server* s, ServerTable& t) {
  cudaStream_t home = s->streams[t.stream];
  for (size_t i = 0; i < s->streams.size(); i++) {
    if (int(i) == t.stream) continue;
    cudaEvent_t e = take_event(s);
    cudaEventRecord(e, s->streams[i]);
    cudaStreamWaitEvent(home, e, 0);
    s->free_events.push_back(e);  // reusable: the wait is already queued
  }
  if (t.offsets) cudaFreeAsync(t.offsets, home);
  if (t.keys) cudaFreeAsync(t.keys, home);
  if (t.idx) cudaFreeAsync(t.idx, home);
  if (t.ready) cudaEventDestroy(t.ready);
  s->bytes -= t.bytes;
}

static void evict(hg_server* s, uint64_t id) {
  auto it = s->tables.find(id);
  if (it == s->tables.end()) return;
  release_table(s, it->second);
  s->lru.erase(it->second.lru);
  s->tables.erase(it);
}

// Evicts least recently used tables until `need` more bytes and one more
// table fit.  Tables in `pinned` (built by the batch being planned, not yet
// launched) are never evicted; if only they are left, the budget is exceeded
// until the next build.
static void make_room(hg_server* s, size_t need, const std::vector<uint64_t>* pinned = nullptr) {
  auto it = s->lru.begin();
  while (it != s->lru.end() && (s->bytes + need > s->budget || s->tables.size() >= size_t(s->max_tables))) {
    const uint64_t id = *it++;
    if (pinned && std::find(pinned->begin(), pinned->end(), id) != pinned->end()) continue;
    evict(s, id);
    s->evictions++;
  }
}

static int pick_stream(hg_server* s, double est) {
  const double now = monotonic_s();
  int best = 0;
  for (size_t i = 1; i < s->streams.size(); i++)
    if (std::max(s->busy_until[i], now) < std::max(s->busy_until[best], now)) best = int(i);
  s->busy_until[best] = std::max(s->busy_until[best], now) + est;
  return best;
}

// Count slots: the next free one after the last handed out; a slot is busy
// from its intersect's submission until poll has read its count.
static hg_status reserve_slot(hg_server* s, uint32_t* slot) {
  for (uint32_t k = 0; k < s->n_slots; k++) {
    const uint32_t c = (s->next_slot + k) % s->n_slots;
    if (!s->slot_busy[c]) {
      s->slot_busy[c] = 1;
      s->next_slot = (c + 1) % s->n_slots;
      *slot = c;
      return HG_OK;
    }
  }
  return lib_fail(HG_ERR_TOO_LARGE, "hg_server: 65536 intersects in flight; poll before submitting more");
}

// `count` contiguous count slots (one copy brings a batch's counts back), or
// HG_ERR_TOO_LARGE when no such run is free.
static hg_status reserve_slot_run(hg_server* s, uint32_t count, uint32_t* first) {
  if (count == 0 || count > s->n_slots) return HG_ERR_TOO_LARGE;
  uint32_t start = s->next_slot + count <= s->n_slots ? s->next_slot : 0;
  for (uint32_t tries = 0; tries < s->n_slots; tries++) {
    uint32_t k = 0;
    while (k < count && !s->slot_busy[start + k]) k++;
    if (k == count) {
      for (uint32_t j = 0; j < count; j++) s->slot_busy[start + j] = 1;
      *first = start;
      s->next_slot = (start + count) % s->n_slots;
      return HG_OK;
    }
    start = start + k + 1;
    if (start + count > s->n_slots) start = 0;
  }
  return lib_fail(HG_ERR_TOO_LARGE, "hg_server: no free run of count slots; poll before submitting more");
}

// The latency clock: a request's completion is its event's time after `ref`
// (a float count of milliseconds) added to ref_host, the host time of `ref`.
// The GPU's event timer and the host clock drift apart by tens of
// microseconds over seconds, so `ref` is re-taken at a poll when it is more
// than REF_MAX_AGE_S old.  It is recorded on a stream of its own that carries
// no work, so it completes at once whatever the other streams hold; ref_host
// is the midpoint of the record and the synchronisation that saw it.
constexpr double REF_MAX_AGE_S = 0.1;

static cudaError_t rebase_clock(hg_server* s) {
  const double t0 = monotonic_s();
  cudaError_t e = cudaEventRecord(s->ref, s->clock_stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(s->ref);
  if (e == cudaSuccess) s->ref_host = 0.5 * (t0 + monotonic_s());
  return e;
}

// One request launched on its own (a library call on the least busy stream).
static hg_status direct_build(hg_server* s, const QueuedReq& r, const std::vector<uint64_t>* pinned) {
  const size_t bytes = (r.n_buckets + 1) * 4 + r.n * (s->key_bytes + (r.with_index ? 4 : 0));
  if (s->tables.count(r.table_id)) evict(s, r.table_id);  // replaced
  make_room(s, bytes, pinned);
  const int si = pick_stream(s, 20e-6 + double(r.n) * 4e-11);
  cudaStream_t st = s->streams[si];
  ServerTable t;
  t.n = r.n;
  t.n_buckets = r.n_buckets;
  t.with_index = r.with_index != 0;
  t.bytes = bytes;
  t.stream = si;
  cudaError_t e = cudaMallocFromPoolAsync(&t.offsets, (r.n_buckets + 1) * 4, s->pool, st);
  if (e == cudaSuccess && r.n) e = cudaMallocFromPoolAsync(&t.keys, r.n * s->key_bytes, s->pool, st);
  if (e == cudaSuccess && r.n && r.with_index)
    e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&t.idx), r.n * 4, s->pool, st);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t.ready, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (t.offsets) cudaFreeAsync(t.offsets, st);
    if (t.keys) cudaFreeAsync(t.keys, st);
    if (t.idx) cudaFreeAsync(t.idx, st);
    return cuda_fail(e, "hg_server_build: table allocation");
  }
  hg_status hs = hg_build_into(r.data, r.n, s->key_bytes, r.n_buckets, t.offsets, t.keys, t.idx,
                               s->ws[si], s->ws_bytes, reinterpret_cast<hg_stream_t>(st));
  if (hs != HG_OK) {
    cudaFreeAsync(t.offsets, st);
    if (t.keys) cudaFreeAsync(t.keys, st);
    if (t.idx) cudaFreeAsync(t.idx, st);
    cudaEventDestroy(t.ready);
    return hs;
  }
  cudaEventRecord(t.ready, st);
  s->lru.push_back(r.table_id);
  t.lru = std::prev(s->lru.end());
  s->bytes += bytes;
  s->tables.emplace(r.table_id, t);
  ServerReq q{r.ticket, 0, 0, r.arrival, take_event(s), 0};
  cudaEventRecord(q.done, st);
  s->inflight.push_back(q);
  return HG_OK;
}

static hg_status direct_intersect(hg_server* s, const QueuedReq& r) {
  uint32_t slot = 0;
  hg_status hs = reserve_slot(s, &slot);
  if (hs != HG_OK) return hs;
  auto it = s->tables.find(r.table_id);
  const int si = pick_stream(s, 20e-6 + double(r.n) * 4e-11);
  cudaStream_t st = s->streams[si];
  ServerReq q{r.ticket, 1, 0, r.arrival, take_event(s), slot};
  if (it == s->tables.end()) {
    q.missed = 1;
  } else {
    ServerTable& t = it->second;
    s->lru.splice(s->lru.end(), s->lru, t.lru);  // most recently used
    cudaStreamWaitEvent(st, t.ready, 0);
    uint32_t* pairs = r.d_pairs ? r.d_pairs : s->pair_buf[si];
    const uint64_t cap = r.d_pairs ? r.pair_cap : std::min<uint64_t>(r.pair_cap, s->max_keys);
    hs = hg_intersect_into(t.offsets, t.keys, t.idx, t.n, t.n_buckets, s->key_bytes, r.data, r.n, nullptr, pairs,
                           cap, s->d_counts + slot, s->ws[si], s->ws_bytes, reinterpret_cast<hg_stream_t>(st));
    if (hs != HG_OK) {
      s->free_events.push_back(q.done);
      s->slot_busy[slot] = 0;
      return hs;
    }
    cudaMemcpyAsync(s->h_counts + slot, s->d_counts + slot, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  }
  cudaEventRecord(q.done, st);
  s->inflight.push_back(q);
  return HG_OK;
}

// True when a queued request names `table_id`.
static bool queue_touches(const hg_server* s, uint64_t table_id) {
  for (const QueuedReq& q : s->queue)
    if (q.table_id == table_id) return true;
  return false;
}

// Launches one segment of the queue (builds, then intersects) as one batch.
static hg_status launch_segment(hg_server* s, const QueuedReq* q, size_t n) {
  uint64_t keys = 0;
  uint32_t isects = 0;
  for (size_t i = 0; i < n; i++) {
    keys += q[i].n;
    isects += q[i].kind == 1;
  }
  uint32_t slot0 = 0, n_isect = 0;  // the segment's intersects count into slots [slot0, slot0 + isects)
  if (isects) {
    hg_status hs = reserve_slot_run(s, isects, &slot0);
    if (hs != HG_OK) return hs;
  }
  const int si = pick_stream(s, 20e-6 + double(keys) * 4e-11);
  cudaStream_t st = s->streams[si];
  std::vector<hg_batch_pair> pairs;
  std::vector<ServerReq> reqs;
  std::vector<uint64_t> built;  // table ids this segment builds
  std::vector<uint64_t> pinned;  // ... and the ids its intersects read: not evicted to make room
  // on failure: the segment's count slots are freed and the tables it
  // registered (never built) are dropped; its requests are not reported
  auto fail = [&](hg_status status) {
    for (uint32_t j = 0; j < isects; j++) s->slot_busy[slot0 + j] = 0;
    for (uint64_t id : built) evict(s, id);
    return status;
  };
  pairs.reserve(n);
  reqs.reserve(n);
  for (size_t i = 0; i < n; i++) {
    const QueuedReq& r = q[i];
    ServerReq sr{r.ticket, r.kind, 0, r.arrival, nullptr, 0};
    if (r.kind == 0) {
      const size_t bytes = (r.n_buckets + 1) * 4 + r.n * (s->key_bytes + (r.with_index ? 4 : 0));
      if (s->tables.count(r.table_id)) evict(s, r.table_id);  // replaced (neither built nor read in this segment)
      make_room(s, bytes, &pinned);
      ServerTable t;
      t.n = r.n;
      t.n_buckets = r.n_buckets;
      t.with_index = r.with_index != 0;
      t.bytes = bytes;
      t.stream = si;
      cudaError_t e = cudaMallocFromPoolAsync(&t.offsets, (r.n_buckets + 1) * 4, s->pool, st);
      if (e == cudaSuccess && r.n) e = cudaMallocFromPoolAsync(&t.keys, r.n * s->key_bytes, s->pool, st);
      if (e == cudaSuccess && r.n && r.with_index)
        e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&t.idx), r.n * 4, s->pool, st);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t.ready, cudaEventDisableTiming);
      if (e != cudaSuccess) {
        cudaGetLastError();
        if (t.offsets) cudaFreeAsync(t.offsets, st);
        if (t.keys) cudaFreeAsync(t.keys, st);
        if (t.idx) cudaFreeAsync(t.idx, st);
        return fail(cuda_fail(e, "hg_server: table allocation"));
      }
      s->lru.push_back(r.table_id);
      t.lru = std::prev(s->lru.end());
      s->bytes += bytes;
      s->tables.emplace(r.table_id, t);
      built.push_back(r.table_id);
      pinned.push_back(r.table_id);
      pairs.push_back(hg_batch_pair{r.data, r.n, r.n_buckets, nullptr, 0, t.offsets, t.keys, t.idx, nullptr, 0,
                                    nullptr});
    } else {
      const uint32_t slot = slot0 + n_isect++;
      sr.slot = slot;
      pinned.push_back(r.table_id);
      auto it = s->tables.find(r.table_id);
      if (it == s->tables.end()) {
        sr.missed = 1;
      } else {
        ServerTable& t = it->second;
        s->lru.splice(s->lru.end(), s->lru, t.lru);
        if (std::find(built.begin(), built.end(), r.table_id) == built.end() && t.stream != si)
          cudaStreamWaitEvent(st, t.ready, 0);
        pairs.push_back(hg_batch_pair{nullptr, t.n, t.n_buckets, r.data, r.n, t.offsets, t.keys, t.idx, r.d_pairs,
                                      r.d_pairs ? r.pair_cap : 0, s->d_counts + slot});
      }
    }
    reqs.push_back(sr);
  }
  if (!pairs.empty()) {
    const size_t k = s->stage_next;
    s->stage_next = (k + 1) % s->stage.size();
    if (s->stage_used[k]) HG_CUDA(cudaEventSynchronize(s->stage_done[k]), "hg_server: descriptor buffer");
    hg_batch* b = nullptr;
    hg_status hs = batch_create_staged(pairs.data(), int(pairs.size()), s->key_bytes, nullptr, st, s->pool,
                                       s->stage[k], STAGE_BYTES, &b);
    if (hs != HG_OK) return fail(hs);
    hs = hg_batch_run(b, reinterpret_cast<hg_stream_t>(st));
    hg_batch_free(b, reinterpret_cast<hg_stream_t>(st));
    if (hs != HG_OK) return fail(hs);
    HG_CUDA(cudaEventRecord(s->stage_done[k], st), "hg_server: event");
    s->stage_used[k] = 1;
    s->batches++;
    s->batched_requests += n;
  }
  for (uint64_t id : built) cudaEventRecord(s->tables[id].ready, st);
  if (isects) {  // missed intersects' slots are zeroed on the device first, so one copy serves all
    for (const ServerReq& sr : reqs)
      if (sr.kind == 1 && sr.missed) cudaMemsetAsync(s->d_counts + sr.slot, 0, sizeof(unsigned long long), st);
    cudaMemcpyAsync(s->h_counts + slot0, s->d_counts + slot0, sizeof(unsigned long long) * isects,
                    cudaMemcpyDeviceToHost, st);
  }
  cudaEvent_t done = take_event(s);  // one completion event for the whole segment
  cudaEventRecord(done, st);
  s->event_refs[done] = static_cast<uint32_t>(reqs.size());
  for (ServerReq& sr : reqs) {
    sr.done = done;
    s->inflight.push_back(sr);
  }
  return HG_OK;
}

// Launches every queued request in segments of at most batch_max requests
// (a build of a table the segment already builds or reads starts the next
// one, and so does a request that would take the segment's tables to the
// table limit or its builds past half the budget).
static hg_status flush_queue(hg_server* s) {
  size_t i = 0;
  const size_t n = s->queue.size();
  hg_status st = HG_OK;
  while (i < n && st == HG_OK) {
    size_t j = i;
    std::vector<uint64_t> builds, reads;
    size_t pinned = 0, build_bytes = 0;  // distinct tables the segment holds; bytes it builds
    auto has = [](const std::vector<uint64_t>& v, uint64_t id) { return std::find(v.begin(), v.end(), id) != v.end(); };
    while (j < n && j - i < s->batch_max) {
      const QueuedReq& r = s->queue[j];
      const bool fresh = !has(builds, r.table_id) && !has(reads, r.table_id);
      // the tables a segment builds or reads cannot be evicted while it is
      // planned: it stops short of the table limit and of half the budget
      if (fresh && j > i && pinned + 1 >= size_t(s->max_tables)) break;
      if (r.kind == 0) {
        // a batch builds all its tables before it probes: a build joins the
        // segment unless the segment builds the same table already or one of
        // its intersects reads that table (it must see the version before)
        if (!fresh) break;
        const size_t bytes = (r.n_buckets + 1) * 4 + r.n * (s->key_bytes + (r.with_index ? 4 : 0));
        if (!builds.empty() && build_bytes + bytes > s->budget / 2) break;
        build_bytes += bytes;
        builds.push_back(r.table_id);
      } else {
        reads.push_back(r.table_id);
      }
      pinned += fresh;
      j++;
    }
    if (j - i < BATCH_MIN_REQUESTS) {  // too few to pay for a batch's fixed launches
      for (size_t k = i; k < j && st == HG_OK; k++) {
        const QueuedReq& r = s->queue[k];
        st = r.kind == 0 ? direct_build(s, r, nullptr) : direct_intersect(s, r);
      }
    } else {
      st = launch_segment(s, s->queue.data() + i, j - i);
    }
    i = j;
  }
  s->queue.clear();
  return st;
}

static hg_status enqueue(hg_server* s, const QueuedReq& r) {
  if (s->queue.empty()) s->queued_since = monotonic_s();
  s->queue.push_back(r);
  if (s->queue.size() >= s->batch_max) return flush_queue(s);
  return HG_OK;
}

}  // namespace hg

using namespace hg;

extern "C" double hg_server_now(void) { return monotonic_s(); }

extern "C" void hg_server_free(hg_server* s) {
  if (!s) return;
  if (!s->queue.empty()) flush_queue(s);  // queued requests still run: their inputs may be the caller's to reuse
  for (auto& st : s->streams) cudaStreamSynchronize(st);
  if (!s->streams.empty()) {
    cudaStream_t st = s->streams[0];
    for (auto& kv : s->tables) {
      if (kv.second.offsets) cudaFreeAsync(kv.second.offsets, st);
      if (kv.second.keys) cudaFreeAsync(kv.second.keys, st);
      if (kv.second.idx) cudaFreeAsync(kv.second.idx, st);
      if (kv.second.ready) cudaEventDestroy(kv.second.ready);
    }
    cudaStreamSynchronize(st);
  }
  {
    std::vector<cudaEvent_t> evs;
    for (auto& r : s->inflight) evs.push_back(r.done);
    std::sort(evs.begin(), evs.end());
    evs.erase(std::unique(evs.begin(), evs.end()), evs.end());
    for (auto e : evs) cudaEventDestroy(e);
  }
  for (auto e : s->free_events) cudaEventDestroy(e);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  for (auto p : s->ws) cudaFree(p);
  for (auto p : s->pair_buf) cudaFree(p);
  if (s->d_counts) cudaFree(s->d_counts);
  if (s->h_counts) cudaFreeHost(s->h_counts);
  for (auto h : s->stage) cudaFreeHost(h);
  for (auto e : s->stage_done) cudaEventDestroy(e);
  if (s->ref) cudaEventDestroy(s->ref);
  if (s->clock_stream) cudaStreamDestroy(s->clock_stream);
  for (auto& st : s->streams) cudaStreamDestroy(st);
  delete s;
}

extern "C" hg_status hg_server_create(size_t budget_bytes, int max_tables, int n_streams, uint64_t max_keys,
                                      int key_bytes, hg_server** out) {
  if (!out) return HG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (key_bytes != 4 && key_bytes != 8) return HG_ERR_KEY_WIDTH;
  if (max_tables <= 0 || n_streams <= 0 || n_streams > 64 || max_keys == 0 || budget_bytes == 0)
    return lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_server_create: tables, streams, keys and budget must be positive");
  if (max_keys >= (1ull << 32)) return lib_fail(HG_ERR_TOO_LARGE, "hg_server_create: max_keys must be below 2^32");
  size_t wb = 0, wq = 0;
  BuildPlan bp;
  ProbePlan pp;
  hg_status st = plan_build(max_keys, key_bytes, max_keys, true, &bp);
  if (st != HG_OK) return st;
  st = plan_probe(max_keys, true, max_keys, max_keys, key_bytes, true, &pp);
  if (st != HG_OK) return st;
  wb = bp.total;
  wq = pp.total;
  hg_server* s = new hg_server();
  cudaGetDevice(&s->device);
  s->key_bytes = key_bytes;
  s->max_tables = max_tables;
  s->budget = budget_bytes;
  s->max_keys = max_keys;
  s->ws_bytes = std::max(wb, wq);
  s->n_slots = 1u << 16;
  s->slot_busy.assign(s->n_slots, 0);
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s->device;
  cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
  if (e == cudaSuccess) {
    uint64_t keep = budget_bytes;
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  for (int i = 0; i < n_streams && e == cudaSuccess; i++) {
    cudaStream_t x = nullptr;
    e = cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking);
    if (e != cudaSuccess) break;
    s->streams.push_back(x);
    void* w = nullptr;
    e = cudaMalloc(&w, s->ws_bytes);
    if (e != cudaSuccess) break;
    s->ws.push_back(w);
    uint32_t* pb = nullptr;
    e = cudaMalloc(&pb, max_keys * 8);
    if (e != cudaSuccess) break;
    s->pair_buf.push_back(pb);
    s->busy_until.push_back(0.0);
  }
  if (e == cudaSuccess) e = cudaMalloc(&s->d_counts, sizeof(unsigned long long) * s->n_slots);
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_counts, sizeof(unsigned long long) * s->n_slots);
  for (int i = 0; i < STAGE_RING && e == cudaSuccess; i++) {
    void* h = nullptr;
    e = cudaMallocHost(&h, STAGE_BYTES);
    if (e != cudaSuccess) break;
    s->stage.push_back(h);
    cudaEvent_t ev = nullptr;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) break;
    s->stage_done.push_back(ev);
    s->stage_used.push_back(0);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->clock_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ref);
  if (e == cudaSuccess) e = rebase_clock(s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    hg_server_free(s);
    return cuda_fail(e, "hg_server_create");
  }
  *out = s;
  return HG_OK;
}

extern "C" hg_status hg_server_reserve(hg_server* s, size_t bytes) {
  if (!s) return HG_ERR_INVALID_ARGUMENT;
  bytes = std::min(bytes, s->budget);
  // 1 GiB blocks taken from the pool and handed back at once: the pool maps
  // them and, its release threshold being the budget, keeps them mapped.
  cudaStream_t st = s->streams[0];
  std::vector<void*> blocks;
  cudaError_t e = cudaSuccess;
  for (size_t done = 0; done < bytes;) {
    const size_t b = std::min(size_t(1) << 30, bytes - done);
    void* p = nullptr;
    e = cudaMallocFromPoolAsync(&p, b, s->pool, st);
    if (e != cudaSuccess) break;
    blocks.push_back(p);
    done += b;
  }
  if (e != cudaSuccess) cudaGetLastError();
  for (void* p : blocks) cudaFreeAsync(p, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "hg_server_reserve");
  return e2 == cudaSuccess ? HG_OK : cuda_fail(e2, "hg_server_reserve: sync");
}

extern "C" hg_status hg_server_build(hg_server* s, uint64_t table_id, const void* d_keys, uint64_t n,
                                     uint64_t n_buckets, int with_index, double arrival_s, uint64_t* ticket) {
  if (!s || !ticket || (n > 0 && !d_keys) || n_buckets == 0) return HG_ERR_INVALID_ARGUMENT;
  if (n > s->max_keys || n_buckets > s->max_keys)
    return lib_fail(HG_ERR_TOO_LARGE, "hg_server_build: more keys or buckets than the server's max_keys");
  *ticket = s->next_ticket++;
  const QueuedReq r{0, table_id, d_keys, n, n_buckets, with_index, nullptr, 0, arrival_s, *ticket};
  if (s->batching && n <= s->batch_small) return enqueue(s, r);
  if (queue_touches(s, table_id)) {  // a queued request on this table goes first
    hg_status qs = flush_queue(s);
    if (qs != HG_OK) return qs;
  }
  std::vector<uint64_t> pinned;  // tables queued intersects will read
  for (const QueuedReq& q : s->queue) pinned.push_back(q.table_id);
  return direct_build(s, r, &pinned);
}

extern "C" hg_status hg_server_intersect(hg_server* s, uint64_t table_id, const void* d_query, uint64_t nq,
                                         uint32_t* d_pairs, uint64_t pair_cap, double arrival_s, uint64_t* ticket) {
  if (!s || !ticket || (nq > 0 && !d_query)) return HG_ERR_INVALID_ARGUMENT;
  if (nq > s->max_keys) return lib_fail(HG_ERR_TOO_LARGE, "hg_server_intersect: more queries than max_keys");
  *ticket = s->next_ticket++;
  const QueuedReq r{1, table_id, d_query, nq, 0, 0, d_pairs, pair_cap, arrival_s, *ticket};
  if (s->batching && nq <= s->batch_small) return enqueue(s, r);
  if (queue_touches(s, table_id)) {  // a queued build of this table goes first
    hg_status qs = flush_queue(s);
    if (qs != HG_OK) return qs;
  }
  return direct_intersect(s, r);
}

extern "C" hg_status hg_server_submit(hg_server* s, const hg_server_request* reqs, int n, uint64_t* tickets,
                                      int* n_done) {
  if (!s || n < 0 || (n > 0 && (!reqs || !tickets)) || !n_done) return HG_ERR_INVALID_ARGUMENT;
  *n_done = 0;
  for (int i = 0; i < n; i++) {
    const hg_server_request& r = reqs[i];
    hg_status st;
    if (r.kind == 0)
      st = hg_server_build(s, r.table_id, r.d_data, r.n, r.n_buckets, r.with_index, r.arrival_s, tickets + i);
    else if (r.kind == 1)
      st = hg_server_intersect(s, r.table_id, r.d_data, r.n, r.d_pairs, r.pair_cap, r.arrival_s, tickets + i);
    else
      st = lib_fail(HG_ERR_INVALID_ARGUMENT, "hg_server_submit: kind is neither 0 (build) nor 1 (intersect)");
    if (st != HG_OK) return st;
    *n_done = i + 1;
  }
  return HG_OK;
}

extern "C" hg_status hg_server_poll(hg_server* s, int block, hg_server_done* out, int max_out, int* n_out) {
  if (!s || !n_out || (max_out > 0 && !out)) return HG_ERR_INVALID_ARGUMENT;
  *n_out = 0;
  if (!s->queue.empty() && (block || monotonic_s() - s->queued_since >= s->batch_wait)) {
    hg_status qs = flush_queue(s);
    if (qs != HG_OK) return qs;
  }
  if (block && !s->inflight.empty() && max_out > 0) {
    const cudaError_t e = cudaEventSynchronize(s->inflight.front().done);
    if (e != cudaSuccess) return cuda_fail(e, "hg_server_poll: wait");
  }
  for (auto it = s->inflight.begin(); it != s->inflight.end() && *n_out < max_out;) {
    const cudaError_t q = cudaEventQuery(it->done);
    if (q == cudaErrorNotReady) {
      ++it;
      continue;
    }
    if (q != cudaSuccess) return cuda_fail(q, "hg_server_poll: query");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s->ref, it->done);
    hg_server_done& d = out[(*n_out)++];
    d.ticket = it->ticket;
    d.kind = it->kind;
    d.missed = it->missed;
    d.count = it->kind == 1 && !it->missed ? s->h_counts[it->slot] : 0ull;
    d.latency_s = std::max(0.0, s->ref_host + 1e-3 * double(ms) - it->arrival);
    if (it->kind == 1) s->slot_busy[it->slot] = 0;
    auto ref = s->event_refs.find(it->done);
    if (ref == s->event_refs.end() || --ref->second == 0) {  // the last request on its event
      if (ref != s->event_refs.end()) s->event_refs.erase(ref);
      s->free_events.push_back(it->done);
    }
    it = s->inflight.erase(it);
  }
  // re-based only when every completed request has been reported against the
  // old `ref` (the loop did not stop at max_out)
  if (*n_out < max_out && monotonic_s() - s->ref_host > REF_MAX_AGE_S) {
    const cudaError_t e = rebase_clock(s);
    if (e != cudaSuccess) return cuda_fail(e, "hg_server_poll: clock");
  }
  return HG_OK;
}

extern "C" hg_status hg_server_stats(const hg_server* s, uint64_t* resident_tables, size_t* resident_bytes,
                                     uint64_t* evictions, uint64_t* inflight) {
  if (!s) return HG_ERR_INVALID_ARGUMENT;
  if (resident_tables) *resident_tables = s->tables.size();
  if (resident_bytes) *resident_bytes = s->bytes;
  if (evictions) *evictions = s->evictions;
  if (inflight) *inflight = s->inflight.size() + s->queue.size();
  return HG_OK;
}

extern "C" hg_status hg_server_set_batching(hg_server* s, int enabled, uint64_t small_max, uint32_t max_queued,
                                            double max_wait_s) {
  if (!s || max_queued == 0 || max_wait_s < 0) return HG_ERR_INVALID_ARGUMENT;
  if (!s->queue.empty()) {
    hg_status st = flush_queue(s);
    if (st != HG_OK) return st;
  }
  s->batching = enabled != 0;
  s->batch_small = small_max;
  s->batch_max = max_queued;
  s->batch_wait = max_wait_s;
  return HG_OK;
}

extern "C" hg_status hg_server_batch_stats(const hg_server* s, uint64_t* batches, uint64_t* batched_requests) {
  if (!s) return HG_ERR_INVALID_ARGUMENT;
  if (batches) *batches = s->batches;
  if (batched_requests) *batched_requests = s->batched_requests;
  return HG_OK;
}
