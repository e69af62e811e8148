"""Serving loop: resident tables, a device-memory budget with LRU eviction,
and build / intersect requests executed concurrently on a pool of CUDA
streams, with per-request latency.

The reference has no serving component (its tables are built and
intersected once per process, test/MultiHashGraphTest.cu:288-338).  This is
the host-side scheduler around the C ABI; all device work goes through the
library's kernels.

A request's latency is measured from its arrival time to the completion of
its last kernel on the device: the end event's time is mapped onto the host
clock through one reference event recorded when the server starts.
"""
from __future__ import annotations

import collections
import ctypes
import time
from dataclasses import dataclass, field

from . import Table, _ptr, _stream, check, lib


@dataclass
class Request:
    kind: str                      # "build" or "intersect"
    table_id: int
    arrival: float                 # host seconds (time.perf_counter) when the request arrives
    keys: object = None            # build: device key tensor
    n_buckets: int = 0
    with_index: bool = False
    queries: object = None         # intersect: device query tensor
    pair_cap: int = 0
    # filled by the server
    count: int | None = None
    latency_s: float | None = None
    missed: bool = False           # intersect against a table no longer resident
    _end: object = field(default=None, repr=False)
    _count_dev: object = field(default=None, repr=False)
    _stream_i: int = field(default=-1, repr=False)


class TableStore:
    """Resident tables keyed by id, least recently used first out, within a
    device-byte budget and a table-count limit."""

    def __init__(self, budget_bytes: int, max_tables: int):
        self.budget = int(budget_bytes)
        self.max_tables = int(max_tables)
        self.tables: collections.OrderedDict[int, Table] = collections.OrderedDict()
        self.bytes = 0
        self.evictions = 0

    @staticmethod
    def table_bytes(t: Table) -> int:
        b = t.offsets.numel() * 4 + t.keys.numel() * t.keys.element_size()
        if t.idx is not None:
            b += t.idx.numel() * 4
        return b

    def get(self, table_id: int) -> Table | None:
        t = self.tables.get(table_id)
        if t is not None:
            self.tables.move_to_end(table_id)
        return t

    def make_room(self, need_bytes: int, keep: int | None = None) -> None:
        while self.tables and (self.bytes + need_bytes > self.budget or len(self.tables) >= self.max_tables):
            victim = next(iter(self.tables))
            if victim == keep:
                break
            t = self.tables.pop(victim)
            self.bytes -= self.table_bytes(t)
            self.evictions += 1

    def put(self, table_id: int, t: Table) -> None:
        old = self.tables.pop(table_id, None)
        if old is not None:
            self.bytes -= self.table_bytes(old)
        self.tables[table_id] = t
        self.bytes += self.table_bytes(t)


class Server:
    """Runs requests on `n_streams` CUDA streams.  Each stream owns a build /
    intersect workspace and a pair buffer sized for `max_keys`."""

    def __init__(self, budget_bytes: int, max_tables: int = 512, n_streams: int = 4, max_keys: int = 1 << 24,
                 key_bytes: int = 8, device=None):
        import torch
        self.torch = torch
        self.device = torch.device(device or "cuda")
        self.store = TableStore(budget_bytes, max_tables)
        self.key_bytes = key_bytes
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(n_streams)]
        L = lib()
        wb, wq = ctypes.c_size_t(0), ctypes.c_size_t(0)
        check(L.hg_build_workspace_size(max_keys, key_bytes, max_keys, 1, ctypes.byref(wb)), "workspace")
        check(L.hg_intersect_workspace_size(max_keys, 1, max_keys, max_keys, key_bytes, 1, ctypes.byref(wq)),
              "workspace")
        ws = max(wb.value, wq.value, 1)
        self.ws = [torch.empty(ws, dtype=torch.uint8, device=self.device) for _ in self.streams]
        self.pairs = [torch.empty((max_keys, 2), dtype=torch.int32, device=self.device) for _ in self.streams]
        self.busy_until = [0.0] * n_streams     # host estimate of each stream's queued work
        self.inflight: list[Request] = []
        torch.cuda.synchronize(self.device)
        self.ref_event = torch.cuda.Event(enable_timing=True)
        self.ref_event.record(torch.cuda.current_stream(self.device))
        self.ref_event.synchronize()
        self.ref_host = time.perf_counter()

    def _pick_stream(self, now: float) -> int:
        return min(range(len(self.streams)), key=lambda i: max(self.busy_until[i], now))

    def submit(self, r: Request, est_s: float = 0.0) -> None:
        torch = self.torch
        now = time.perf_counter()
        i = self._pick_stream(now)
        self.busy_until[i] = max(self.busy_until[i], now) + est_s
        s = self.streams[i]
        r._stream_i = i
        L = lib()
        with torch.cuda.stream(s):
            if r.kind == "build":
                n = r.keys.numel()
                self.store.make_room((r.n_buckets + 1) * 4 + n * (self.key_bytes + (4 if r.with_index else 0)),
                                     keep=None)
                t = Table(r.n_buckets, self.key_bytes, r.with_index, n, self.device, workspace=False)
                check(L.hg_build_into(_ptr(r.keys), n, self.key_bytes, r.n_buckets, _ptr(t.offsets), _ptr(t.keys),
                                      _ptr(t.idx), _ptr(self.ws[i]), self.ws[i].numel(), _stream(s)),
                      "serve build")
                t.n = n
                # intersects on other streams wait for the build to finish
                t.ready = torch.cuda.Event()
                t.ready.record(s)
                self.store.put(r.table_id, t)
            else:
                t = self.store.get(r.table_id)
                r._count_dev = torch.zeros(1, dtype=torch.int64, device=self.device)
                if t is None:
                    r.missed = True
                else:
                    s.wait_event(t.ready)
                    # the table's memory is not reused while this stream reads it,
                    # even if the table is evicted or replaced meanwhile
                    for a in (t.offsets, t.keys, t.idx):
                        if a is not None:
                            a.record_stream(s)
                    nq = r.queries.numel()
                    check(L.hg_intersect_into(_ptr(t.offsets), _ptr(t.keys), _ptr(t.idx), t.n, t.n_buckets,
                                              self.key_bytes, _ptr(r.queries), nq, None, _ptr(self.pairs[i]),
                                              min(r.pair_cap, self.pairs[i].shape[0]), _ptr(r._count_dev),
                                              _ptr(self.ws[i]), self.ws[i].numel(), _stream(s)),
                          "serve intersect")
            r._end = torch.cuda.Event(enable_timing=True)
            r._end.record(s)
        self.inflight.append(r)

    def poll(self, block: bool = False) -> list[Request]:
        done, rest = [], []
        for r in self.inflight:
            if block:
                r._end.synchronize()
            if block or r._end.query():
                gpu_t = self.ref_host + self.ref_event.elapsed_time(r._end) * 1e-3
                r.latency_s = max(gpu_t - r.arrival, 0.0)
                if r.kind == "intersect":
                    r.count = int(r._count_dev.item())
                done.append(r)
            else:
                rest.append(r)
        self.inflight = rest
        return done


def run_open_loop(server: Server, requests: list[Request], est=lambda r: 0.0) -> float:
    """Submits every request at its arrival time (open loop; arrivals do not
    wait for completions) and returns the makespan in seconds."""
    t0 = time.perf_counter()
    base = requests[0].arrival if requests else 0.0
    for r in requests:
        r.arrival = t0 + (r.arrival - base)
    k = 0
    while k < len(requests):
        now = time.perf_counter()
        while k < len(requests) and requests[k].arrival <= now:
            server.submit(requests[k], est(requests[k]))
            k += 1
        server.poll()
        if k < len(requests):
            wait = requests[k].arrival - time.perf_counter()
            if wait > 0:
                time.sleep(min(wait, 0.0005))
    server.poll(block=True)
    return time.perf_counter() - t0


def latency_summary(requests: list[Request]) -> dict:
    import statistics
    lat = sorted(r.latency_s for r in requests if r.latency_s is not None)
    if not lat:
        return {}

    def pct(p):
        return lat[min(len(lat) - 1, int(p * len(lat)))] * 1e3

    return {"p50_ms": pct(0.50), "p99_ms": pct(0.99), "mean_ms": statistics.fmean(lat) * 1e3,
            "max_ms": lat[-1] * 1e3}
