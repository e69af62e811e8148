"""Serving loop over the native serving engine (hg_server_* of the C ABI).

The engine keeps resident tables under a device-memory budget and a table
limit (least recently used out first), spreads build and intersect requests
over a pool of CUDA streams, orders an intersect after its table's build, and
measures each request's latency from its arrival stamp to the device
completion of its last operation.  This module adds the request objects, an
open-loop driver (requests are submitted at their arrival times whatever the
completions) and latency percentiles.

The reference has no serving component (its tables are built and
intersected once per process, test/MultiHashGraphTest.cu:288-338).
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

from . import _ptr, check, lib
from ._capi import ServerDone, ServerRequest


@dataclass
class Request:
    kind: str                      # "build" or "intersect"
    table_id: int
    arrival: float                 # seconds on hg_server_now()'s clock (CLOCK_MONOTONIC)
    keys: object = None            # build: device key tensor (valid until completion)
    n_buckets: int = 0
    with_index: bool = False
    queries: object = None         # intersect: device query tensor
    pair_cap: int = 0
    pairs: object = None           # intersect: optional int32 [pair_cap, 2] device tensor for the pairs
    # filled when the request completes
    count: int | None = None
    latency_s: float | None = None
    missed: bool = False           # intersect against a table no longer resident
    ticket: int = field(default=0, repr=False)


def now() -> float:
    """The clock arrival stamps use (the engine's CLOCK_MONOTONIC seconds)."""
    return float(lib().hg_server_now())


class Server:
    """A native serving engine on the current device: `budget_bytes` of
    resident tables at most, `max_tables` tables at most, `n_streams` CUDA
    streams, tables of up to `max_keys` keys and buckets.  With `batching`,
    requests of at most `batch_small` keys are coalesced into batched launches
    (continuous batching: at most `batch_max` per launch, none waiting longer
    than `batch_wait_s` once the caller polls)."""

    def __init__(self, budget_bytes: int, max_tables: int = 512, n_streams: int = 4, max_keys: int = 1 << 24,
                 key_bytes: int = 8, device=None, batching: bool = True, batch_small: int = 1 << 16,
                 batch_max: int = 256, batch_wait_s: float = 100e-6):
        import torch
        if device is not None:
            torch.cuda.set_device(torch.device(device))
        self.key_bytes = key_bytes
        self._h = ctypes.c_void_p()
        check(lib().hg_server_create(int(budget_bytes), int(max_tables), int(n_streams), int(max_keys), key_bytes,
                                     ctypes.byref(self._h)), "hg_server_create")
        check(lib().hg_server_set_batching(self._h, int(batching), int(batch_small), int(batch_max),
                                           float(batch_wait_s)), "hg_server_set_batching")
        self._pending: dict[int, Request] = {}
        self._done = (ServerDone * 1024)()

    def reserve(self, nbytes: int) -> None:
        """Maps `nbytes` (at most the budget) into the table pool up front."""
        check(lib().hg_server_reserve(self._h, int(nbytes)), "hg_server_reserve")

    def submit(self, r: Request) -> None:
        L = lib()
        t = ctypes.c_uint64(0)
        if r.kind == "build":
            check(L.hg_server_build(self._h, r.table_id, _ptr(r.keys), r.keys.numel(), r.n_buckets, int(r.with_index),
                                    r.arrival, ctypes.byref(t)), "hg_server_build")
        else:
            pairs = _ptr(r.pairs) if r.pairs is not None else None
            cap = min(r.pair_cap, r.pairs.shape[0]) if r.pairs is not None else r.pair_cap
            check(L.hg_server_intersect(self._h, r.table_id, _ptr(r.queries), r.queries.numel(), pairs, cap,
                                        r.arrival, ctypes.byref(t)), "hg_server_intersect")
        r.ticket = t.value
        self._pending[r.ticket] = r

    def submit_many(self, reqs: list[Request]) -> None:
        """Submits the requests in order with one call into the engine
        (hg_server_submit): the same as submit() on each, without the host's
        per-call cost."""
        if not reqs:
            return
        arr = (ServerRequest * len(reqs))()
        for a, r in zip(arr, reqs):
            a.arrival_s = r.arrival
            a.table_id = r.table_id
            if r.kind == "build":
                a.kind, a.with_index, a.d_data, a.n = 0, int(r.with_index), r.keys.data_ptr(), r.keys.numel()
                a.n_buckets = r.n_buckets
            else:
                a.kind, a.d_data, a.n = 1, r.queries.data_ptr(), r.queries.numel()
                if r.pairs is not None:
                    a.d_pairs = r.pairs.data_ptr()
                    a.pair_cap = min(r.pair_cap, r.pairs.shape[0])
                else:
                    a.pair_cap = r.pair_cap
        tickets = (ctypes.c_uint64 * len(reqs))()
        done = ctypes.c_int(0)
        st = lib().hg_server_submit(self._h, arr, len(reqs), tickets, ctypes.byref(done))
        for i in range(done.value):
            reqs[i].ticket = tickets[i]
            self._pending[tickets[i]] = reqs[i]
        check(st, "hg_server_submit")

    def poll(self, block: bool = False) -> list[Request]:
        """Completed requests (block: wait until at least the oldest one is)."""
        out = []
        n = ctypes.c_int(0)
        while True:
            check(lib().hg_server_poll(self._h, int(block and not out), self._done, len(self._done), ctypes.byref(n)),
                  "hg_server_poll")
            for i in range(n.value):
                d = self._done[i]
                r = self._pending.pop(d.ticket)
                r.latency_s = d.latency_s
                r.missed = bool(d.missed)
                if d.kind == 1:
                    r.count = int(d.count)
                out.append(r)
            if n.value < len(self._done):
                return out

    def drain(self) -> list[Request]:
        out = []
        while self._pending:
            out += self.poll(block=True)
        return out

    def stats(self) -> dict:
        t, e, f = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_uint64(0)
        b = ctypes.c_size_t(0)
        check(lib().hg_server_stats(self._h, ctypes.byref(t), ctypes.byref(b), ctypes.byref(e), ctypes.byref(f)),
              "hg_server_stats")
        nb, nr = ctypes.c_uint64(0), ctypes.c_uint64(0)
        check(lib().hg_server_batch_stats(self._h, ctypes.byref(nb), ctypes.byref(nr)), "hg_server_batch_stats")
        return {"resident_tables": t.value, "resident_bytes": b.value, "evictions": e.value, "inflight": f.value,
                "batches": nb.value, "batched_requests": nr.value}

    def free(self) -> None:
        if self._h:
            lib().hg_server_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def run_open_loop(server, requests: list[Request], clock=now, sleep=time.sleep) -> float:
    """Submits every request at its arrival time (open loop: arrivals do not
    wait for completions), collects completions meanwhile, and returns the
    makespan in seconds.  Arrival times are taken relative to the first
    request and re-stamped on `clock`."""
    if not requests:
        return 0.0
    t0 = clock()
    base = requests[0].arrival
    for r in requests:
        r.arrival = t0 + (r.arrival - base)
    k = 0
    while k < len(requests):
        t = clock()
        while k < len(requests) and requests[k].arrival <= t:
            server.submit(requests[k])
            k += 1
        server.poll()
        if k < len(requests):
            wait = requests[k].arrival - clock()
            if wait > 0:
                sleep(min(wait, 0.0005))
    server.drain()
    return clock() - t0


def latency_summary(requests: list[Request]) -> dict:
    import statistics
    lat = sorted(r.latency_s for r in requests if r.latency_s is not None)
    if not lat:
        return {}

    def pct(p):
        return lat[min(len(lat) - 1, int(p * len(lat)))] * 1e3

    return {"p50_ms": pct(0.50), "p99_ms": pct(0.99), "mean_ms": statistics.fmean(lat) * 1e3,
            "max_ms": lat[-1] * 1e3}
