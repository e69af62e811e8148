"""The serving loop on the GPU: concurrent requests on several streams give
the same intersect counts as a serial run, evictions happen under a small
budget, and every request gets a latency."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_counts_equal_serial(hg):
    import torch
    from hashgraph_b200.serve import Request, Server, run_open_loop
    import bench
    arena_keys = 1 << 20
    arena = hg.gen_uniform(arena_keys, 8, 9)
    specs = bench.serving_requests(200, 20000.0, arena_keys, lo_log2=6, hi_log2=15, seed=11)

    def make(sp):
        kind, tid, t, off, size = sp
        sl = arena[off:off + size]
        if kind == "build":
            return Request("build", tid, t, keys=sl, n_buckets=size)
        return Request("intersect", tid, t, queries=sl, pair_cap=size)

    # a budget of ~8 average tables forces evictions (and some misses)
    server = Server(budget_bytes=8 << 20, max_tables=24, n_streams=4, max_keys=1 << 15)
    reqs = [make(sp) for sp in specs]
    run_open_loop(server, reqs)
    assert all(r.latency_s is not None and r.latency_s >= 0 for r in reqs)
    assert server.store.evictions > 0
    assert len(server.store.tables) <= 24
    serial = Server(budget_bytes=1 << 40, max_tables=1 << 20, n_streams=1, max_keys=1 << 15)
    checked = 0
    for sp, r in zip(specs, reqs):
        q = make(sp)
        serial.submit(q)
        serial.poll(block=True)
        if q.kind == "intersect" and not r.missed:
            assert q.count == r.count
            checked += 1
    assert checked > 50
    assert hg.device_error() == 0
