"""The native serving engine on the GPU: concurrent requests on several
streams give the same intersect counts as a serial run, the byte budget and
the table limit hold (evictions happen), a request against an evicted table
is reported as missed, and every request gets a latency."""
import pytest

pytestmark = pytest.mark.gpu


def test_served_counts_equal_serial(hg):
    import torch
    from hashgraph_b200.serve import Request, Server, run_open_loop
    import bench
    arena_keys = 1 << 20
    arena = hg.gen_uniform(arena_keys, 8, 9)
    torch.cuda.synchronize()
    specs = bench.serving_requests(200, 20000.0, arena_keys, lo_log2=6, hi_log2=15, seed=11)

    def make(sp):
        kind, tid, t, off, size = sp
        sl = arena[off:off + size]
        if kind == "build":
            return Request("build", tid, t, keys=sl, n_buckets=size)
        return Request("intersect", tid, t, queries=sl, pair_cap=size)

    # a budget of ~8 average tables forces evictions (and some misses)
    server = Server(budget_bytes=8 << 20, max_tables=24, n_streams=4, max_keys=1 << 15)
    server.reserve(1 << 30)  # capped at the budget
    reqs = [make(sp) for sp in specs]
    run_open_loop(server, reqs)
    assert all(r.latency_s is not None and r.latency_s >= 0 for r in reqs)
    st = server.stats()
    assert st["evictions"] > 0 and st["resident_tables"] <= 24 and st["resident_bytes"] <= 8 << 20
    assert st["inflight"] == 0
    serial = Server(budget_bytes=1 << 40, max_tables=1 << 20, n_streams=1, max_keys=1 << 15)
    checked = 0
    for sp, r in zip(specs, reqs):
        q = make(sp)
        serial.submit(q)
        serial.drain()
        if q.kind == "intersect" and not r.missed:
            assert q.count == r.count
            checked += 1
    assert checked > 50
    assert hg.device_error() == 0


def test_missed_and_replaced_tables(hg):
    import torch
    from hashgraph_b200.serve import Request, Server, now
    import oracle
    from tests.conftest import from_np_u
    a = oracle.gen_uniform(5000, 8, 1)
    b = oracle.gen_uniform(5000, 8, 2)
    da, db = from_np_u(a), from_np_u(b)
    torch.cuda.synchronize()
    srv = Server(budget_bytes=1 << 30, max_tables=1, n_streams=2, max_keys=1 << 14)
    srv.submit(Request("build", 1, now(), keys=da, n_buckets=4096))
    srv.submit(Request("intersect", 1, now(), queries=da, pair_cap=5000))
    srv.submit(Request("build", 2, now(), keys=db, n_buckets=4096))   # evicts table 1
    r_miss = Request("intersect", 1, now(), queries=da, pair_cap=5000)
    r_hit = Request("intersect", 2, now(), queries=db, pair_cap=5000)
    srv.submit(r_miss)
    srv.submit(r_hit)
    done = srv.drain()
    assert len(done) == 5
    assert r_miss.missed and r_miss.count == 0
    assert not r_hit.missed and r_hit.count == 5000
    srv.submit(Request("build", 2, now(), keys=da, n_buckets=1000))    # replaced
    r2 = Request("intersect", 2, now(), queries=db, pair_cap=5000)
    srv.submit(r2)
    srv.drain()
    assert r2.count == oracle.join_count(a, b)
    assert srv.stats()["resident_tables"] == 1
    srv.free()
