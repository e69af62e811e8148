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


def _served_specs(n_req, seed):
    """Builds of table ids 0..15 (ids reused, so tables get replaced) and
    intersects against them, sizes 2^U(6,14); slices of one key arena."""
    import numpy as np
    rng = np.random.default_rng(seed)
    specs, built = [], {}
    for k in range(n_req):
        size = int(2 ** rng.uniform(6, 14))
        if k < 8 or rng.uniform() < 0.35:
            tid = int(rng.integers(0, 16))
            off = int(rng.integers(0, (1 << 20) - size))
            built[tid] = (off, size)
            specs.append(("build", tid, off, size))
        else:
            tid = int(rng.choice(sorted(built)))
            toff, tn = built[tid]
            off = min(toff + tn // 2, (1 << 20) - size)
            specs.append(("intersect", tid, off, size))
    return specs


def test_submit_many_equals_submit(hg):
    """hg_server_submit (one call for a burst) serves the same requests as
    one hg_server_build / hg_server_intersect call each: identical counts
    and pairs, the same misses."""
    import numpy as np
    import torch

    import oracle
    from hashgraph_b200.serve import Request, Server, now
    from tests.conftest import to_np_u
    arena_h = oracle.gen_uniform(1 << 20, 8, 41)
    arena = torch.from_numpy(arena_h.view(np.int64)).cuda()
    specs = _served_specs(200, 43)

    def make(sp):
        kind, tid, off, size = sp
        sl = arena[off:off + size]
        if kind == "build":
            return Request("build", tid, now(), keys=sl, n_buckets=size, with_index=True)
        return Request("intersect", tid, now(), queries=sl, pair_cap=size,
                       pairs=torch.full((size, 2), -1, dtype=torch.int32, device="cuda"))

    torch.cuda.synchronize()
    results = []
    for many in (False, True):
        srv = Server(budget_bytes=1 << 30, max_tables=64, n_streams=4, max_keys=1 << 15)
        reqs = [make(sp) for sp in specs]
        if many:
            srv.submit_many(reqs)
        else:
            for r in reqs:
                srv.submit(r)
        srv.drain()
        out = []
        for r in reqs:
            if r.kind == "intersect":
                p = to_np_u(r.pairs[:r.count], 4).astype(np.uint64)
                out.append((r.count, r.missed, np.sort(p[:, 0] << 32 | p[:, 1]).tobytes()))
        results.append(out)
        srv.free()
    assert results[0] == results[1] and len(results[0]) > 50
    assert hg.device_error() == 0


def test_served_pairs_equal_oracle_and_alone(hg):
    """Saturated load: every request submitted at once, so the engine
    coalesces them into batched launches (continuous batching).  Each served
    intersect's count and sorted (index, query) pairs equal the oracle's on
    the table resident when the request was submitted, and the same request
    served alone (no batching, one request at a time) gives the same pairs."""
    import numpy as np
    import torch

    import oracle
    from hashgraph_b200.serve import Request, Server, now
    from tests.conftest import to_np_u
    arena_h = oracle.gen_uniform(1 << 20, 8, 19)
    arena = torch.from_numpy(arena_h.view(np.int64)).cuda()
    specs = _served_specs(300, 23)

    def make(sp, t):
        kind, tid, off, size = sp
        sl = arena[off:off + size]
        if kind == "build":
            return Request("build", tid, t, keys=sl, n_buckets=size, with_index=True)
        return Request("intersect", tid, t, queries=sl, pair_cap=size,
                       pairs=torch.full((size, 2), -1, dtype=torch.int32, device="cuda"))

    torch.cuda.synchronize()
    server = Server(budget_bytes=1 << 30, max_tables=64, n_streams=4, max_keys=1 << 15, batch_max=64)
    t0 = now()
    reqs = [make(sp, t0) for sp in specs]
    for r in reqs:
        server.submit(r)
    server.drain()
    st = server.stats()
    # requests came through batched launches (segments of fewer than four
    # requests, cut where a build follows an intersect, go one by one)
    assert st["batches"] >= 4 and st["batched_requests"] >= len(specs) // 2
    alone = Server(budget_bytes=1 << 30, max_tables=64, n_streams=1, max_keys=1 << 15, batching=False)
    tables = {}
    checked = 0
    for sp, r in zip(specs, reqs):
        kind, tid, off, size = sp
        q = make(sp, now())
        alone.submit(q)
        alone.drain()
        if kind == "build":
            tables[tid] = oracle.build(arena_h[off:off + size], size, True)
            continue
        o_off, o_keys, o_idx = tables[tid]
        oc, op = oracle.intersect(o_off, o_keys, o_idx, arena_h[off:off + size], pair_cap=size)
        assert not r.missed and r.count == oc == q.count
        got = to_np_u(r.pairs[:oc], 4).astype(np.uint64)
        solo = to_np_u(q.pairs[:oc], 4).astype(np.uint64)
        exp = op.astype(np.uint64)
        key = lambda p: np.sort(p[:, 0] << 32 | p[:, 1])  # noqa: E731
        np.testing.assert_array_equal(key(got), key(exp))
        np.testing.assert_array_equal(key(solo), key(exp))
        checked += 1
    assert checked > 100
    server.free()
    alone.free()
    assert hg.device_error() == 0
