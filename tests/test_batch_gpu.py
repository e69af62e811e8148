"""GPU parity of the batched build + intersect (hg_batch_*) against the oracle
and against one plain call per pair, and its replay from a captured CUDA graph.

Each pair's result must equal the single-pair path's: offsets bit-exact,
canonical buckets equal, the exact match count, and the same pairs (in the
same query order for pairs the batch runs in the direct form; a_ref compared
through the key it names when the table has no index, since positions inside
a bucket are in atomic order)."""
import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u, to_np_u

pytestmark = pytest.mark.gpu


def _sorted_pairs(p):
    p = np.asarray(p, dtype=np.uint32).reshape(-1, 2).astype(np.uint64)
    return np.sort(p[:, 0] << np.uint64(32) | p[:, 1])


def _make_batch_inputs(kb, n_pairs, seed, max_log2=13, dups=True):
    rng = np.random.default_rng(seed)
    keys, queries, buckets, with_index = [], [], [], []
    for i in range(n_pairs):
        n = 0 if i % 11 == 3 else int(2 ** rng.uniform(0, max_log2))
        nq = 0 if i % 13 == 5 else int(2 ** rng.uniform(0, max_log2))
        a = oracle.gen_uniform(n, kb, 1000 + i)
        if dups and i % 7 == 2 and n:  # duplicates: the multiset join multiplies
            a = (a % a.dtype.type(max(n // 4, 1))).astype(a.dtype)
        q = oracle.gen_overlap(nq, a, float(rng.uniform(0, 1)), 5000 + i) if n else oracle.gen_uniform(nq, kb, 5000 + i)
        B = 1 if i % 17 == 1 else max(1, n if i % 2 else int(rng.integers(1, 3 * max(n, 1) + 1)))
        keys.append(a)
        queries.append(q)
        buckets.append(B)
        with_index.append(bool(i % 3))
    return keys, queries, buckets, with_index


def _oracle_pair(a, q, B, wi):
    off, k, idx = oracle.build(a, B, True)
    c, _ = oracle.intersect(off, k, idx, q, pair_cap=0)
    c, pairs = oracle.intersect(off, k, idx, q, pair_cap=max(c, 1))
    return off, k, idx, c, pairs


def _check_pair(hg, batch, i, a, q, B, wi, kb):
    off, k, idx, c, op = _oracle_pair(a, q, B, wi)
    g_off = to_np_u(batch.offsets[i], 4)
    np.testing.assert_array_equal(g_off, off)
    n = a.size
    g_keys = to_np_u(batch.table_keys[i][:n], kb)
    g_idx = to_np_u(batch.table_idx[i][:n], 4) if wi else None
    ck, ci = oracle.canonicalize(off, g_keys.copy(), None if g_idx is None else g_idx.copy())
    rk, ri = oracle.canonicalize(off, k.copy(), idx.copy() if wi else None)
    np.testing.assert_array_equal(ck, rk)
    if wi:
        np.testing.assert_array_equal(ci, ri)
    gc = int(batch.counts[i].item())
    assert gc == c, (i, gc, c)
    cap = batch.pairs[i].shape[0]
    if c and c <= cap:
        gp = to_np_u(batch.pairs[i][:c], 4)
        if wi:
            np.testing.assert_array_equal(_sorted_pairs(gp), _sorted_pairs(op))
        else:  # a_ref is a CSR position: compare the keys it names
            assert np.all(g_keys[gp[:, 0]] == q[gp[:, 1]])
            np.testing.assert_array_equal(np.sort(gp[:, 1]), np.sort(op[:, 1]))


@pytest.mark.parametrize("kb", [4, 8])
def test_batch_matches_oracle(hg, kb):
    keys, queries, buckets, wi = _make_batch_inputs(kb, 60, 7 + kb)
    caps = [max(_oracle_pair(keys[i], queries[i], buckets[i], wi[i])[3], 1) for i in range(len(keys))]
    b = hg.Batch([from_np_u(a) for a in keys], [from_np_u(q) for q in queries], buckets, wi, caps).run()
    import torch
    torch.cuda.synchronize()
    assert hg.device_error() == 0
    for i in range(len(keys)):
        _check_pair(hg, b, i, keys[i], queries[i], buckets[i], wi[i], kb)
    b.free()


def test_batch_partitioned_matches_oracle(hg):
    """Pairs of 2^14 .. 2^17 keys take the partitioned form (pass 1 straight
    into fine partitions, then the fine build and fine probe); one with heavy
    duplicates overflows its partitions and is redone by the direct kernels."""
    import torch
    rng = np.random.default_rng(77)
    keys, queries, buckets, wi = [], [], [], []
    for i in range(12):
        n = int(2 ** rng.uniform(14, 17))
        nq = int(2 ** rng.uniform(14, 17)) if i % 5 else 100  # a small query set stays direct
        a = oracle.gen_uniform(n, 8, 300 + i)
        if i == 4:  # all copies of a few keys: the partitions overflow
            a = (a % np.uint64(37)).astype(np.uint64)
        q = oracle.gen_overlap(nq, a, float(rng.uniform(0.1, 0.9)), 400 + i)
        keys.append(a)
        queries.append(q)
        buckets.append(n if i % 3 else int(rng.integers(n // 2, 2 * n)))
        wi.append(bool(i % 2))
    caps = [max(_oracle_pair(keys[i], queries[i], buckets[i], wi[i])[3], 1) for i in range(len(keys))]
    b = hg.Batch([from_np_u(a) for a in keys], [from_np_u(q) for q in queries], buckets, wi, caps).run()
    torch.cuda.synchronize()
    assert hg.device_error() == 0
    for i in range(len(keys)):
        _check_pair(hg, b, i, keys[i], queries[i], buckets[i], wi[i], 8)
    # a second run over the same buffers gives the same results
    b.run()
    torch.cuda.synchronize()
    for i in range(len(keys)):
        _check_pair(hg, b, i, keys[i], queries[i], buckets[i], wi[i], 8)


def test_batch_equals_plain_calls(hg):
    """Same offsets and, with an index, the same pairs as one direct-path
    build + intersect per pair: in the same order for the pairs the batch
    runs in the direct form, as the same set for the partitioned ones."""
    import torch
    kb = 8
    keys, queries, buckets, _ = _make_batch_inputs(kb, 24, 99, max_log2=16, dups=False)
    wi = [True] * len(keys)
    dk = [from_np_u(a) for a in keys]
    dq = [from_np_u(q) for q in queries]
    b = hg.Batch(dk, dq, buckets, wi).run()
    for i in range(len(keys)):
        t = hg.Table.build(dk[i], buckets[i], with_index=True, path=hg.PATH_DIRECT)
        count, pairs = t.intersect(dq[i], path=hg.PATH_DIRECT)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(to_np_u(b.offsets[i], 4), to_np_u(t.offsets, 4))
        c = int(count.item())
        assert int(b.counts[i].item()) == c
        if keys[i].size < (1 << 14) or queries[i].size < (1 << 14):
            np.testing.assert_array_equal(to_np_u(b.pairs[i][:c], 4), to_np_u(pairs[:c], 4))
        else:
            np.testing.assert_array_equal(_sorted_pairs(to_np_u(b.pairs[i][:c], 4)),
                                          _sorted_pairs(to_np_u(pairs[:c], 4)))
    assert hg.device_error() == 0


def test_batch_pair_capacity(hg):
    import torch
    a = oracle.gen_uniform(5000, 8, 3)
    q = oracle.gen_overlap(5000, a, 1.0, 4)
    b = hg.Batch([from_np_u(a)], [from_np_u(q)], [4096], [True], pair_caps=[100]).run()
    torch.cuda.synchronize()
    assert int(b.counts[0].item()) == 5000  # exact beyond the capacity
    assert hg.device_error() == hg.ERR_PAIR_CAPACITY
    assert hg.device_error() == 0  # read clears it
    off, k, idx, c, op = _oracle_pair(a, q, 4096, True)
    got = to_np_u(b.pairs[0][:100], 4)
    # the first 100 pairs in query order
    np.testing.assert_array_equal(np.sort(got[:, 1]), np.sort(op[:, 1])[:100])


def test_batch_count_only(hg):
    import torch
    keys, queries, buckets, wi = _make_batch_inputs(8, 16, 5)
    b = hg.Batch([from_np_u(a) for a in keys], [from_np_u(q) for q in queries], buckets, wi, emit=False).run()
    torch.cuda.synchronize()
    for i in range(len(keys)):
        off, k, idx, c, _ = _oracle_pair(keys[i], queries[i], buckets[i], wi[i])
        assert int(b.counts[i].item()) == c


def test_batch_empty_and_single(hg):
    import torch
    b = hg.Batch([], [], []).run()
    torch.cuda.synchronize()
    a = oracle.gen_uniform(1, 4, 1)
    b = hg.Batch([from_np_u(a)], [from_np_u(a)], [1], [True]).run()
    torch.cuda.synchronize()
    assert int(b.counts[0].item()) == 1
    assert to_np_u(b.pairs[0][:1], 4).tolist() == [[0, 0]]


def test_batch_graph_replay(hg):
    """hg_batch_run captured once into a CUDA graph; inputs refilled in place
    and the graph replayed give the new inputs' results."""
    import torch
    kb = 8
    keys, queries, buckets, wi = _make_batch_inputs(kb, 32, 21, max_log2=12, dups=False)
    dk = [from_np_u(a) for a in keys]
    dq = [from_np_u(q) for q in queries]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b = hg.Batch(dk, dq, buckets, wi)
        b.run(stream=s)  # warm-up outside the capture
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.run(stream=s)
    # new inputs of the same sizes, written into the same buffers
    keys2 = [oracle.gen_uniform(a.size, kb, 77_000 + i) for i, a in enumerate(keys)]
    queries2 = [oracle.gen_overlap(q.size, keys2[i], 0.5, 88_000 + i) if keys2[i].size else q
                for i, q in enumerate(queries)]
    for i in range(len(keys)):
        if keys2[i].size:
            dk[i].copy_(from_np_u(keys2[i]))
        if queries2[i].size:
            dq[i].copy_(from_np_u(queries2[i]))
    torch.cuda.synchronize()
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    assert hg.device_error() == 0
    for i in range(len(keys)):
        _check_pair(hg, b, i, keys2[i], queries2[i], buckets[i], wi[i], kb)
    del g


def test_batch_large_tables_partitioned_probe(hg):
    """Pairs whose table exceeds the L2 form's 24 MB budget (2^21 u64 keys with
    an index) take the partitioned probe; one of them has its queries drawn
    from a handful of keys, so its query partitions overflow and the gated
    direct probe redoes the partitioned probes.  Small pairs ride along in
    the direct form."""
    import torch
    rng = np.random.default_rng(5)
    keys, queries, buckets, wi = [], [], [], []
    for i, (n, nq, dup) in enumerate([((1 << 21) + 3, 1 << 21, False), (1 << 21, (1 << 21) - 7, True),
                                       (3000, 2000, False), (100, 5000, False)]):
        a = oracle.gen_uniform(n, 8, 700 + i)
        q = oracle.gen_overlap(nq, a, 0.5, 800 + i)
        if dup:  # every query one of 16 keys of A: a few query partitions hold them all
            q = a[rng.integers(0, 16, size=nq)]
        keys.append(a)
        queries.append(q)
        buckets.append(n)
        wi.append(True)
    caps = [max(_oracle_pair(keys[i], queries[i], buckets[i], wi[i])[3], 1) for i in range(len(keys))]
    b = hg.Batch([from_np_u(a) for a in keys], [from_np_u(q) for q in queries], buckets, wi, caps).run()
    torch.cuda.synchronize()
    assert hg.device_error() == 0
    for i in range(len(keys)):
        _check_pair(hg, b, i, keys[i], queries[i], buckets[i], wi[i], 8)


@pytest.mark.parametrize("params", [{"part_min": 1 << 10, "l2_table_bytes": 0},
                                    {"part_min": 1 << 12, "l2_table_bytes": 1 << 20},
                                    {"part_min": 1 << 20, "l2_table_bytes": 24 << 20}])
def test_batch_size_classes_match_oracle(hg, params):
    """Every choice of size-class boundaries gives the oracle's results: with
    part_min 2^10 and no L2 form, mid-sized pairs take the partitioned probe;
    with a 1 MB L2 budget some take the L2 form and some the partitioned one;
    with part_min 2^20 everything is direct."""
    import torch
    keys, queries, buckets, wi = _make_batch_inputs(8, 40, 31, max_log2=16)
    caps = [max(_oracle_pair(keys[i], queries[i], buckets[i], wi[i])[3], 1) for i in range(len(keys))]
    b = hg.Batch([from_np_u(a) for a in keys], [from_np_u(q) for q in queries], buckets, wi, caps,
                 params=params).run()
    torch.cuda.synchronize()
    assert hg.device_error() == 0
    for i in range(len(keys)):
        _check_pair(hg, b, i, keys[i], queries[i], buckets[i], wi[i], 8)


def test_batch_autotune(hg):
    """The autotuner returns boundaries from its candidate set and the
    re-planned batch still gives the oracle's results."""
    import torch
    keys, queries, buckets, wi = _make_batch_inputs(8, 48, 41, max_log2=17)
    caps = [max(_oracle_pair(keys[i], queries[i], buckets[i], wi[i])[3], 1) for i in range(len(keys))]
    b = hg.Batch([from_np_u(a) for a in keys], [from_np_u(q) for q in queries], buckets, wi, caps)
    params, ms = b.autotune()
    assert params["part_min"] in (1 << 12, 1 << 13, 1 << 14, 1 << 15, 1 << 16)
    assert params["l2_table_bytes"] in (0, 12 << 20, 24 << 20, 48 << 20)
    assert ms > 0
    b.run()
    torch.cuda.synchronize()
    assert hg.device_error() == 0
    for i in range(len(keys)):
        _check_pair(hg, b, i, keys[i], queries[i], buckets[i], wi[i], 8)


@pytest.mark.parametrize("kb", [4, 8])
def test_batch_probe_only_and_build_only_pairs(hg, kb):
    """Probe-only pairs (d_keys NULL: the table was built before, by plain
    calls, or by a build-only pair of the same batch) and build-only pairs
    (nq = 0, no count): tables and pairs equal the oracle's."""
    import ctypes

    import torch
    from hashgraph_b200._capi import BatchPair
    L = hg.lib()
    P = ctypes.c_void_p
    s = P(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(31 + kb)
    sizes = [int(2 ** rng.uniform(4, 17)) for _ in range(24)] + [1 << 15, 1 << 16]
    keys = [oracle.gen_uniform(n, kb, 700 + i) for i, n in enumerate(sizes)]
    queries = [oracle.gen_overlap(n, keys[i], 0.5, 800 + i) for i, n in enumerate(sizes)]
    dk = [from_np_u(a) for a in keys]
    dq = [from_np_u(q) for q in queries]
    kdt = torch.int32 if kb == 4 else torch.int64
    offs = [torch.empty(n + 1, dtype=torch.int32, device="cuda") for n in sizes]
    tkeys = [torch.empty(n, dtype=kdt, device="cuda") for n in sizes]
    tidx = [torch.empty(n, dtype=torch.int32, device="cuda") for n in sizes]
    counts = torch.zeros(len(sizes), dtype=torch.int64, device="cuda")
    pairs = [torch.empty((n, 2), dtype=torch.int32, device="cuda") for n in sizes]
    # even pairs: built beforehand by plain calls; odd pairs: built by a
    # build-only pair of the batch
    for i in range(0, len(sizes), 2):
        t = hg.Table.build(dk[i], sizes[i], with_index=True)
        offs[i].copy_(t.offsets)
        tkeys[i].copy_(t.view_keys())
        tidx[i].copy_(t.view_idx())
    desc = []
    for i, n in enumerate(sizes):
        if i % 2:  # build-only
            desc.append(BatchPair(P(dk[i].data_ptr()), n, n, None, 0, P(offs[i].data_ptr()), P(tkeys[i].data_ptr()),
                                  P(tidx[i].data_ptr()), None, 0, None))
    for i, n in enumerate(sizes):  # probe-only
        desc.append(BatchPair(None, n, n, P(dq[i].data_ptr()), n, P(offs[i].data_ptr()), P(tkeys[i].data_ptr()),
                              P(tidx[i].data_ptr()), P(pairs[i].data_ptr()), n, P(counts.data_ptr() + 8 * i)))
    arr = (BatchPair * len(desc))(*desc)
    for _ in range(2):  # a batch can be run again
        b = ctypes.c_void_p()
        assert L.hg_batch_create(arr, len(desc), kb, s, ctypes.byref(b)) == 0
        assert L.hg_batch_run(b, s) == 0
        L.hg_batch_free(b, s)
        torch.cuda.synchronize()
        assert hg.device_error() == 0
        for i, n in enumerate(sizes):
            off, k, idx, c, op = _oracle_pair(keys[i], queries[i], n, True)
            np.testing.assert_array_equal(to_np_u(offs[i], 4), off)
            assert int(counts[i].item()) == c
            np.testing.assert_array_equal(_sorted_pairs(to_np_u(pairs[i][:c], 4)), _sorted_pairs(op))
