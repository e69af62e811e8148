"""GPU parity of intersect (probe + count + pair emission) against the oracle.

The bar: the match count is exact, and the sorted (a_ref, q_ref) pairs equal
the oracle's sorted pairs (the reference's multiset-join semantics)."""
import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u, to_np_u

pytestmark = pytest.mark.gpu


def _sorted_pairs(p):
    p = np.asarray(p, dtype=np.uint32).reshape(-1, 2).astype(np.uint64)
    return np.sort(p[:, 0] << np.uint64(32) | p[:, 1])


def _oracle_pairs(a_keys_np, B, with_index, q_np):
    off, k, i = oracle.build(a_keys_np, B, True)
    c, _ = oracle.intersect(off, k, i, q_np, pair_cap=0)
    c, pairs = oracle.intersect(off, k, i, q_np, pair_cap=max(c, 1))
    return c, pairs


@pytest.mark.parametrize("probe_path", [0, 1, 2])
@pytest.mark.parametrize("path", [0, 1])
@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("na,nq,B,frac", [(1 << 16, 1 << 16, 1 << 16, 0.5), (70_001, 30_000, 12_345, 0.25),
                                          (5000, 90_000, 1 << 14, 1.0), (1 << 15, 1 << 15, 1, 0.1),
                                          (300_000, 200_000, 1 << 20, 0.5)])
def test_intersect_pairs_with_index(hg, probe_path, path, kb, na, nq, B, frac):
    a = oracle.gen_uniform(na, kb, 31 + na)
    q = oracle.gen_overlap(nq, a, frac, 37 + nq)
    t = hg.Table.build(from_np_u(a), B, with_index=True, path=path)
    count, pairs = t.intersect(from_np_u(q), pair_cap=nq * 2, path=probe_path)
    c = int(count.item())
    oc, op = _oracle_pairs(a, B, True, q)
    assert c == oc
    np.testing.assert_array_equal(_sorted_pairs(to_np_u(pairs[:c], 4)), _sorted_pairs(op))
    count2, _ = t.intersect(from_np_u(q), emit=False, path=probe_path)
    assert int(count2.item()) == oc
    assert hg.device_error() == 0


@pytest.mark.parametrize("probe_path", [0, 1, 2])
def test_intersect_without_index_table(hg, probe_path):
    a = oracle.gen_uniform(200_000, 8, 41)
    q = oracle.gen_overlap(150_000, a, 0.3, 42)
    t = hg.Table.build(from_np_u(a), 1 << 17, with_index=False, path=1)
    count, pairs = t.intersect(from_np_u(q), path=probe_path)
    c = int(count.item())
    p = to_np_u(pairs[:c], 4)
    csr_keys = to_np_u(t.view_keys(), 8)
    assert np.all(csr_keys[p[:, 0]] == q[p[:, 1]])
    oc, op = _oracle_pairs(a, 1 << 17, True, q)
    assert c == oc
    np.testing.assert_array_equal(np.sort(p[:, 1]), np.sort(op[:, 1]))


@pytest.mark.parametrize("kb", [4, 8])
def test_intersect_without_index_refers_to_csr_positions(hg, kb):
    a = oracle.gen_uniform(40_000, kb, 5)
    q = oracle.gen_overlap(40_000, a, 0.5, 6)
    t = hg.Table.build(from_np_u(a), 40_000, with_index=False)
    count, pairs = t.intersect(from_np_u(q))
    c = int(count.item())
    p = to_np_u(pairs[:c], 4)
    csr_keys = to_np_u(t.view_keys(), kb)
    # a_ref is a CSR position in A holding the query's key
    assert np.all(csr_keys[p[:, 0]] == q[p[:, 1]])
    oc, op = _oracle_pairs(a, 40_000, True, q)
    assert c == oc
    np.testing.assert_array_equal(np.sort(q[p[:, 1]]), np.sort(q[op[:, 1]]))


@pytest.mark.parametrize("probe_path", [0, 1, 2])
def test_intersect_duplicates_multiply(hg, probe_path):
    """Multiset join: k copies in A and m in the queries give k*m matches.
    The partitioned probe overflows its query partitions / spills owners here."""
    a = (oracle.gen_uniform(30_000, 8, 8) % np.uint64(200)).astype(np.uint64)
    q = (oracle.gen_uniform(20_000, 8, 9) % np.uint64(300)).astype(np.uint64)
    t = hg.Table.build(from_np_u(a), 4096, with_index=True)
    expect = oracle.join_count(a, q)
    count, _ = t.intersect(from_np_u(q), emit=False, path=probe_path)
    assert int(count.item()) == expect
    count, pairs = t.intersect(from_np_u(q), pair_cap=expect, path=probe_path)
    assert int(count.item()) == expect
    oc, op = _oracle_pairs(a, 4096, True, q)
    np.testing.assert_array_equal(_sorted_pairs(to_np_u(pairs, 4)), _sorted_pairs(op))


@pytest.mark.parametrize("probe_path", [0, 1, 2])
def test_intersect_pair_capacity(hg, probe_path):
    """Too small a pair buffer: exact count, pairs truncated, error recorded."""
    a = oracle.gen_uniform(1 << 15, 4, 10)
    q = oracle.gen_overlap(1 << 15, a, 0.75, 11)
    t = hg.Table.build(from_np_u(a), 1 << 15, with_index=True)
    full, _ = t.intersect(from_np_u(q), emit=False, path=probe_path)
    c = int(full.item())
    assert hg.device_error() == 0
    cap = c // 3
    count, pairs = t.intersect(from_np_u(q), pair_cap=cap, path=probe_path)
    assert int(count.item()) == c
    assert hg.device_error() == hg.ERR_PAIR_CAPACITY
    p = to_np_u(pairs[:cap], 4)
    assert np.all(a[p[:, 0]] == q[p[:, 1]])
    assert hg.device_error() == 0


def test_intersect_empty_inputs(hg):
    import torch
    a = oracle.gen_uniform(1000, 8, 1)
    t = hg.Table.build(from_np_u(a), 1000, with_index=True)
    count, _ = t.intersect(torch.empty(0, dtype=torch.int64, device="cuda"))
    assert int(count.item()) == 0
    t0 = hg.Table.build(torch.empty(0, dtype=torch.int64, device="cuda"), 1000, with_index=True)
    count, _ = t0.intersect(from_np_u(a))
    assert int(count.item()) == 0


def test_intersect_tables_matches_reference_semantics(hg):
    """Table-vs-table form (MultiHashGraph::intersect): B's CSR keys are the
    queries; the matched-key multiset equals the reference's output of B keys."""
    import ctypes

    import torch
    L = hg.lib()
    a = oracle.gen_uniform(50_000, 8, 21)
    b = oracle.gen_overlap(60_000, a, 0.5, 22)
    da, db = from_np_u(a), from_np_u(b)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ta, tb = ctypes.c_void_p(), ctypes.c_void_p()
    assert L.hg_build(ctypes.c_void_p(da.data_ptr()), a.size, 8, 1 << 16, 0, ctypes.byref(ta), s) == 0
    assert L.hg_build(ctypes.c_void_p(db.data_ptr()), b.size, 8, 1 << 16, 1, ctypes.byref(tb), s) == 0
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    pairs = torch.empty((b.size, 2), dtype=torch.int32, device="cuda")
    assert L.hg_intersect_tables(ta, tb, ctypes.c_void_p(pairs.data_ptr()), b.size,
                                 ctypes.c_void_p(cnt.data_ptr()), s) == 0
    c = int(cnt.item())
    assert c == oracle.join_count(a, b)
    p = to_np_u(pairs[:c], 4)
    # A's 64-bit keys are distinct, so each B key matches once if it is in A;
    # q_ref is B's input position because B was built with an index
    assert np.unique(a).size == a.size
    np.testing.assert_array_equal(np.sort(b[p[:, 1]]), np.sort(b[np.isin(b, a)]))
    # mismatched bucket counts are refused, as the reference refuses them
    tc = ctypes.c_void_p()
    assert L.hg_build(ctypes.c_void_p(da.data_ptr()), a.size, 8, 1000, 0, ctypes.byref(tc), s) == 0
    assert L.hg_intersect_tables(ta, tc, None, 0, ctypes.c_void_p(cnt.data_ptr()), s) == -9
    for t in (ta, tb, tc):
        L.hg_table_free(t)


def test_partitioned_probe_of_unaligned_table(hg):
    """A table whose arrays start off a 16-byte boundary is probed with plain
    loads instead of bulk copies; results are unchanged."""
    import ctypes

    import torch
    L = hg.lib()
    n, B = 300_000, 1 << 18
    a = oracle.gen_uniform(n, 8, 51)
    q = oracle.gen_overlap(n, a, 0.4, 52)
    da, dq = from_np_u(a), from_np_u(q)
    off_buf = torch.empty(B + 2, dtype=torch.int32, device="cuda")
    key_buf = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    idx_buf = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    off, keys, idx = off_buf[1:], key_buf[1:], idx_buf[1:]
    assert off.data_ptr() % 16 and keys.data_ptr() % 16 and idx.data_ptr() % 16
    ws = torch.empty(hg.build_workspace_bytes(n, 8, B, True, 1), dtype=torch.uint8, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    P = ctypes.c_void_p
    assert L.hg_build_into_path(P(da.data_ptr()), n, 8, B, P(off.data_ptr()), P(keys.data_ptr()),
                                P(idx.data_ptr()), P(ws.data_ptr()), ws.numel(), 1, s) == 0
    wsz = ctypes.c_size_t()
    assert L.hg_intersect_workspace_size_path(n, 1, B, n, 8, 1, 1, ctypes.byref(wsz)) == 0
    pws = torch.empty(max(wsz.value, 1), dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    pairs = torch.empty((n, 2), dtype=torch.int32, device="cuda")
    assert L.hg_intersect_into_path(P(off.data_ptr()), P(keys.data_ptr()), P(idx.data_ptr()), n, B, 8,
                                    P(dq.data_ptr()), n, None, P(pairs.data_ptr()), n, P(cnt.data_ptr()),
                                    P(pws.data_ptr()), pws.numel(), 1, s) == 0
    c = int(cnt.item())
    oc, op = _oracle_pairs(a, B, True, q)
    assert c == oc
    np.testing.assert_array_equal(_sorted_pairs(to_np_u(pairs[:c], 4)), _sorted_pairs(op))
    assert hg.device_error() == 0


@pytest.mark.parametrize("probe_path", [0, 1, 2])
def test_intersect_zipf_count(hg, probe_path):
    """Zipf(1.1) keys on both sides (a few keys hold most of the mass): the
    exact multiset-join count; long buckets for the head keys."""
    cdf = oracle.zipf_cdf(1 << 14, 1.1)
    a = oracle.gen_zipf(1 << 16, 8, cdf, 21)
    q = oracle.gen_zipf(1 << 16, 8, cdf, 22)
    t = hg.Table.build(from_np_u(a), 1 << 16, with_index=True)
    count, _ = t.intersect(from_np_u(q), emit=False, path=probe_path)
    assert int(count.item()) == oracle.join_count(a, q)
    assert hg.device_error() == 0


@pytest.mark.parametrize("probe_path", [0, 1, 2])
@pytest.mark.parametrize("kb", [4, 8])
def test_intersect_count_heavy_keys(hg, probe_path, kb):
    """Count only, head keys with tens of thousands of copies in A (buckets
    far above the heavy-key threshold): the heavy keys take their count from
    the set, the rest of the long buckets are scanned by whole warps."""
    cdf = oracle.zipf_cdf(1 << 10, 1.1)
    a = oracle.gen_zipf(1 << 18, kb, cdf, 61)
    q = oracle.gen_zipf(1 << 17, kb, cdf, 62)
    t = hg.Table.build(from_np_u(a), 1 << 18, with_index=False)
    count, _ = t.intersect(from_np_u(q), emit=False, path=probe_path)
    assert int(count.item()) == oracle.join_count(a, q)
    assert hg.device_error() == 0


@pytest.mark.parametrize("kb", [4, 8])
def test_intersect_count_absent_keys_in_long_buckets(hg, kb):
    """Count only, every bucket of A long, and most queries are keys A does
    not hold: the set of A's long-bucket keys is complete, so those queries
    count zero without scanning; the rest take their counts from the set."""
    cdf = oracle.zipf_cdf(1 << 10, 1.1)
    a = oracle.gen_zipf(1 << 18, kb, cdf, 71)
    present = oracle.gen_zipf(1 << 14, kb, cdf, 72)
    absent = oracle.gen_uniform(1 << 16, kb, 73)
    q = np.concatenate([absent, present, absent[:100]])
    t = hg.Table.build(from_np_u(a), 1024, with_index=False)
    count, _ = t.intersect(from_np_u(q), emit=False, path=0)
    assert int(count.item()) == oracle.join_count(a, q)
    assert hg.device_error() == 0


@pytest.mark.parametrize("n_buckets", [1, 64])
def test_intersect_count_many_long_buckets(hg, n_buckets):
    """Every bucket long, with far more distinct keys in them than the
    heavy-key set holds: a key finds no slot, the set is not used, and every
    bucket is scanned by its warp.  The count stays exact."""
    a = (oracle.gen_uniform(1 << 20, 8, 63) % np.uint64(1 << 16)).astype(np.uint64)
    q = (oracle.gen_uniform(1 << 15, 8, 64) % np.uint64(1 << 17)).astype(np.uint64)
    t = hg.Table.build(from_np_u(a), n_buckets, with_index=False)
    count, _ = t.intersect(from_np_u(q), emit=False, path=0)
    assert int(count.item()) == oracle.join_count(a, q)
    assert hg.device_error() == 0


@pytest.mark.parametrize("probe_path", [0, -1])
@pytest.mark.parametrize("kb", [4, 8])
def test_intersect_count_mid_length_buckets(hg, probe_path, kb):
    """Count only, buckets of 16 to 63 entries (keys with 16 to 48 copies
    among unique keys): their keys go into the heavy-key set and take their
    counts from it; queries of unique keys, of keys A lacks, and of
    duplicated keys all count exactly."""
    rng = np.random.default_rng(81)
    uniq = oracle.gen_uniform(1 << 19, kb, 82)
    dup = oracle.gen_uniform(1 << 13, kb, 83)
    a = np.concatenate([uniq, np.repeat(dup, rng.integers(16, 49, dup.size))])
    a = a[rng.permutation(a.size)]
    absent = oracle.gen_uniform(1 << 14, kb, 84)
    q = np.concatenate([dup[rng.integers(0, dup.size, 1 << 16)], uniq[: 1 << 15], absent])
    t = hg.Table.build(from_np_u(a), 1 << 20, with_index=False)
    count, _ = t.intersect(from_np_u(q), emit=False, path=probe_path)
    assert int(count.item()) == oracle.join_count(a, q)
    assert hg.device_error() == 0


@pytest.mark.parametrize("probe_path", [1, 2])
def test_intersect_one_query_key_overflows(hg, probe_path):
    """Every query is the same key: its bucket range gets all the queries,
    overflows its slots in pass 1, and the gated direct probe answers."""
    a = oracle.gen_uniform(1 << 15, 8, 31)
    q = np.full(10_000, a[5], dtype=np.uint64)
    t = hg.Table.build(from_np_u(a), 1 << 15, with_index=True)
    count, pairs = t.intersect(from_np_u(q), pair_cap=10_000, path=probe_path)
    assert int(count.item()) == 10_000
    p = to_np_u(pairs, 4)
    assert np.all(p[:, 0] == 5)
    np.testing.assert_array_equal(np.sort(p[:, 1]), np.arange(10_000, dtype=np.uint32))
    assert hg.device_error() == 0
