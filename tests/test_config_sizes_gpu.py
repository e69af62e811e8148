"""GPU parity at the full sizes of the benchmarked workloads.

The smaller parity tests cover every path and edge case; these run the CUDA
path at the sizes the benchmark times, with the default (planner-chosen)
paths, so that the geometry those sizes select is checked too: pass-1 coarse
partitions, the split, the coarse probe's bucket ranges, 64-bit run offsets
and tables of 2^31 buckets.  Each is compared with the oracle on the same
seeded inputs, as the reference checks its own results:
  * the CSR: offsets bit-exact and every bucket's multiset of keys (and input
    positions) equal after the canonical per-bucket sort (the reference's
    multi-vs-single check, src/MultiHashGraph.cu:797-857);
  * the intersect: the exact match count and the pairs (the reference's
    multiset-join check, test/MultiHashGraphTest.cu:340-425).

Pairs of a table built without the input positions name CSR positions, which
depend on the unspecified in-bucket order; for those the test checks that
every pair joins equal keys, that no pair repeats, and that each query
appears as often as in the oracle's pairs -- together the same set of pairs.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u, to_np_u

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _threads():
    return oracle.max_threads()


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _free_cuda():
    import gc

    import torch
    gc.collect()
    torch.cuda.empty_cache()


def _check_csr(t, keys_np, B, with_index):
    """Offsets bit-exact and canonical buckets equal to the oracle's."""
    kb = keys_np.dtype.itemsize
    o_off, o_keys, o_idx = oracle.build(keys_np, B, with_index, threads=_threads())
    off = to_np_u(t.offsets, 4)
    assert np.array_equal(off, o_off), "offsets differ from the oracle"
    got_k = to_np_u(t.view_keys(), kb).copy()
    got_i = to_np_u(t.view_idx(), 4).copy() if with_index else None
    kc, ic = oracle.canonicalize(off, got_k, got_i)
    okc, oic = oracle.canonicalize(o_off, o_keys, o_idx)
    assert np.array_equal(kc, okc), "bucket contents differ from the oracle"
    if with_index:
        assert np.array_equal(ic, oic), "bucket input positions differ from the oracle"
    return o_off, o_keys, o_idx


def _check_pairs_by_position(t, q_dev, pairs, c, oracle_q_refs):
    """Pairs of a table without input positions: (CSR position, query)."""
    import torch
    p = pairs[:c].long()
    a_ref, q_ref = p[:, 0], p[:, 1]
    assert bool((a_ref >= 0).all()) and bool((a_ref < t.n).all())
    assert bool((t.keys[a_ref] == q_dev[q_ref]).all()), "a pair joins different keys"
    comp = torch.sort(a_ref * (1 << 32) + q_ref).values
    assert c < 2 or not bool((comp[1:] == comp[:-1]).any()), "a pair repeats"
    del comp
    got_q = torch.sort(q_ref).values
    exp_q = torch.sort(torch.from_numpy(oracle_q_refs.astype(np.int64)).to(q_dev.device)).values
    assert torch.equal(got_q, exp_q), "per-query match counts differ from the oracle"


def _check_pairs_by_index(pairs, c, o_pairs, device):
    """Pairs of a table with input positions: equal to the oracle's, sorted."""
    import torch
    p = pairs[:c].long()
    got = torch.sort(p[:, 0] * (1 << 32) + p[:, 1]).values
    del p
    op = torch.from_numpy(o_pairs.astype(np.int64)).to(device)
    exp = torch.sort(op[:, 0] * (1 << 32) + op[:, 1]).values
    del op
    assert torch.equal(got, exp), "pairs differ from the oracle"


def _oracle_pairs(o_off, o_keys, o_idx, q, threads):
    c, _ = oracle.intersect(o_off, o_keys, o_idx, q, pair_cap=0, threads=threads)
    c2, pairs = oracle.intersect(o_off, o_keys, o_idx, q, pair_cap=max(c, 1), threads=threads)
    assert c2 == c
    return c, pairs


# ---------------------------------------------------------------------------
# small: 2^20 u32, B = 2^20, 50% overlap -- against the reference's own digest
# ---------------------------------------------------------------------------
def _ref_digest():
    with open(os.path.join(GOLDEN, "ref_multi_cases.json")) as f:
        return json.load(f)["digest"]


@pytest.mark.parametrize("probe_path", [-1, 0, 1, 2])
@pytest.mark.parametrize("path", [-1, 0, 1])
def test_small_config_matches_reference_digest(hg, path, probe_path):
    """A = 2^20 u32 (seed 1), queries = 2^20 u32 with 50% drawn from A (seed
    2), B = 2^20, no index: offsets, canonical keys, match count and sorted
    matched keys hash to the digest of the reference MultiHashGraph's own
    results on these inputs (run on a B200; tests/golden/make_golden.py)."""
    from tests.golden.make_golden import make_inputs
    d = _ref_digest()
    a, q = make_inputs(d["key_bytes"], d["n_a"], d["n_b"], d["kind"], d["seed_a"], d["seed_b"], d["frac"])
    B = d["n_buckets"]
    t = hg.Table.build(from_np_u(a), B, with_index=False, path=path)
    off = to_np_u(t.offsets, 4)
    assert _sha(off) == d["offsets_sha256"]
    kc, _ = oracle.canonicalize(off, to_np_u(t.view_keys(), 4).copy(), None)
    assert _sha(kc) == d["canonical_keys_sha256"]
    dq = from_np_u(q)
    count, pairs = t.intersect(dq, pair_cap=q.size, path=probe_path)
    c = int(count.item())
    assert c == d["common"]
    qref = to_np_u(pairs[:c], 4)[:, 1]
    assert _sha(np.sort(q[qref])) == d["matched_keys_sha256"]
    o_off, o_keys, _ = oracle.build(a, B, False)
    oc, op = _oracle_pairs(o_off, o_keys, None, q, _threads())
    assert oc == c
    _check_pairs_by_position(t, dq, pairs, c, op[:, 1])
    assert hg.device_error() == 0


@pytest.mark.parametrize("path", [0, 1])
def test_small_config_pairs_with_index(hg, path):
    """The same inputs built with input positions: sorted (index_A, query)
    pairs equal the oracle's."""
    from tests.golden.make_golden import make_inputs
    d = _ref_digest()
    a, q = make_inputs(d["key_bytes"], d["n_a"], d["n_b"], d["kind"], d["seed_a"], d["seed_b"], d["frac"])
    B = d["n_buckets"]
    t = hg.Table.build(from_np_u(a), B, with_index=True, path=path)
    o_off, o_keys, o_idx = _check_csr(t, a, B, True)
    count, pairs = t.intersect(from_np_u(q), pair_cap=q.size)
    c = int(count.item())
    oc, op = _oracle_pairs(o_off, o_keys, o_idx, q, _threads())
    assert c == oc == d["common"]
    _check_pairs_by_index(pairs, c, op, t.device)


# ---------------------------------------------------------------------------
# large: 2^28 u64, B = 2^28, 25% overlap, no index (the benchmark's step)
# ---------------------------------------------------------------------------
def test_large_config_uniform(hg):
    """A = 2^28 u64 uniform (seed 3), queries = 2^28 u64 with 25% drawn from A
    (seed 30), B = 2^28, no index, pairs emitted: the benchmark's default
    step on its default paths (pass 1 into 512 coarse partitions, the
    256-way split, the fine build, the coarse probe over 2^20-bucket
    ranges)."""
    import torch
    n = 1 << 28
    a = oracle.gen_uniform(n, 8, 3)
    q = oracle.gen_overlap(n, a, 0.25, 30)
    da = hg.gen_uniform(n, 8, 3, device="cuda")
    dq = hg.gen_overlap(n, da, 0.25, 30)
    assert np.array_equal(to_np_u(dq, 8), q), "device generator differs from the oracle's"
    t = hg.Table.build(da, n, with_index=False)
    del da
    o_off, o_keys, _ = _check_csr(t, a, n, False)
    count, pairs = t.intersect(dq, pair_cap=n)
    torch.cuda.synchronize()
    c = int(count.item())
    oc, op = _oracle_pairs(o_off, o_keys, None, q, _threads())
    del o_off, o_keys, a
    assert c == oc
    _check_pairs_by_position(t, dq, pairs, c, op[:, 1])
    assert hg.device_error() == 0
    del t, pairs, dq, count
    _free_cuda()


def test_large_config_zipf_count(hg):
    """A and queries = 2^28 u64 Zipf(1.1) over one 2^24-key universe (seeds 3
    and 30), B = 2^28, count only: the exact multiset-join count,
    sum over keys of multA * multQ (about 1.4e15, in 64 bits), with buckets
    of tens of millions of copies of the head keys."""
    import torch
    n = 1 << 28
    cdf = oracle.zipf_cdf(1 << 24, 1.1)
    a = oracle.gen_zipf(n, 8, cdf, 3)
    q = oracle.gen_zipf(n, 8, cdf, 30)
    expected = oracle.join_count_hashed(a, q, max_distinct=1 << 24, threads=_threads())
    dcdf = hg.zipf_cdf(1 << 24, 1.1, device="cuda")
    da = hg.gen_zipf(n, 8, dcdf, 3)
    dq = hg.gen_zipf(n, 8, dcdf, 30)
    assert np.array_equal(to_np_u(da, 8), a) and np.array_equal(to_np_u(dq, 8), q)
    t = hg.Table.build(da, n, with_index=False)
    del da
    _check_csr(t, a, n, False)
    count, _ = t.intersect(dq, emit=False)
    torch.cuda.synchronize()
    assert int(count.item()) == expected
    assert hg.device_error() == 0
    del t, dq, count
    _free_cuda()


# ---------------------------------------------------------------------------
# capacity: 2^30 u32 + index, B = 2^31 (load factor 0.5), 10% overlap
# ---------------------------------------------------------------------------
def test_capacity_config_lf05(hg):
    """A = 2^30 u32 uniform (seed 4) with input positions, B = 2^31 buckets
    (load factor 0.5), queries = 2^30 u32 with 10% drawn from A (seed 40):
    offsets (2^31 + 1 of them) bit-exact, canonical (key, index) buckets,
    the count and the sorted (index_A, query) pairs equal to the oracle's."""
    import torch
    n, B = 1 << 30, 1 << 31
    a = oracle.gen_uniform(n, 4, 4)
    q = oracle.gen_overlap(n, a, 0.1, 40)
    t = hg.Table.build(from_np_u(a), B, with_index=True)
    o_off, o_keys, o_idx = _check_csr(t, a, B, True)
    del a
    t.workspace = None
    _free_cuda()
    dq = from_np_u(q)
    oc, op = _oracle_pairs(o_off, o_keys, o_idx, q, _threads())
    del o_off, o_keys, o_idx, q
    count, pairs = t.intersect(dq, pair_cap=oc)
    torch.cuda.synchronize()
    c = int(count.item())
    assert c == oc
    del dq, t
    _free_cuda()
    _check_pairs_by_index(pairs, c, op, pairs.device)
    assert hg.device_error() == 0
    del pairs, count
    _free_cuda()
