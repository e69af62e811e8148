"""CPU tests of the oracle: pinned to the reference's own outputs (golden
fixtures), then checked against independent numpy restatements."""
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Known answers of the reference's hash_murmur compiled on the host
# (include/SingleHashGraphOperators.cuh:31-69).
KNOWN = {0: 0x2362F9DE, 1: 0xFBF1402A, 2: 0x40B23B7F, 42: 0xBC5B91E3, 0xFFFFFFFF: 0x76293B50}


def test_murmur_known_answers():
    for k, h in KNOWN.items():
        assert oracle.lib().or_murmur3_low32(k) == h
    # only the low 32 bits of a 64-bit key reach the hash
    assert oracle.lib().or_murmur3_low32((1 << 32) + 5) == oracle.lib().or_murmur3_low32(5)


def test_murmur_matches_reference_fixture():
    g = np.load(os.path.join(GOLDEN, "murmur_ref.npz"))
    keys = g["keys"]
    ours = oracle.murmur(keys)
    np.testing.assert_array_equal(ours, g["hash_single"])
    np.testing.assert_array_equal(ours, g["hash_multi"])


def _np_murmur(keys):
    k = (keys.astype(np.uint64) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    with np.errstate(over="ignore"):
        k = k * np.uint32(0xCC9E2D51)
        k = (k << np.uint32(15)) | (k >> np.uint32(17))
        k = k * np.uint32(0x1B873593)
        h = (k << np.uint32(13)) | (k >> np.uint32(19))
        h = h * np.uint32(5) + np.uint32(0xE6546B64)
        h ^= np.uint32(4)
        h ^= h >> np.uint32(16)
        h = h * np.uint32(0x85EBCA6B)
        h ^= h >> np.uint32(13)
        h = h * np.uint32(0xC2B2AE35)
        h ^= h >> np.uint32(16)
    return h


def test_murmur_numpy_restatement():
    keys = oracle.gen_uniform(1 << 16, 8, 99)
    np.testing.assert_array_equal(_np_murmur(keys), oracle.murmur(keys))


def test_fastmod_exact():
    L = oracle.lib()
    rng = np.random.default_rng(5)
    divisors = [1, 2, 3, 5, 7, 1000, 999_983, 1 << 20, (1 << 20) + 1, 3 << 29, (1 << 31) - 1,
                1 << 31, (1 << 31) + 1, (1 << 32) - 1, (1 << 32) - 2]
    divisors += [int(x) for x in rng.integers(1, 1 << 32, 40, dtype=np.uint64)]
    nums = [0, 1, 2, (1 << 31) - 1, 1 << 31, (1 << 32) - 1, (1 << 32) - 2]
    nums += [int(x) for x in rng.integers(0, 1 << 32, 300, dtype=np.uint64)]
    for d in divisors:
        m = L.or_fastmod_magic(d)
        for a in nums:
            assert L.or_fastmod(a, m, d) == a % d, (a, d)
    # exhaustive over a contiguous window of numerators for awkward divisors
    for d in (3, 7, 641, (1 << 32) - 1):
        m = L.or_fastmod_magic(d)
        for a in range((1 << 32) - 3000, 1 << 32):
            assert L.or_fastmod(a, m, d) == a % d


def test_generators_deterministic_and_shaped():
    a1 = oracle.gen_uniform(1 << 14, 4, 1)
    a2 = oracle.gen_uniform(1 << 14, 4, 1)
    np.testing.assert_array_equal(a1, a2)
    assert not np.array_equal(a1, oracle.gen_uniform(1 << 14, 4, 2))
    b = oracle.gen_overlap(1 << 14, a1, 0.5, 2)
    # exactly half drawn from distinct positions of A (a1 is duplicate-free here)
    assert np.unique(a1).size == a1.size
    assert np.isin(b, a1).sum() == (1 << 13)
    # the shuffle is a bijection: permuting 0..n-1 covers every index
    L = oracle.lib()
    for n in (1, 2, 3, 1000, 4096, 5000):
        perm = [L.or_perm(i, n, 7) for i in range(n)]
        assert sorted(perm) == list(range(n))


def test_zipf_head_mass():
    cdf = oracle.zipf_cdf(1 << 16, 1.1)
    keys = oracle.gen_zipf(1 << 18, 8, cdf, 5)
    _, counts = np.unique(keys, return_counts=True)
    top = counts.max() / keys.size
    h = np.sum(np.arange(1, (1 << 16) + 1, dtype=np.float64) ** -1.1)
    assert abs(top - 1.0 / h) < 0.01


def _np_build(keys, B):
    b = oracle.buckets(keys, B)
    order = np.argsort(b, kind="stable")
    counts = np.bincount(b.astype(np.int64), minlength=B)
    offsets = np.zeros(B + 1, dtype=np.uint64)
    np.cumsum(counts, out=offsets[1:])
    return offsets.astype(np.uint32), keys[order], order.astype(np.uint32)


@pytest.mark.parametrize("kb,n,B", [(4, 0, 7), (4, 1, 1), (8, 1000, 1), (4, 5000, 4999),
                                    (8, 1 << 14, 1 << 14), (4, 1 << 15, 1 << 12), (8, 3000, 100_000)])
def test_build_matches_numpy_and_mt(kb, n, B):
    keys = oracle.gen_uniform(n, kb, 123 + n)
    off, k, i = oracle.build(keys, B, True)
    o2, k2, i2 = _np_build(keys, B)
    np.testing.assert_array_equal(off, o2)
    np.testing.assert_array_equal(k, k2)
    np.testing.assert_array_equal(i, i2)
    o3, k3, i3 = oracle.build(keys, B, True, threads=4)
    np.testing.assert_array_equal(off, o3)
    np.testing.assert_array_equal(k, k3)
    np.testing.assert_array_equal(i, i3)


def test_canonicalize_and_intersect_semantics():
    a = oracle.gen_uniform(4000, 8, 3) % np.uint64(300)  # heavy duplicates
    q = oracle.gen_uniform(3000, 8, 4) % np.uint64(400)
    off, k, i = oracle.build(a, 257, True)
    c, pairs = oracle.intersect(off, k, i, q, pair_cap=10_000_000)
    assert c == oracle.join_count(a, q)
    # every pair joins equal keys, each (a, q) pair at most once
    assert np.all(a[pairs[:, 0]] == q[pairs[:, 1]])
    assert np.unique(pairs, axis=0).shape[0] == c
    c_mt, pairs_mt = oracle.intersect(off, k, i, q, pair_cap=10_000_000, threads=4)
    assert c_mt == c
    np.testing.assert_array_equal(pairs_mt, pairs)
    # truncated output keeps the exact count
    c2, p2 = oracle.intersect(off, k, i, q, pair_cap=17)
    assert c2 == c and p2.shape == (17, 2)
    kc, ic = oracle.canonicalize(off, k.copy(), i.copy())
    for b in range(0, 257, 16):
        s, e = off[b], off[b + 1]
        seg = list(zip(kc[s:e], ic[s:e]))
        assert seg == sorted(seg)


def _load_ref_cases():
    p = os.path.join(GOLDEN, "ref_multi_cases.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


REF = _load_ref_cases()


@pytest.mark.skipif(REF is None, reason="reference MultiHashGraph fixtures not generated yet")
@pytest.mark.parametrize("case", REF["cases"] if REF else [], ids=lambda c: c["name"])
def test_oracle_matches_reference_multihashgraph(case):
    """Oracle CSR and intersect vs the reference MultiHashGraph run on a B200."""
    from tests.golden.make_golden import make_inputs
    g = np.load(os.path.join(GOLDEN, f"ref_multi_{case['name']}.npz"))
    a, b = make_inputs(case["key_bytes"], case["n_a"], case["n_b"], case["kind"], case["seed_a"],
                       case["seed_b"], case["frac"])
    off, k, _ = oracle.build(a, case["n_buckets"], False)
    np.testing.assert_array_equal(off, g["offsets"])
    kc, _ = oracle.canonicalize(off, k.copy(), None)
    np.testing.assert_array_equal(kc, g["keys"])
    c, pairs = oracle.intersect(off, k, None, b, pair_cap=1 << 24)
    assert c == g["common"]
    np.testing.assert_array_equal(np.sort(k[pairs[:, 0]]), g["matched_keys"])


@pytest.mark.skipif(REF is None, reason="reference MultiHashGraph fixtures not generated yet")
def test_oracle_matches_reference_digest_config1():
    import hashlib

    from tests.golden.make_golden import make_inputs
    d = REF["digest"]
    a, b = make_inputs(d["key_bytes"], d["n_a"], d["n_b"], d["kind"], d["seed_a"], d["seed_b"],
                       d["frac"])
    off, k, _ = oracle.build(a, d["n_buckets"], False, threads=oracle.max_threads())
    assert hashlib.sha256(off.tobytes()).hexdigest() == d["offsets_sha256"]
    kc, _ = oracle.canonicalize(off, k.copy(), None)
    assert hashlib.sha256(kc.tobytes()).hexdigest() == d["canonical_keys_sha256"]
    c, pairs = oracle.intersect(off, k, None, b, pair_cap=1 << 22, threads=oracle.max_threads())
    assert c == d["common"]
    mk = np.sort(k[pairs[:, 0]])
    assert hashlib.sha256(mk.tobytes()).hexdigest() == d["matched_keys_sha256"]
