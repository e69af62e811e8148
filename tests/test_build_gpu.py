"""GPU parity of the CSR build against the oracle (through the C ABI).

The bar: offsets bit-exact; every bucket holds exactly the oracle's multiset
of (key, input position) -- compared after the canonical per-bucket sort,
since the in-bucket order is unspecified (as in the reference)."""
import numpy as np
import pytest

import oracle
from tests.conftest import device_array, from_np_u, to_np_u

pytestmark = pytest.mark.gpu

PATHS = [0, 1]  # direct, partitioned


def _check_table(t, keys_np, B, with_index):
    kb = keys_np.dtype.itemsize
    off = to_np_u(t.offsets, 4)
    keys = to_np_u(t.view_keys(), kb).copy()
    idx = to_np_u(t.view_idx(), 4).copy() if with_index else None
    o_off, o_keys, o_idx = oracle.build(keys_np, B, with_index)
    np.testing.assert_array_equal(off, o_off)
    kc, ic = oracle.canonicalize(off, keys, idx)
    okc, oic = oracle.canonicalize(o_off, o_keys.copy(), None if o_idx is None else o_idx.copy())
    np.testing.assert_array_equal(kc, okc)
    if with_index:
        np.testing.assert_array_equal(ic, oic)


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("with_index", [False, True])
@pytest.mark.parametrize("n,B", [(1 << 16, 1 << 16), (100_003, 77_777), (50_000, 1 << 18),
                                 (1 << 17, 1 << 12), (3000, 1)])
def test_build_parity(hg, path, kb, with_index, n, B):
    keys = oracle.gen_uniform(n, kb, 1000 + n + kb)
    t = hg.Table.build(from_np_u(keys), B, with_index=with_index, path=path)
    _check_table(t, keys, B, with_index)
    assert hg.device_error() == 0


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("n", [0, 1, 31, 33, 1023])
def test_build_edge_sizes(hg, path, n):
    keys = oracle.gen_uniform(n, 8, 7 + n)
    t = hg.Table.build(from_np_u(keys), 1000, with_index=True, path=path)
    _check_table(t, keys, 1000, True)


@pytest.mark.parametrize("path", PATHS)
def test_build_heavy_duplicates(hg, path):
    """All keys equal / few distinct keys: hot buckets serialise atomics and
    overflow the partitioned path's slot ranges (device-side fallback)."""
    n = 200_000
    for keys in (np.full(n, 123456789, dtype=np.uint64),
                 (oracle.gen_uniform(n, 8, 3) % np.uint64(50)).astype(np.uint64)):
        t = hg.Table.build(from_np_u(keys), 1 << 16, with_index=True, path=path)
        _check_table(t, keys, 1 << 16, True)
        assert hg.device_error() == 0


@pytest.mark.parametrize("path", PATHS)
def test_build_zipf(hg, path):
    cdf = oracle.zipf_cdf(1 << 14, 1.1)
    keys = oracle.gen_zipf(1 << 18, 8, cdf, 9)
    t = hg.Table.build(from_np_u(keys), 1 << 18, with_index=True, path=path)
    _check_table(t, keys, 1 << 18, True)


@pytest.mark.parametrize("kb", [4, 8])
def test_build_zipf_grouped_fallback(hg, kb):
    """Partitioned build of skewed keys with an index: the skew check flags
    the overflow before pass 1 and the fallback groups the keys by coarse
    partition into exactly sized runs before its direct build."""
    cdf = oracle.zipf_cdf(1 << 16, 1.1)
    n = 1 << 22
    keys = oracle.gen_zipf(n, kb, cdf, 17)
    t = hg.Table.build(from_np_u(keys), n, with_index=True, path=1)
    _check_table(t, keys, n, True)
    assert hg.device_error() == 0


def test_build_late_overflow_grouped_fallback(hg):
    """A partition a little over its slots: the 8192-key sample does not flag
    it, pass 1 overflows, and the fallback (grouping, then the direct build)
    redoes the table from the input."""
    n = B = 1 << 22
    base = oracle.gen_uniform(n, 8, 23)
    extra = oracle.gen_uniform(1 << 18, 8, 24)
    # about 2% more keys in the first of the 8 coarse partitions (2^19 buckets)
    extra = extra[oracle.buckets(extra, B) < (1 << 19)][:10_000]
    keys = np.concatenate([base[: n - extra.size], extra])
    keys = keys[np.random.default_rng(25).permutation(keys.size)]
    t = hg.Table.build(from_np_u(keys), B, with_index=True, path=1)
    _check_table(t, keys, B, True)
    assert hg.device_error() == 0


def test_build_unaligned_input(hg):
    """Keys that do not start on a 16-byte boundary take the scalar-load path."""
    import torch
    keys = oracle.gen_uniform(10_001, 4, 5)
    dev = from_np_u(np.concatenate([np.zeros(1, np.uint32), keys]))
    sub = dev[1:]
    assert sub.data_ptr() % 16 != 0
    for path in PATHS:
        t = hg.Table.build(sub, 4096, with_index=True, path=path)
        _check_table(t, keys, 4096, True)
    torch.cuda.synchronize()


@pytest.mark.parametrize("path", PATHS)
def test_rebuild_reuses_table(hg, path):
    """A second build into the same buffers (smaller n) gives a fresh table."""
    k1 = oracle.gen_uniform(1 << 16, 4, 1)
    k2 = oracle.gen_uniform(40_000, 4, 2)
    t = hg.Table.build(from_np_u(k1), 1 << 15, with_index=True, path=path)
    t.rebuild(from_np_u(k2))
    _check_table(t, k2, 1 << 15, True)


def test_library_owned_table_api(hg):
    """hg_build / hg_table_view / hg_table_free on a library-owned table."""
    import ctypes

    import torch
    L = hg.lib()
    keys = oracle.gen_uniform(70_000, 8, 17)
    dk = from_np_u(keys)
    tbl = ctypes.c_void_p()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.hg_build(ctypes.c_void_p(dk.data_ptr()), keys.size, 8, 50_000, 1, ctypes.byref(tbl), s) == 0
    po, pk, pi = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    n, B, kb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int()
    assert L.hg_table_view(tbl, ctypes.byref(po), ctypes.byref(pk), ctypes.byref(pi), ctypes.byref(n),
                           ctypes.byref(B), ctypes.byref(kb)) == 0
    assert (n.value, B.value, kb.value) == (keys.size, 50_000, 8)
    torch.cuda.synchronize()
    off = device_array(po.value, 50_001, np.uint32)
    got_k = device_array(pk.value, keys.size, np.uint64)
    got_i = device_array(pi.value, keys.size, np.uint32)
    o_off, o_k, o_i = oracle.build(keys, 50_000, True)
    np.testing.assert_array_equal(off, o_off)
    kc, ic = oracle.canonicalize(off, got_k, got_i)
    okc, oic = oracle.canonicalize(o_off, o_k.copy(), o_i.copy())
    np.testing.assert_array_equal(kc, okc)
    np.testing.assert_array_equal(ic, oic)
    nbytes = ctypes.c_size_t()
    assert L.hg_table_device_bytes(tbl, ctypes.byref(nbytes)) == 0 and nbytes.value > 0
    L.hg_table_free(tbl)
