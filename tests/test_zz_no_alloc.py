"""The allocation-free build entry point, hg_build_into_noalloc.

It exists for callers that must not allocate device memory when they build a
table (their HBM belongs to their own pool allocator, they run inside another
allocator's callback, or they forbid cudaMalloc after start-up).  Its scratch
is a fixed array inside the library, so it accepts at most 2^25 buckets.

Checked here through the C ABI: on two calls in a row its table equals the
oracle's and the regular entry point's (hg_build_into) -- offsets bit-exact,
every bucket the same multiset of (key, input position) --, a call takes no
device memory (free memory unchanged across it), and a bucket count above the
limit is refused.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u, to_np_u

pytestmark = pytest.mark.gpu

LIMIT = 1 << 25


def _noalloc(hg, keys_dev, n_buckets, with_index):
    import torch
    n = keys_dev.numel()
    kb = keys_dev.element_size()
    offsets = torch.empty(n_buckets + 1, dtype=torch.int32, device="cuda")
    keys_out = torch.empty(max(n, 1), dtype=keys_dev.dtype, device="cuda")
    idx_out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda") if with_index else None
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = hg.lib().hg_build_into_noalloc(
        ctypes.c_void_p(keys_dev.data_ptr()), n, kb, n_buckets, ctypes.c_void_p(offsets.data_ptr()),
        ctypes.c_void_p(keys_out.data_ptr()), ctypes.c_void_p(idx_out.data_ptr()) if with_index else None, s)
    return st, offsets, keys_out[:n], None if idx_out is None else idx_out[:n]


def _canonical(offsets, keys, idx):
    kc, ic = oracle.canonicalize(offsets, keys.copy(), None if idx is None else idx.copy())
    return kc, ic


@pytest.mark.parametrize("kb,with_index", [(8, True), (4, False)])
def test_noalloc_build_equals_regular_build_twice(hg, kb, with_index):
    # two calls in a row on the shared scratch, different shapes
    for n, n_buckets, seed in ((300_000, 1 << 18, 71), (123_457, 99_991, 72)):
        keys = oracle.gen_uniform(n, kb, seed)
        dev = from_np_u(keys)
        st, off, k, i = _noalloc(hg, dev, n_buckets, with_index)
        assert st == 0, hg.status_str(st)
        off_a = to_np_u(off, 4)
        ka, ia = _canonical(off_a, to_np_u(k, kb), None if i is None else to_np_u(i, 4))
        # against the oracle
        o_off, o_keys, o_idx = oracle.build(keys, n_buckets, with_index)
        np.testing.assert_array_equal(off_a, o_off)
        ok, oi = _canonical(o_off, o_keys, o_idx)
        np.testing.assert_array_equal(ka, ok)
        if with_index:
            np.testing.assert_array_equal(ia, oi)
        # against the regular entry point
        ref = hg.Table.build(dev, n_buckets, with_index=with_index)
        off_b = to_np_u(ref.offsets, 4)
        np.testing.assert_array_equal(off_a, off_b)
        kb_, ib = _canonical(off_b, to_np_u(ref.view_keys(), kb),
                             None if ref.idx is None else to_np_u(ref.view_idx(), 4))
        np.testing.assert_array_equal(ka, kb_)
        if with_index:
            np.testing.assert_array_equal(ia, ib)
        assert hg.device_error() == 0


def test_noalloc_call_takes_no_device_memory(hg):
    """After a first call on the device (which looks up the scratch array's
    address), a call leaves the device's free memory unchanged."""
    import torch
    n, n_buckets = 200_000, 1 << 17
    keys = from_np_u(oracle.gen_uniform(n, 8, 73))
    offsets = torch.empty(n_buckets + 1, dtype=torch.int32, device="cuda")
    keys_out = torch.empty(n, dtype=torch.int64, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    P = ctypes.c_void_p
    L = hg.lib()
    assert L.hg_build_into_noalloc(P(keys.data_ptr()), n, 8, n_buckets, P(offsets.data_ptr()),
                                   P(keys_out.data_ptr()), None, s) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert L.hg_build_into_noalloc(P(keys.data_ptr()), n, 8, n_buckets, P(offsets.data_ptr()),
                                   P(keys_out.data_ptr()), None, s) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    o_off, _, _ = oracle.build(oracle.gen_uniform(n, 8, 73), n_buckets, False)
    np.testing.assert_array_equal(to_np_u(offsets, 4), o_off)


def test_noalloc_refuses_more_buckets_than_its_scratch(hg):
    keys = from_np_u(oracle.gen_uniform(1000, 8, 5))
    st, *_ = _noalloc(hg, keys, LIMIT + 1, False)
    assert st == -6  # HG_ERR_TOO_LARGE
    assert b"2^25" in hg.lib().hg_last_error()
    st, off, k, _ = _noalloc(hg, keys, LIMIT, False)
    assert st == 0
    assert int(to_np_u(off, 4)[-1]) == 1000
