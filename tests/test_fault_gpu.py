"""A bounded device-side wait that runs out ends in a clean error status.

The decoupled look-back of the scans gives up after a bounded number of polls
and records a device fault (HG_ERR_DEVICE_TIMEOUT).  From then on every
kernel of the library returns at entry, writing nothing, until
hg_device_error() reads and clears the fault -- so a wait that gave up never
turns into writes through wrong offsets.  The reference has no such path (it
prints and calls exit(0), include/MultiHashGraph.cuh:56-57).

Here the poll limit is lowered to 1 with the test hook hg_debug_set_wait_limit,
so the look-back of a direct build over 2^28 buckets (65536 scan tiles, each
waiting on its predecessor) runs out; nothing faults or hangs the GPU.
"""
import ctypes

import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u, to_np_u

pytestmark = pytest.mark.gpu


def test_lookback_timeout_is_reported_and_the_device_recovers(hg):
    import torch
    n, B = 1 << 22, 1 << 28
    keys = oracle.gen_uniform(n, 8, 91)
    dk = from_np_u(keys)
    t = hg.Table(B, 8, False, n, path=0)  # the direct build: count, look-back scan, scatter
    L = hg.lib()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert hg.device_error() == 0
    code = 0
    for _ in range(3):  # a poll limit of 1 runs out in practice on the first attempt
        t.keys.fill_(-1)
        assert L.hg_debug_set_wait_limit(1, s) == 0
        try:
            t.rebuild(dk)  # returns OK: the host cannot see the device's state
            code = hg.device_error()
        finally:
            assert L.hg_debug_set_wait_limit(0, s) == 0
        if code != 0:
            break
        # no wait ran out this time: the table must be right
        o_off, _, _ = oracle.build(keys, B, False, threads=oracle.max_threads())
        np.testing.assert_array_equal(to_np_u(t.offsets, 4), o_off)
    assert code == -5  # HG_ERR_DEVICE_TIMEOUT
    # the scatter after the scan returned at entry: no key was written
    assert bool((t.keys == -1).all())
    # the fault was cleared by the read; the device answers and builds right
    assert hg.device_error() == 0
    t.rebuild(dk)
    o_off, o_keys, _ = oracle.build(keys, B, False, threads=oracle.max_threads())
    off = to_np_u(t.offsets, 4)
    np.testing.assert_array_equal(off, o_off)
    kc, _ = oracle.canonicalize(off, to_np_u(t.view_keys(), 8).copy(), None)
    okc, _ = oracle.canonicalize(o_off, o_keys, None)
    np.testing.assert_array_equal(kc, okc)
    assert hg.device_error() == 0


def test_pending_fault_stops_later_kernels(hg):
    """While a fault is pending, a probe writes no pair (its count, cleared by
    the host before the kernels, stays 0); once the fault is read, the same
    probe gives the oracle's answer."""
    import torch
    n, B = 1 << 22, 1 << 28
    keys = oracle.gen_uniform(n, 8, 93)
    q = oracle.gen_overlap(1 << 16, keys, 0.5, 94)
    dk, dq = from_np_u(keys), from_np_u(q)
    L = hg.lib()
    P = ctypes.c_void_p
    s = P(torch.cuda.current_stream().cuda_stream)
    a = hg.Table.build(dk, 1 << 22, with_index=True)
    ws = torch.empty(hg.intersect_workspace_bytes(a, q.size, True), dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    pairs = torch.empty((q.size, 2), dtype=torch.int32, device="cuda")

    def probe():
        pairs.fill_(-1)
        count.fill_(-1)
        assert L.hg_intersect_into_path(P(a.offsets.data_ptr()), P(a.keys.data_ptr()), P(a.idx.data_ptr()), a.n,
                                        a.n_buckets, 8, P(dq.data_ptr()), q.size, None, P(pairs.data_ptr()),
                                        q.size, P(count.data_ptr()), P(ws.data_ptr()), ws.numel(), -1, s) == 0

    t = hg.Table(B, 8, False, n, path=0)
    code = 0
    for _ in range(3):
        assert L.hg_debug_set_wait_limit(1, s) == 0
        try:
            t.rebuild(dk)
        finally:
            assert L.hg_debug_set_wait_limit(0, s) == 0
        probe()  # with the fault (if one was recorded) still pending
        torch.cuda.synchronize()
        code = hg.device_error()
        if code != 0:
            break
    assert code == -5  # HG_ERR_DEVICE_TIMEOUT
    assert int(count.item()) == 0
    assert bool((pairs == -1).all())
    probe()
    o_off, o_keys, o_idx = oracle.build(keys, 1 << 22, True)
    oc, op = oracle.intersect(o_off, o_keys, o_idx, q, pair_cap=q.size)
    c = int(count.item())
    assert c == oc
    got = to_np_u(pairs[:c], 4).astype(np.uint64)
    exp = op.astype(np.uint64)
    np.testing.assert_array_equal(np.sort(got[:, 0] << 32 | got[:, 1]), np.sort(exp[:, 0] << 32 | exp[:, 1]))
    assert hg.device_error() == 0
