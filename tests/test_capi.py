"""CPU checks of the C-ABI library: it loads, exports every symbol the headers
declare, and its host-side logic (hash, argument checks, planning) behaves.
No call here launches device work."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hashgraph_b200.h")


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(hg_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def capi():
    from hashgraph_b200 import _capi
    _capi.build_library()
    return _capi


def test_library_exports_every_declared_symbol(capi):
    names = declared_functions(HEADER)
    assert len(names) >= 20
    L = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the binding declares a signature for each
    assert set(names) <= set(capi.SIGNATURES), set(names) - set(capi.SIGNATURES)


def test_host_hash_matches_oracle(capi):
    L = capi.lib()
    keys = oracle.gen_uniform(2048, 8, 77)
    ours = np.array([L.hg_hash(int(k)) for k in keys], dtype=np.uint32)
    np.testing.assert_array_equal(ours, oracle.murmur(keys))
    assert L.hg_hash(0) == 0x2362F9DE


def test_status_strings(capi):
    L = capi.lib()
    for code in capi.STATUS_NAMES:
        assert L.hg_status_str(code)
    assert b"sm_100a" in L.hg_version()


def test_argument_checks_without_device(capi):
    L = capi.lib()
    out = ctypes.c_size_t(0)
    assert L.hg_build_workspace_size(1000, 3, 1000, 0, ctypes.byref(out)) == -8
    assert L.hg_build_workspace_size(1000, 4, 0, 0, ctypes.byref(out)) == -1
    assert L.hg_build_workspace_size(1 << 32, 4, 1000, 0, ctypes.byref(out)) == -6
    assert L.hg_build_workspace_size(1000, 4, (1 << 32) + 1, 0, ctypes.byref(out)) == -6
    assert L.hg_build_workspace_size(1000, 4, 1000, 0, None) == -1
    assert L.hg_intersect_workspace_size(1000, 0, 1000, 10, 5, 1, ctypes.byref(out)) == -8
    assert L.hg_build_into(None, 10, 8, 10, None, None, None, None, 0, None) == -1
    assert L.hg_table_create(10, 8, 10, 0, None) == -1
    assert L.hg_zipf_cdf(None, 10, 1.1) == -1
    # batched build + intersect: descriptors are checked before any device call
    h = ctypes.c_void_p()
    pairs = (capi.BatchPair * 1)()
    assert L.hg_batch_create(pairs, 1, 3, None, ctypes.byref(h)) == -8
    assert L.hg_batch_create(pairs, -1, 8, None, ctypes.byref(h)) == -1
    assert L.hg_batch_create(pairs, 1, 8, None, None) == -1
    pairs[0].n, pairs[0].n_buckets = 10, 0  # no buckets
    assert L.hg_batch_create(pairs, 1, 8, None, ctypes.byref(h)) == -1
    pairs[0].n_buckets, pairs[0].d_offsets, pairs[0].d_count = 16, 16, 16  # keys but no key buffer
    assert L.hg_batch_create(pairs, 1, 8, None, ctypes.byref(h)) == -1
    pairs[0].d_keys, pairs[0].d_keys_out, pairs[0].n = 16, 16, 1 << 32
    assert L.hg_batch_create(pairs, 1, 8, None, ctypes.byref(h)) == -6
    assert not h.value
    assert L.hg_batch_run(None, None) == -1


def test_workspace_plans(capi):
    L = capi.lib()
    out = ctypes.c_size_t(0)
    # direct path: only scan status and flags
    assert L.hg_build_workspace_size_path(1 << 20, 4, 1 << 20, 0, 0, ctypes.byref(out)) == 0
    direct = out.value
    assert direct < (1 << 20)
    # partitioned path: coarse and fine partition buffers each hold every key
    # (+ index) with a few percent of slack
    assert L.hg_build_workspace_size_path(1 << 20, 4, 1 << 20, 1, 1, ctypes.byref(out)) == 0
    part = out.value
    assert 2 * (1 << 20) * 8 <= part < (1 << 20) * 8 * 2.5
    # the planner picks the partitioned path for a 2^28 x u64 table
    assert L.hg_build_workspace_size(1 << 28, 8, 1 << 28, 0, ctypes.byref(out)) == 0
    assert out.value >= (1 << 28) * 8
    # and the coarse probe for 2^28 queries against it: one pass of the queries
    # (+ their positions) into L2-sized bucket ranges, no fine partitions
    assert L.hg_intersect_workspace_size(1 << 28, 0, 1 << 28, 1 << 28, 8, 1, ctypes.byref(out)) == 0
    assert (1 << 28) * 12 <= out.value < (1 << 28) * 12 * 1.1
    # the partitioned probe, asked for, stages coarse and fine partitions
    assert L.hg_intersect_workspace_size_path(1 << 28, 0, 1 << 28, 1 << 28, 8, 1, 1, ctypes.byref(out)) == 0
    assert out.value >= 2 * (1 << 28) * 12
    # an unknown path is an argument error
    assert L.hg_intersect_workspace_size_path(1 << 20, 0, 1 << 20, 1 << 20, 8, 1, 3, ctypes.byref(out)) == -1
    # a single bucket: the partitioned probe still plans (A's slice is read in
    # place), the partitioned build cannot stage it and plans the direct one
    assert L.hg_intersect_workspace_size_path(1 << 15, 0, 1, 1 << 15, 4, 1, 1, ctypes.byref(out)) == 0
    assert L.hg_build_workspace_size_path(1 << 15, 4, 1, 0, 1, ctypes.byref(out)) == 0
    assert out.value < (1 << 16)
    # a small probe stays direct: only tile status words
    assert L.hg_intersect_workspace_size(1 << 16, 0, 1 << 16, 1 << 16, 8, 1, ctypes.byref(out)) == 0
    assert out.value < (1 << 16)


def test_zipf_cdf_matches_oracle(capi):
    L = capi.lib()
    U = 1 << 12
    ours = np.empty(U, dtype=np.uint64)
    assert L.hg_zipf_cdf(ours.ctypes.data_as(ctypes.c_void_p), U, 1.1) == 0
    np.testing.assert_array_equal(ours, oracle.zipf_cdf(U, 1.1))


def test_table_file_header_checks_without_device(capi, tmp_path):
    """hg_table_file_info reads only the header: no device needed."""
    import struct
    L = capi.lib()
    n, nb = ctypes.c_uint64(0), ctypes.c_uint64(0)
    kb, wi = ctypes.c_int(0), ctypes.c_int(0)
    args = (ctypes.byref(n), ctypes.byref(nb), ctypes.byref(kb), ctypes.byref(wi))
    assert L.hg_table_file_info(str(tmp_path / "missing").encode(), *args) == -1
    # a valid header for 3 u64 keys in 2 buckets with index: 64 + 12 + 24 + 12 bytes
    hdr = b"HGB2TBL\0" + struct.pack("<4I3Q2Q", 1, 8, 1, 1, 3, 2, 0, 0, 0)
    good = tmp_path / "good.hgt"
    good.write_bytes(hdr + bytes(12 + 24 + 12))
    assert L.hg_table_file_info(str(good).encode(), *args) == 0
    assert (n.value, nb.value, kb.value, wi.value) == (3, 2, 8, 1)
    (tmp_path / "short.hgt").write_bytes(hdr + bytes(10))
    assert L.hg_table_file_info(str(tmp_path / "short.hgt").encode(), *args) == -1
    (tmp_path / "magic.hgt").write_bytes(b"XGB2TBL\0" + hdr[8:] + bytes(48))
    assert L.hg_table_file_info(str(tmp_path / "magic.hgt").encode(), *args) == -1
    wide = b"HGB2TBL\0" + struct.pack("<4I3Q2Q", 1, 5, 1, 1, 3, 2, 0, 0, 0)
    (tmp_path / "width.hgt").write_bytes(wide + bytes(48))
    assert L.hg_table_file_info(str(tmp_path / "width.hgt").encode(), *args) == -8


def test_server_argument_checks_without_device(capi):
    """hg_server_* check their arguments before any device call."""
    L = capi.lib()
    h = ctypes.c_void_p()
    assert L.hg_server_create(1 << 30, 8, 2, 1 << 20, 3, ctypes.byref(h)) == -8
    assert L.hg_server_create(1 << 30, 0, 2, 1 << 20, 8, ctypes.byref(h)) == -1
    assert L.hg_server_create(1 << 30, 8, 0, 1 << 20, 8, ctypes.byref(h)) == -1
    assert L.hg_server_create(1 << 30, 8, 65, 1 << 20, 8, ctypes.byref(h)) == -1
    assert L.hg_server_create(0, 8, 2, 1 << 20, 8, ctypes.byref(h)) == -1
    assert L.hg_server_create(1 << 30, 8, 2, 1 << 32, 8, ctypes.byref(h)) == -6
    assert L.hg_server_create(1 << 30, 8, 2, 1 << 20, 8, None) == -1
    assert not h.value
    t = ctypes.c_uint64(0)
    n = ctypes.c_int(0)
    assert L.hg_server_build(None, 0, None, 0, 1, 0, 0.0, ctypes.byref(t)) == -1
    assert L.hg_server_intersect(None, 0, None, 0, None, 0, 0.0, ctypes.byref(t)) == -1
    assert L.hg_server_poll(None, 0, None, 0, ctypes.byref(n)) == -1
    from hashgraph_b200._capi import ServerRequest
    reqs = (ServerRequest * 1)()
    tick = (ctypes.c_uint64 * 1)()
    assert L.hg_server_submit(None, reqs, 1, tick, ctypes.byref(n)) == -1
    assert L.hg_server_submit(None, None, 0, None, None) == -1
    assert L.hg_server_stats(None, None, None, None, None) == -1
    assert L.hg_server_reserve(None, 1 << 20) == -1
    L.hg_server_free(None)
    t0 = L.hg_server_now()
    assert t0 > 0 and L.hg_server_now() >= t0


def test_shard_argument_checks_without_device(capi):
    """hg_shard_* check ranges and splits before any device call."""
    L = capi.lib()
    f = 16  # a stand-in device pointer: no call below reaches the device
    out = ctypes.c_size_t(0)
    # lo >= hi, hi > B, an unaligned range of a 2^32-bucket table, key width
    assert L.hg_shard_build_into(f, None, 4, 8, 100, 50, 50, f, f, None, f, 1 << 20, None) == -1
    assert L.hg_shard_build_into(f, None, 4, 8, 100, 50, 101, f, f, None, f, 1 << 20, None) == -1
    assert L.hg_shard_build_into(f, None, 4, 8, 1 << 32, 3, 1 << 20, f, f, None, f, 1 << 20, None) == -6
    assert L.hg_shard_build_into(f, None, 4, 5, 100, 0, 50, f, f, None, f, 1 << 20, None) == -8
    assert L.hg_shard_intersect_into(f, f, None, 4, 100, 60, 40, 8, f, 4, None, None, 0, f, f, 1 << 20, None) == -1
    # splits that do not start at 0 / end at B, or that decrease
    for bad in ([0, 60, 50, 100], [1, 50, 70, 100], [0, 50, 70, 99]):
        sp = np.array(bad, dtype=np.uint64)
        assert L.hg_shard_route(f, 4, 8, 100, sp.ctypes.data_as(ctypes.c_void_p), 3, 0, f, None, f, f,
                                1 << 20, None) == -1
    sp = np.array([0, 100], dtype=np.uint64)
    assert L.hg_shard_route(f, 4, 8, 100, sp.ctypes.data_as(ctypes.c_void_p), 0, 0, f, None, f, f, 1 << 20, None) == -1
    # global indices past 2^32
    assert L.hg_shard_route(f, 4, 8, 100, sp.ctypes.data_as(ctypes.c_void_p), 1, (1 << 32) - 2, f, f, f, f,
                            1 << 20, None) == -6
    assert L.hg_shard_route_workspace_size(1000, 65, ctypes.byref(out)) == -1
    assert L.hg_shard_route_workspace_size(1000, 8, ctypes.byref(out)) == 0 and out.value > 0
    assert L.hg_shard_histogram(f, 10, 8, 100, 40000, f, None) == -6
    assert L.hg_shard_histogram(f, 10, 8, 0, 16, f, None) == -1


def test_batch_params_without_device(capi):
    """Size-class defaults, and argument checks of the parameterised create and
    the autotuner before any device call."""
    L = capi.lib()
    prm = capi.BatchParams()
    assert L.hg_batch_params_default(ctypes.byref(prm)) == 0
    assert (prm.part_min, prm.l2_table_bytes) == (1 << 14, 24 << 20)
    assert L.hg_batch_params_default(None) == -1
    h = ctypes.c_void_p()
    pairs = (capi.BatchPair * 1)()
    bad = capi.BatchParams(0, 1 << 20)
    assert L.hg_batch_create_params(pairs, 1, 8, ctypes.byref(bad), None, ctypes.byref(h)) == -1
    assert L.hg_batch_create_params(pairs, 1, 8, None, None, None) == -1
    assert L.hg_batch_autotune(pairs, 1, 8, None, None, None) == -1


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("with_index", [0, 1])
def test_planner_over_shapes(capi, kb, with_index):
    """Every build and probe plan over a grid of table shapes succeeds, and the
    workspaces stay within their bounds: the coarse probe holds one pass of
    the query records (+ slack), the partitioned forms two, the direct forms
    only status words."""
    L = capi.lib()
    out = ctypes.c_size_t(0)
    for n in (0, 1, 1000, 1 << 20, 1 << 26, (1 << 30) - 1):
        for B in (1, 7, max(n, 1), 2 * max(n, 1), 1 << 32):
            if B > (1 << 32):
                continue
            rec = kb + 4 * with_index
            for path in (-1, 0, 1):
                assert L.hg_build_workspace_size_path(n, kb, B, with_index, path, ctypes.byref(out)) == 0
                # records twice with slack, plus per-partition slack slots and counters on
                # the partitioned path (up to about 0.15 byte per bucket for a sparse table;
                # the planner takes it from 48 MB of keys on, so a near-empty table with
                # many buckets stays direct)
                per_bucket = B // 512 if path == 0 else B // 6
                assert out.value <= 2.6 * n * rec + per_bucket + (64 << 20), (n, B, path, out.value)
            nq = n
            for path in (-1, 0, 1, 2):
                assert L.hg_intersect_workspace_size_path(n, with_index, B, nq, kb, 1, path,
                                                          ctypes.byref(out)) == 0, (n, B, path)
                bound = {0: 8 * (nq // 1024 + 1) + 4096,
                         1: 2.6 * nq * (kb + 4) + B // 6 + (64 << 20),
                         2: 1.3 * nq * (kb + 4) + B // 512 + (64 << 20)}
                # the planner's own choice (-1) is the direct or the coarse probe here
                assert out.value <= bound[path if path >= 0 else 2] + 8 * (nq // 1024 + 1), (n, B, path,
                                                                                             out.value)
    # beyond the 32-bit limits: a clear error, no plan
    assert L.hg_build_workspace_size(1 << 32, kb, 1 << 20, with_index, ctypes.byref(out)) == -6
    assert L.hg_intersect_workspace_size(1 << 20, with_index, 1 << 20, 1 << 32, kb, 1, ctypes.byref(out)) == -6


def test_sparse_table_plans_direct(capi):
    """One key into 2^32 buckets: the planner keeps the direct path and its
    workspace of scan status words (8 MB), not the partitioned one's slack."""
    L = capi.lib()
    out = ctypes.c_size_t(0)
    assert L.hg_build_workspace_size(1, 8, 1 << 32, 1, ctypes.byref(out)) == 0
    assert out.value < (16 << 20)
