"""Table files: save a built table, load it back, and the arrays (and every
intersect against them) are unchanged; damaged files are refused."""
import os

import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u, to_np_u

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kb,with_index,n,B", [(8, False, 300_000, 1 << 18), (4, True, 100_000, 77_777),
                                               (8, True, 0, 5), (4, False, 1, 1)])
def test_save_load_roundtrip(hg, tmp_path, kb, with_index, n, B):
    a = oracle.gen_uniform(n, kb, 12)
    t = hg.Table.build(from_np_u(a), B, with_index=with_index)
    path = tmp_path / "t.hgt"
    t.save(path)
    u = hg.Table.load(path)
    assert (u.n, u.n_buckets, u.key_bytes, u.with_index) == (n, B, kb, with_index)
    np.testing.assert_array_equal(to_np_u(u.offsets, 4), to_np_u(t.offsets, 4))
    np.testing.assert_array_equal(to_np_u(u.view_keys(), kb), to_np_u(t.view_keys(), kb))
    if with_index:
        np.testing.assert_array_equal(to_np_u(u.view_idx(), 4), to_np_u(t.view_idx(), 4))
    if n:
        q = oracle.gen_overlap(n, a, 0.5, 13)
        c1, p1 = t.intersect(from_np_u(q))
        c2, p2 = u.intersect(from_np_u(q))
        c = int(c1.item())
        assert c == int(c2.item())
        np.testing.assert_array_equal(np.sort(to_np_u(p1[:c], 4)[:, 1]), np.sort(to_np_u(p2[:c], 4)[:, 1]))
    # a loaded table can be rebuilt in place
    b = oracle.gen_uniform(n, kb, 14)
    u.rebuild(from_np_u(b))
    off, _, _ = oracle.build(b, B, True)
    np.testing.assert_array_equal(to_np_u(u.offsets, 4), off)


def test_damaged_files_are_refused(hg, tmp_path):
    a = oracle.gen_uniform(50_000, 8, 3)
    t = hg.Table.build(from_np_u(a), 40_000, with_index=True)
    path = tmp_path / "t.hgt"
    t.save(path)
    raw = bytearray(open(path, "rb").read())
    # one payload bit flipped: checksum mismatch
    bad = bytearray(raw)
    bad[64 + 4 * 40_001 + 100] ^= 1
    open(tmp_path / "flip.hgt", "wb").write(bad)
    with pytest.raises(hg.HGError):
        hg.Table.load(tmp_path / "flip.hgt")
    # truncated
    open(tmp_path / "short.hgt", "wb").write(raw[:-4])
    with pytest.raises(hg.HGError):
        hg.Table.load(tmp_path / "short.hgt")
    # bad magic
    bad = bytearray(raw)
    bad[0] = ord("X")
    open(tmp_path / "magic.hgt", "wb").write(bad)
    with pytest.raises(hg.HGError):
        hg.Table.load(tmp_path / "magic.hgt")
    assert hg.device_error() == 0


def _fnv1a64(data: bytes) -> int:
    """FNV-1a 64 of `data` (the file checksum), byte by byte: the files here
    are kept small."""
    h = 0xcbf29ce484222325
    for b in data:
        h ^= b
        h = (h * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    return h


def _rewrite_with_checksum(raw: bytearray) -> bytearray:
    import struct
    out = bytearray(raw)
    out[40:48] = struct.pack("<Q", _fnv1a64(bytes(out[64:])))
    return out


def test_forged_offsets_are_refused(hg, tmp_path):
    """Offsets that decrease or pass n are refused even when the file's
    checksum was recomputed (a crafted or hand-edited file): the probes read
    each bucket's keys straight from the offsets."""
    import struct
    n, B = 2000, 1000
    a = oracle.gen_uniform(n, 4, 21)
    t = hg.Table.build(from_np_u(a), B, with_index=False)
    path = tmp_path / "t.hgt"
    t.save(path)
    raw = bytearray(open(path, "rb").read())
    assert _rewrite_with_checksum(raw) == raw  # the checksum restated here matches the library's
    off0 = 64
    # a decreasing pair of offsets in the middle
    bad = bytearray(raw)
    v = struct.unpack_from("<I", bad, off0 + 4 * 500)[0]
    struct.pack_into("<I", bad, off0 + 4 * 500, v + 50)
    open(tmp_path / "dec.hgt", "wb").write(_rewrite_with_checksum(bad))
    with pytest.raises(hg.HGError) as e:
        hg.Table.load(tmp_path / "dec.hgt")
    assert e.value.status == -1
    assert b"offsets decrease" in hg.lib().hg_last_error()
    # an offset beyond n
    bad = bytearray(raw)
    struct.pack_into("<I", bad, off0 + 4 * 999, n + 7)
    open(tmp_path / "big.hgt", "wb").write(_rewrite_with_checksum(bad))
    with pytest.raises(hg.HGError):
        hg.Table.load(tmp_path / "big.hgt")
    assert hg.device_error() == 0


def test_index_requested_from_a_file_without_one_is_refused(hg, tmp_path):
    import ctypes

    import torch
    a = oracle.gen_uniform(1000, 8, 22)
    t = hg.Table.build(from_np_u(a), 512, with_index=False)
    path = tmp_path / "t.hgt"
    t.save(path)
    off = torch.empty(513, dtype=torch.int32, device="cuda")
    keys = torch.empty(1000, dtype=torch.int64, device="cuda")
    idx = torch.empty(1000, dtype=torch.int32, device="cuda")
    P = ctypes.c_void_p
    s = P(torch.cuda.current_stream().cuda_stream)
    L = hg.lib()
    assert L.hg_table_load_arrays(str(path).encode(), P(off.data_ptr()), P(keys.data_ptr()), P(idx.data_ptr()),
                                  1000, 512, 8, s) == -1
    assert L.hg_table_load_arrays(str(path).encode(), P(off.data_ptr()), P(keys.data_ptr()), None,
                                  1000, 512, 8, s) == 0
    np.testing.assert_array_equal(to_np_u(off, 4), to_np_u(t.offsets, 4))
