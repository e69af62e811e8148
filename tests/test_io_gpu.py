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
