"""GPU parity of the sharding kernels (hg_shard_*) and of a sharded table.

* hg_shard_route equals a stable partition by destination shard (bit-exact:
  keys, global indices, group sizes); hg_shard_histogram equals a bincount.
* G shards built one after another on one device from the routed keys (each
  with its own range, no collective): every shard equals the global oracle
  table restricted to its range, for the direct and the partitioned build,
  aligned power-of-two ranges (mask form) and unaligned ones (remainder form
  minus the range start); each shard's probe of its routed queries gives the
  global oracle's pairs in its range, for both probe paths.
* ShardedTable over an NCCL group of one rank gives the plain table's result.
"""
import socket

import numpy as np
import pytest

import oracle
from tests.conftest import from_np_u, to_np_u
from tests.test_shard_cpu import CpuShardOps, _from_np, _to_np

pytestmark = pytest.mark.gpu


def _key(p):
    p = np.asarray(p).view(np.uint32).reshape(-1, 2).astype(np.uint64)
    return np.sort(p[:, 0] << np.uint64(32) | p[:, 1])


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("n", [0, 1, 4095, 4097, 100_003])
@pytest.mark.parametrize("G", [1, 3, 8, 64])
def test_route_matches_stable_partition(hg, kb, n, G):
    from hashgraph_b200.shard import DeviceShardOps
    rng = np.random.default_rng(n + G + kb)
    B = 1_000_003 if G % 2 else 1 << 20
    inner = np.sort(rng.integers(0, B, size=G - 1))
    if G >= 8:
        inner[2] = inner[1]  # an empty range
    splits = [0] + [int(x) for x in inner] + [B]
    k = oracle.gen_uniform(n, kb, 500 + n)
    dev = DeviceShardOps()
    out, idx, counts = dev.route(from_np_u(k), B, splits, 12345, True)
    ref_out, ref_idx, ref_counts = CpuShardOps().route(_from_np(k), B, splits, 12345, True)
    assert counts == ref_counts
    np.testing.assert_array_equal(to_np_u(out, kb), _to_np(ref_out))
    np.testing.assert_array_equal(to_np_u(idx, 4), _to_np(ref_idx))
    out2, idx2, _ = dev.route(from_np_u(k), B, splits, 0, False)
    assert idx2 is None
    np.testing.assert_array_equal(to_np_u(out2, kb), _to_np(ref_out))


@pytest.mark.parametrize("n_bins", [7, 16000, 32768])
def test_histogram_matches_bincount(hg, n_bins):
    from hashgraph_b200.shard import DeviceShardOps
    k = oracle.gen_uniform(300_000, 8, 77)
    for B in (1 << 22, 999_983, 1000):  # 1000 < n_bins: bin width 1
        got = DeviceShardOps().histogram(from_np_u(k), B, n_bins).cpu().numpy()
        ref = CpuShardOps().histogram(_from_np(k), B, n_bins).numpy()
        np.testing.assert_array_equal(got, ref)


def _check_shard(part, off, k, idx, lo, hi, kb):
    exp_off = (off[lo:hi + 1] - off[lo]).astype(np.uint32)
    np.testing.assert_array_equal(to_np_u(part.offsets, 4), exp_off)
    ek, ei = oracle.canonicalize(exp_off, k[off[lo]:off[hi]].copy(), idx[off[lo]:off[hi]].copy())
    gk, gi = oracle.canonicalize(exp_off, to_np_u(part.keys[: part.n], kb).copy(), to_np_u(part.idx[: part.n], 4).copy())
    np.testing.assert_array_equal(gk, ek)
    np.testing.assert_array_equal(gi, ei)


@pytest.mark.parametrize("case", ["pow2_aligned", "pow2_balanced", "odd_buckets"])
@pytest.mark.parametrize("path,probe_path", [(0, 0), (1, 1), (1, 2)])
def test_emulated_shards_equal_global_table(hg, case, path, probe_path):
    import torch
    from hashgraph_b200.shard import DeviceShardOps, shard_splits
    kb, G = 8, 4
    n = 1 << 21
    B = {"pow2_aligned": 1 << 21, "pow2_balanced": 1 << 21, "odd_buckets": 2_000_003}[case]
    A = oracle.gen_uniform(n, kb, 91)
    Q = oracle.gen_overlap(n // 2, A, 0.4, 92)
    dev = DeviceShardOps(path=path, probe_path=probe_path)
    dA, dQ = from_np_u(A), from_np_u(Q)
    if case == "pow2_aligned":
        splits = [r * (B // G) for r in range(G + 1)]
    else:
        splits = shard_splits(dev.histogram(dA, B, 16000).cpu().numpy(), B, G)
    ra, ria, ca = dev.route(dA, B, splits, 0, True)
    rq, riq, cq = dev.route(dQ, B, splits, 0, True)
    off, k, idx = oracle.build(A, B, True)
    c_all, pairs = oracle.intersect(off, k, idx, Q, pair_cap=4 * Q.size)
    b = oracle.buckets(A, B)
    total = 0
    sa = np.concatenate([[0], np.cumsum(ca)])
    sq = np.concatenate([[0], np.cumsum(cq)])
    for r in range(G):
        lo, hi = splits[r], splits[r + 1]
        part = dev.build(ra[sa[r]:sa[r + 1]], ria[sa[r]:sa[r + 1]], B, lo, hi, True)
        torch.cuda.synchronize()
        _check_shard(part, off, k, idx, lo, hi, kb)
        nq = int(cq[r])
        count, pr = dev.intersect(part, B, rq[sq[r]:sq[r + 1]], riq[sq[r]:sq[r + 1]], max(4 * nq, 1))
        c = int(count.item())
        mine = pairs[(b[pairs[:, 0]] >= lo) & (b[pairs[:, 0]] < hi)]
        assert c == mine.shape[0]
        np.testing.assert_array_equal(_key(to_np_u(pr[:c], 4)), _key(mine))
        total += c
    assert total == c_all
    assert hg.device_error() == 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_sharded_table_over_nccl_one_rank(hg):
    """The collective path end to end on one GPU: histogram, all-reduce,
    route, all-to-all (to itself), shard build, probe, all-reduce."""
    import torch
    import torch.distributed as dist
    from hashgraph_b200.shard import ShardedTable
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        A = oracle.gen_uniform(300_000, 8, 5)
        Q = oracle.gen_overlap(200_000, A, 0.3, 6)
        t = ShardedTable.build(from_np_u(A), 262_139, with_index=True)
        assert t.splits == [0, 262_139]
        off, k, idx = oracle.build(A, 262_139, True)
        _check_shard(t.part, off, k, idx, 0, 262_139, 8)
        res = t.intersect(from_np_u(Q))
        c, pairs = oracle.intersect(off, k, idx, Q, pair_cap=4 * Q.size)
        assert res.count == c == res.local_count
        np.testing.assert_array_equal(_key(to_np_u(res.pairs, 4)), _key(pairs))
    finally:
        dist.destroy_process_group()
    assert hg.device_error() == 0
