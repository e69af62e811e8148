"""Host logic of the sharded table (hashgraph_b200.shard) on CPU.

* The split rule (hg_shard_splits, host code of the library) on hand-worked
  histograms of the reference's rule (include/MultiHashGraphHostOperators.cuh:80-88).
* A sharded build + intersect over two gloo ranks whose device steps are done
  by numpy and the oracle's hash (CpuShardOps, test infrastructure): each
  shard must equal the global oracle table restricted to its bucket range
  (offsets rebased, canonical buckets, global indices), and the pairs found
  over all ranks the global oracle's pairs.
"""
import os
import socket

import numpy as np
import pytest

import oracle


def _to_np(t):
    a = t.detach().cpu().numpy()
    return a.view(np.uint32 if a.dtype == np.int32 else np.uint64)


def _from_np(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32 if a.dtype == np.uint32 else np.int64).copy())


class CpuShardOps:
    """The device steps of hashgraph_b200.shard restated on the CPU."""

    def __init__(self):
        import torch
        self.device = torch.device("cpu")

    def histogram(self, keys, n_buckets, n_bins):
        import torch
        b = oracle.buckets(_to_np(keys), n_buckets).astype(np.int64)
        width = -(-n_buckets // n_bins)
        return torch.from_numpy(np.bincount(b // width, minlength=n_bins).astype(np.int64))

    def route(self, keys, n_buckets, splits, index_base, with_index):
        import torch
        k = _to_np(keys)
        b = oracle.buckets(k, n_buckets).astype(np.int64)
        G = len(splits) - 1
        dest = np.searchsorted(np.asarray(splits, dtype=np.int64), b, side="right") - 1
        order = np.argsort(dest, kind="stable")
        idx = torch.from_numpy((index_base + order).astype(np.int64).astype(np.uint32).view(np.int32))
        return _from_np(k[order]), (idx if with_index else None), np.bincount(dest, minlength=G).tolist()

    def build(self, keys, key_idx, n_buckets, lo, hi, with_index):
        import torch
        from hashgraph_b200.shard import ShardPart
        k = _to_np(keys)
        local = oracle.buckets(k, n_buckets).astype(np.int64) - lo
        assert k.size == 0 or (local.min() >= 0 and local.max() < hi - lo)
        order = np.argsort(local, kind="stable")
        off = np.concatenate([[0], np.cumsum(np.bincount(local, minlength=hi - lo))]).astype(np.uint32)
        idx = None
        if with_index:
            src = _to_np(key_idx) if key_idx is not None else np.arange(k.size, dtype=np.uint32)
            idx = _from_np(src[order].astype(np.uint32))
        return ShardPart(torch.from_numpy(off.view(np.int32)), _from_np(k[order]), idx, k.size, lo, hi)

    def intersect(self, part, n_buckets, queries, query_idx, pair_cap, emit=True):
        import torch
        a = _to_np(part.keys)[: part.n]
        aref = _to_np(part.idx)[: part.n] if part.idx is not None else np.arange(part.n, dtype=np.uint32)
        q = _to_np(queries)
        qref = _to_np(query_idx) if query_idx is not None else np.arange(q.size, dtype=np.uint32)
        ao = np.argsort(a, kind="stable")
        sa = a[ao]
        lo = np.searchsorted(sa, q, side="left")
        cnt = np.searchsorted(sa, q, side="right") - lo
        total = int(cnt.sum())
        qi = np.repeat(np.arange(q.size), cnt)
        start = np.repeat(lo - np.concatenate([[0], np.cumsum(cnt)[:-1]]), cnt) if q.size else np.zeros(0, np.int64)
        apos = start + np.arange(total)
        pairs = np.stack([aref[ao[apos]], qref[qi]], axis=1).astype(np.uint32)[:pair_cap]
        return torch.tensor([total], dtype=torch.int64), torch.from_numpy(pairs.view(np.int32).copy())

    def empty_keys(self, n, like):
        import torch
        return torch.empty(n, dtype=like.dtype)

    def empty_idx(self, n):
        import torch
        return torch.empty(n, dtype=torch.int32)


def test_splits_rule():
    from hashgraph_b200.shard import shard_splits
    # bins [5, 0, 0, 5], B = 8 (width 2), two shards: avg 5, ps = [0, 5, 5, 5, 10];
    # the search for 5 meets ps[2] first -> split 2 * 2 = 4
    assert shard_splits([5, 0, 0, 5], 8, 2) == [0, 4, 8]
    # uniform bins: equal ranges
    assert shard_splits([10] * 16, 1 << 20, 4) == [0, 1 << 18, 1 << 19, 3 << 18, 1 << 20]
    # everything in one bin: the other shards get empty ranges
    s = shard_splits([0, 0, 100, 0], 400, 3)
    assert s[0] == 0 and s[-1] == 400 and all(x <= y for x, y in zip(s, s[1:]))
    # top bins empty: the last split is still B
    assert shard_splits([4, 4, 0, 0], 40, 2)[-1] == 40
    # no keys at all, one shard, more shards than bins
    assert shard_splits([0] * 8, 64, 3)[-1] == 64
    assert shard_splits([7], 10, 1) == [0, 10]
    s = shard_splits([1, 1], 2, 8)
    assert len(s) == 9 and s[-1] == 2


def test_splits_argument_checks():
    from hashgraph_b200 import HGError
    from hashgraph_b200.shard import shard_splits
    with pytest.raises(HGError):
        shard_splits([1, 2], 10, 0)
    with pytest.raises(HGError):
        shard_splits([1, 2], 10, 65)
    with pytest.raises(HGError):
        shard_splits([1] * 40000, 1 << 20, 2)


def test_cpu_ops_build_equals_global():
    """The CPU stand-in itself: one shard over the whole range is the oracle's table."""
    k = oracle.gen_uniform(3000, 8, 5)
    ops = CpuShardOps()
    part = ops.build(_from_np(k), None, 1000, 0, 1000, True)
    off, kk, ii = oracle.build(k, 1000, True)
    np.testing.assert_array_equal(_to_np(part.offsets).view(np.uint32), off)
    np.testing.assert_array_equal(_to_np(part.keys), kk)
    np.testing.assert_array_equal(_to_np(part.idx), ii)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


N_PER_RANK = [2500, 1700]
NQ_PER_RANK = [1900, 2600]


def _rank_keys(kb, r):
    return oracle.gen_uniform(N_PER_RANK[r], kb, 40 + r)


def _rank_queries(kb, r, all_keys):
    return oracle.gen_overlap(NQ_PER_RANK[r], all_keys, 0.5, 60 + r)


def _worker(rank, world, port, kb, n_buckets, n_bins):
    import torch.distributed as dist

    from hashgraph_b200.shard import ShardedTable
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ops = CpuShardOps()
        A = np.concatenate([_rank_keys(kb, r) for r in range(world)])
        Q = np.concatenate([_rank_queries(kb, r, A) for r in range(world)])
        t = ShardedTable.build(_from_np(_rank_keys(kb, rank)), n_buckets, with_index=True, n_bins=n_bins, ops=ops)
        lo, hi = t.splits[rank], t.splits[rank + 1]
        assert t.n_total == A.size
        off, k, idx = oracle.build(A, n_buckets, True)
        # the shard is the global table restricted to [lo, hi)
        exp_off = (off[lo:hi + 1] - off[lo]).astype(np.uint32)
        got_off = _to_np(t.part.offsets).view(np.uint32) if hi > lo else np.zeros(1, np.uint32)
        np.testing.assert_array_equal(got_off, exp_off)
        ek, ei = oracle.canonicalize(exp_off, k[off[lo]:off[hi]].copy(), idx[off[lo]:off[hi]].copy())
        gk, gi = oracle.canonicalize(exp_off, _to_np(t.part.keys)[: t.part.n].copy(),
                                     _to_np(t.part.idx)[: t.part.n].copy() if t.part.n else np.zeros(0, np.uint32))
        np.testing.assert_array_equal(gk, ek)
        np.testing.assert_array_equal(gi, ei)
        # every shard non-empty for uniform keys, and the ranges are balanced
        assert hi > lo and abs(t.part.n - A.size / world) < 0.2 * A.size
        # intersect: the count over all shards and this shard's pairs
        c, pairs = oracle.intersect(off, k, idx, Q, pair_cap=4 * Q.size)
        res = t.intersect(_from_np(_rank_queries(kb, rank, A)))
        assert res.count == c
        b = oracle.buckets(A, n_buckets)
        mine = pairs[(b[pairs[:, 0]] >= lo) & (b[pairs[:, 0]] < hi)]
        assert res.local_count == mine.shape[0]
        got = np.sort(_to_np(res.pairs).view(np.uint32).reshape(-1, 2).astype(np.uint64) @ np.array([1 << 32, 1],
                                                                                                      np.uint64))
        exp = np.sort(mine.astype(np.uint64) @ np.array([1 << 32, 1], np.uint64))
        np.testing.assert_array_equal(got, exp)
        # the queries as a second table on the same splits: the same pairs
        tq = ShardedTable.build(_from_np(_rank_queries(kb, rank, A)), n_buckets, with_index=True, splits=t.splits,
                                ops=ops)
        res2 = t.intersect_table(tq)
        assert res2.count == c and res2.local_count == res.local_count
        got2 = np.sort(_to_np(res2.pairs).view(np.uint32).reshape(-1, 2).astype(np.uint64) @ np.array([1 << 32, 1],
                                                                                                        np.uint64))
        np.testing.assert_array_equal(got2, exp)
        # a rank with no keys still takes part in every collective
        empty = _from_np(np.zeros(0, dtype=A.dtype)) if rank == 1 else _from_np(_rank_keys(kb, rank))
        te = ShardedTable.build(empty, n_buckets, with_index=True, splits=t.splits, ops=ops)
        assert te.n_total == N_PER_RANK[0]
        re = te.intersect(_from_np(_rank_queries(kb, rank, A)))
        oe, ke, ie = oracle.build(_rank_keys(kb, 0), n_buckets, True)
        assert re.count == oracle.intersect(oe, ke, ie, Q)[0]
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kb,n_buckets", [(8, 4096), (4, 3000)])
def test_sharded_build_intersect_two_gloo_ranks(kb, n_buckets):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(2, _free_port(), kb, n_buckets, 64), nprocs=2, join=True,
                       start_method="spawn")
