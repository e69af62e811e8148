"""One table sharded over the ranks of a process group by bucket range: the
multi-device MultiHashGraph (build src/MultiHashGraph.cu:408-629, intersect
:631-740) with one process per GPU and the key exchange as an all-to-all of
the group (NCCL over NVLink between GPUs).

Build (every rank calls it with its own keys):
  1. the bucket ids of the local keys are histogrammed into n_bins bins
     (hg_shard_histogram) and the histograms summed over the group
     (all-reduce) -- the reference's countBinSizes + host sum;
  2. every rank derives the same split points from the sum (hg_shard_splits);
  3. the local keys are grouped by destination shard with their global
     indices (hg_shard_route) -- countKeyBuffSizes + binKeyValues;
  4. the group sizes go round (all-to-all), then the keys and the indices
     (all-to-all with those sizes) -- the reference's peer copies;
  5. rank r builds shard r of the table over buckets [splits[r], splits[r+1])
     (hg_shard_build_into; no decrHash pass: the range's bucket map does it).
Intersect routes the queries by the same splits, exchanges them, probes the
shard (hg_shard_intersect_into) and sums the counts (all-reduce).  Pairs
(a's global index, query's global index) stay on the rank that found them,
as the reference keeps each GPU's output on that GPU.  A second table built
with the first one's splits (`splits=`, the reference's build(false, tid))
intersects shard by shard without an exchange (`intersect_table`).

The device steps go through an `ops` object; `DeviceShardOps`, the default,
calls the C ABI on the rank's GPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import PATH_AUTO, HGError, _check_cuda, _key_bytes, _ptr, _stream, check, lib

DEFAULT_BINS = 16000  # the reference's default binCount (test/MultiHashGraphTest.cu:145)


def shard_splits(bins, n_buckets: int, n_shards: int) -> list[int]:
    """Split points [n_shards + 1] from a summed bin histogram (host, no
    device): hg_shard_splits."""
    import numpy as np
    h = np.ascontiguousarray(np.asarray(bins, dtype=np.uint64))
    out = np.zeros(n_shards + 1, dtype=np.uint64)
    check(lib().hg_shard_splits(h.ctypes.data_as(ctypes.c_void_p), h.size, int(n_buckets), int(n_shards),
                                out.ctypes.data_as(ctypes.c_void_p)), "hg_shard_splits")
    return [int(x) for x in out]


@dataclass
class ShardPart:
    """A shard's table: buckets [lo, hi) of a table of n_buckets; `offsets`
    has hi - lo + 1 entries, `idx` the keys' global indices (or None)."""
    offsets: object
    keys: object
    idx: object
    n: int
    lo: int
    hi: int


class DeviceShardOps:
    """The device steps of a sharded build / intersect on one GPU, through the
    C ABI (hg_shard_*)."""

    def __init__(self, device=None, path: int = PATH_AUTO, probe_path: int | None = None):
        import torch
        self.device = torch.device(device or "cuda")
        self.path = path  # the build's path
        self.probe_path = path if probe_path is None else probe_path

    def histogram(self, keys, n_buckets: int, n_bins: int):
        import torch
        _check_cuda(keys, "keys")
        bins = torch.zeros(n_bins, dtype=torch.int64, device=self.device)
        check(lib().hg_shard_histogram(_ptr(keys), keys.numel(), _key_bytes(keys), int(n_buckets), int(n_bins),
                                       _ptr(bins), _stream()), "hg_shard_histogram")
        return bins

    def route(self, keys, n_buckets: int, splits: list[int], index_base: int, with_index: bool):
        """(keys grouped by shard, their global indices or None, group sizes)."""
        import numpy as np
        import torch
        _check_cuda(keys, "keys")
        n, G = keys.numel(), len(splits) - 1
        ws_bytes = ctypes.c_size_t(0)
        check(lib().hg_shard_route_workspace_size(n, G, ctypes.byref(ws_bytes)), "hg_shard_route_workspace_size")
        ws = torch.empty(max(ws_bytes.value, 1), dtype=torch.uint8, device=self.device)
        out = torch.empty_like(keys)
        idx = torch.empty(n, dtype=torch.int32, device=self.device) if with_index else None
        offs = torch.empty(G + 1, dtype=torch.int64, device=self.device)
        sp = np.asarray(splits, dtype=np.uint64)
        check(lib().hg_shard_route(_ptr(keys), n, _key_bytes(keys), int(n_buckets),
                                   sp.ctypes.data_as(ctypes.c_void_p), G, int(index_base), _ptr(out), _ptr(idx),
                                   _ptr(offs), _ptr(ws), ws.numel(), _stream()), "hg_shard_route")
        o = offs.cpu().tolist()
        return out, idx, [o[r + 1] - o[r] for r in range(G)]

    def build(self, keys, key_idx, n_buckets: int, lo: int, hi: int, with_index: bool) -> ShardPart:
        import torch
        from . import build_workspace_bytes
        n, kb = keys.numel(), _key_bytes(keys)
        offsets = torch.empty(hi - lo + 1, dtype=torch.int32, device=self.device)
        out = torch.empty(max(n, 1), dtype=keys.dtype, device=self.device)
        idx = torch.empty(max(n, 1), dtype=torch.int32, device=self.device) if with_index else None
        ws = torch.empty(max(build_workspace_bytes(n, kb, hi - lo, with_index, self.path), 1), dtype=torch.uint8,
                         device=self.device)
        check(lib().hg_shard_build_into_path(_ptr(keys), _ptr(key_idx), n, kb, int(n_buckets), int(lo), int(hi),
                                             _ptr(offsets), _ptr(out), _ptr(idx), _ptr(ws), ws.numel(), self.path,
                                             _stream()), "hg_shard_build_into")
        return ShardPart(offsets, out, idx, n, lo, hi)

    def intersect(self, part: ShardPart, n_buckets: int, queries, query_idx, pair_cap: int, emit: bool = True):
        """(count: 1-element int64 tensor, pairs [pair_cap, 2] int32 or None)."""
        import torch
        nq, kb = queries.numel(), _key_bytes(queries)
        out = ctypes.c_size_t(0)
        check(lib().hg_intersect_workspace_size_path(part.n, int(part.idx is not None), part.hi - part.lo, nq, kb,
                                                     int(emit), self.probe_path, ctypes.byref(out)),
              "intersect workspace")
        ws = torch.empty(max(out.value, 1), dtype=torch.uint8, device=self.device)
        count = torch.empty(1, dtype=torch.int64, device=self.device)
        pairs = torch.empty((max(int(pair_cap), 1), 2), dtype=torch.int32, device=self.device) if emit else None
        check(lib().hg_shard_intersect_into_path(
            _ptr(part.offsets), _ptr(part.keys), _ptr(part.idx), part.n, int(n_buckets), part.lo, part.hi, kb,
            _ptr(queries), nq, _ptr(query_idx), _ptr(pairs), int(pair_cap) if emit else 0, _ptr(count), _ptr(ws),
            ws.numel(), self.probe_path, _stream()), "hg_shard_intersect_into")
        return count, pairs

    def empty_keys(self, n: int, like):
        import torch
        return torch.empty(n, dtype=like.dtype, device=self.device)

    def empty_idx(self, n: int):
        import torch
        return torch.empty(n, dtype=torch.int32, device=self.device)


@dataclass
class ShardedResult:
    count: int          # matches over all shards
    local_count: int    # matches found on this rank
    pairs: object       # this rank's (a global index, query global index) rows, or None


def _dist():
    import torch.distributed as dist
    return dist


def _all_gather_int(v: int, device, group) -> list[int]:
    import torch
    dist = _dist()
    world = dist.get_world_size(group)
    t = torch.tensor([v], dtype=torch.int64, device=device)
    out = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    return [int(x.item()) for x in out]


def _exchange(ops, send, send_counts: list[int], device, group, make_recv):
    """All-to-all of `send` (grouped by destination, send_counts[r] rows for
    rank r); returns (received rows grouped by source, recv_counts)."""
    import torch
    dist = _dist()
    sc = torch.tensor(send_counts, dtype=torch.int64, device=device)
    rc = torch.empty_like(sc)
    dist.all_to_all_single(rc, sc, group=group)
    recv_counts = [int(x) for x in rc.cpu().tolist()]
    recv = make_recv(sum(recv_counts))
    dist.all_to_all_single(recv, send, recv_counts, send_counts, group=group)
    return recv, recv_counts


class ShardedTable:
    """Shard `rank` of a table of n_buckets sharded over the ranks of `group`."""

    def __init__(self, part: ShardPart, splits: list[int], n_buckets: int, key_bytes: int, with_index: bool,
                 n_total: int, ops, group):
        self.part, self.splits, self.n_buckets = part, splits, int(n_buckets)
        self.key_bytes, self.with_index, self.n_total = key_bytes, with_index, n_total
        self.ops, self.group = ops, group

    @classmethod
    def build(cls, keys, n_buckets: int, with_index: bool = True, n_bins: int = DEFAULT_BINS, splits=None,
              group=None, ops=None) -> "ShardedTable":
        """Collective: every rank of `group` passes its own keys."""
        dist = _dist()
        ops = ops or DeviceShardOps(keys.device)
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        counts = _all_gather_int(keys.numel(), ops.device, group)
        n_total, index_base = sum(counts), sum(counts[:rank])
        if with_index and n_total >= (1 << 32):
            raise HGError(-6, "a sharded table with an index holds fewer than 2^32 keys in all")
        if splits is None:
            bins = ops.histogram(keys, n_buckets, n_bins)
            dist.all_reduce(bins, group=group)
            splits = shard_splits(bins.cpu().numpy().astype("uint64"), n_buckets, world)
        if len(splits) != world + 1:
            raise HGError(-1, f"{len(splits) - 1} shards for {world} ranks")
        routed, ridx, send = ops.route(keys, n_buckets, splits, index_base, with_index)
        rkeys, _ = _exchange(ops, routed, send, ops.device, group, lambda m: ops.empty_keys(m, keys))
        rid = None
        if with_index:
            rid, _ = _exchange(ops, ridx, send, ops.device, group, ops.empty_idx)
        lo, hi = splits[rank], splits[rank + 1]
        if hi > lo:
            part = ops.build(rkeys, rid, n_buckets, lo, hi, with_index)
        else:  # an empty range holds no bucket
            part = ShardPart(None, rkeys[:0], None if rid is None else rid[:0], 0, lo, hi)
        return cls(part, list(splits), n_buckets, _key_bytes(keys), with_index, n_total, ops, group)

    def _probe(self, queries, qidx, pair_cap, emit):
        import torch
        if self.part.hi == self.part.lo or queries.numel() == 0:
            z = torch.zeros(1, dtype=torch.int64, device=self.ops.device)
            return z, (queries.new_zeros((0, 2), dtype=torch.int32) if emit else None)
        return self.ops.intersect(self.part, self.n_buckets, queries, qidx, pair_cap, emit)

    def _finish(self, count, pairs, pair_cap) -> ShardedResult:
        dist = _dist()
        local = count.clone()
        dist.all_reduce(count, group=self.group)
        lc = int(local.item())
        rows = None if pairs is None else pairs[: min(lc, pair_cap)]
        return ShardedResult(int(count.item()), lc, rows)

    def intersect(self, queries, pair_cap: int | None = None, emit: bool = True) -> ShardedResult:
        """Collective: every rank passes its own queries; the queries' global
        indices follow the rank order, as the keys' do."""
        dist = _dist()
        if _key_bytes(queries) != self.key_bytes:
            raise HGError(-8, "query key width differs from the table's")
        rank = dist.get_rank(self.group)
        counts = _all_gather_int(queries.numel(), self.ops.device, self.group)
        base = sum(counts[:rank])
        if sum(counts) >= (1 << 32):
            raise HGError(-6, "fewer than 2^32 queries in all")
        routed, ridx, send = self.ops.route(queries, self.n_buckets, self.splits, base, True)
        rq, _ = _exchange(self.ops, routed, send, self.ops.device, self.group,
                          lambda m: self.ops.empty_keys(m, queries))
        rid, _ = _exchange(self.ops, ridx, send, self.ops.device, self.group, self.ops.empty_idx)
        cap = rq.numel() if pair_cap is None else int(pair_cap)
        count, pairs = self._probe(rq, rid, cap, emit)
        return self._finish(count, pairs, cap)

    def intersect_table(self, other: "ShardedTable", pair_cap: int | None = None,
                        emit: bool = True) -> ShardedResult:
        """Shard-by-shard intersect with a table built on the same splits (the
        reference's MultiHashGraph::intersect of two tables, the second built
        with build(false, tid)); q_ref is `other`'s global index."""
        if other.splits != self.splits or other.n_buckets != self.n_buckets:
            raise HGError(-1, "intersect_table needs two tables on the same splits")
        if not other.with_index:
            raise HGError(-1, "intersect_table needs the other table's global indices (with_index)")
        q = other.part.keys[: other.part.n]
        qidx = other.part.idx[: other.part.n] if other.part.idx is not None else None
        cap = other.part.n if pair_cap is None else int(pair_cap)
        count, pairs = self._probe(q, qidx, cap, emit)
        return self._finish(count, pairs, cap)
