"""Build + intersect over batches that live in host memory, pipelined.

A batch is a set of keys and a set of queries in pinned host memory.  For each
batch, `HostPipeline.run` builds the table of the keys on the device, probes
the queries against it and brings the match count and the pairs back to host
memory.  Three CUDA streams overlap batch k+1's upload (host to device),
batch k's build + probe, and batch k-1's pair download (device to host).  The
two copy directions use separate copy engines, so a run of batches proceeds
at the upload's pace: on a B200 the upload (PCIe) is about eight times slower
than the build + probe of the same keys.

The reference has no host-side batching (its test copies each input to the
GPU once, test/MultiHashGraphTest.cu:80-125); this is the host half of the
build + intersect path for callers whose keys arrive in host memory.
"""
from __future__ import annotations

import ctypes

from . import PATH_AUTO, HGError, Table, _key_bytes, check, intersect_workspace_bytes, lib


class HostPipeline:
    """Device buffers and streams for batches of at most `n` keys and `nq`
    queries (key width `key_bytes`), tables of `n_buckets` buckets, up to
    `pair_cap` pairs per batch (default nq)."""

    def __init__(self, n: int, nq: int, n_buckets: int, key_bytes: int = 8, with_index: bool = False,
                 emit: bool = True, pair_cap: int | None = None, device=None, build_path: int = PATH_AUTO,
                 probe_path: int = PATH_AUTO):
        import torch
        self.device = torch.device(device or "cuda")
        self.n, self.nq, self.n_buckets, self.key_bytes = int(n), int(nq), int(n_buckets), int(key_bytes)
        self.emit = emit
        self.pair_cap = int(nq if pair_cap is None else pair_cap) if emit else 0
        self.probe_path = probe_path
        kdt = torch.int32 if key_bytes == 4 else torch.int64
        dev = self.device
        self.d_keys = [torch.empty(max(self.n, 1), dtype=kdt, device=dev) for _ in range(2)]
        self.d_q = [torch.empty(max(self.nq, 1), dtype=kdt, device=dev) for _ in range(2)]
        self.table = Table(self.n_buckets, key_bytes, with_index, self.n, dev, build_path)
        self.table.n = self.n  # the probe workspace is planned for a full batch
        self.ws = torch.empty(max(intersect_workspace_bytes(self.table, self.nq, emit, probe_path), 1),
                              dtype=torch.uint8, device=dev)
        self.pairs = ([torch.empty((max(self.pair_cap, 1), 2), dtype=torch.int32, device=dev) for _ in range(2)]
                      if emit else [None, None])
        self.count = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(2)]
        self.h_count = [torch.zeros(1, dtype=torch.int64, pin_memory=True) for _ in range(2)]
        self.s_in = torch.cuda.Stream(dev)
        self.s_comp = torch.cuda.Stream(dev)
        self.s_out = torch.cuda.Stream(dev)
        mk = lambda: [torch.cuda.Event() for _ in range(2)]  # noqa: E731
        self.ev_in, self.ev_free, self.ev_cnt, self.ev_out = mk(), mk(), mk(), mk()
        torch.cuda.synchronize(dev)

    def _check_batch(self, h_keys, h_q):
        for t, cap, name in ((h_keys, self.n, "keys"), (h_q, self.nq, "queries")):
            if t.is_cuda or (t.numel() and not t.is_pinned()):  # an empty tensor has no storage to pin
                raise HGError(-1, f"{name} must be a pinned host tensor")
            if t.numel() > cap:
                raise HGError(-6, f"{t.numel()} {name} exceed the pipeline's {cap}")
            if _key_bytes(t) != self.key_bytes:
                raise HGError(-8, f"{name} key width differs from the pipeline's")

    def run(self, batches, h_pairs=None, start_event=None, end_event=None) -> list[int]:
        """Builds + probes every (h_keys, h_queries) batch; returns the match
        counts.  h_pairs[k] (a pinned int32 [>= pair_cap, 2] tensor, or None)
        receives batch k's first min(count, pair_cap) pairs.  start_event /
        end_event (optional CUDA events) are recorded before the first upload
        and after the last download."""
        import torch
        batches = list(batches)
        for hk, hq in batches:
            self._check_batch(hk, hq)
        h_pairs = list(h_pairs) if h_pairs is not None else [None] * len(batches)
        L = lib()
        counts = [0] * len(batches)
        if start_event is not None:
            start_event.record(self.s_in)

        def download(k):
            b = k & 1
            self.ev_cnt[b].synchronize()
            c = int(self.h_count[b].item())
            counts[k] = c
            m = min(c, self.pair_cap)
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(self.ev_cnt[b])
                if self.emit and m and h_pairs[k] is not None:
                    h_pairs[k][:m].copy_(self.pairs[b][:m], non_blocking=True)
                self.ev_out[b].record(self.s_out)

        for k, (hk, hq) in enumerate(batches):
            b = k & 1
            na, nq = hk.numel(), hq.numel()
            with torch.cuda.stream(self.s_in):
                if k >= 2:
                    self.s_in.wait_event(self.ev_free[b])  # batch k-2 is done with these buffers
                if na:
                    self.d_keys[b][:na].copy_(hk, non_blocking=True)
                if nq:
                    self.d_q[b][:nq].copy_(hq, non_blocking=True)
                self.ev_in[b].record(self.s_in)
            s = self.s_comp
            s.wait_event(self.ev_in[b])
            if k >= 2:
                s.wait_event(self.ev_out[b])  # batch k-2's pairs are downloaded
            sptr = ctypes.c_void_p(s.cuda_stream)
            self.table.rebuild(self.d_keys[b][:na], s)
            t = self.table
            pairs = self.pairs[b]
            check(L.hg_intersect_into_path(
                ctypes.c_void_p(t.offsets.data_ptr()), ctypes.c_void_p(t.keys.data_ptr()),
                ctypes.c_void_p(t.idx.data_ptr()) if t.idx is not None else None, t.n, t.n_buckets,
                self.key_bytes, ctypes.c_void_p(self.d_q[b].data_ptr()), nq, None,
                ctypes.c_void_p(pairs.data_ptr()) if self.emit else None, self.pair_cap,
                ctypes.c_void_p(self.count[b].data_ptr()), ctypes.c_void_p(self.ws.data_ptr()), self.ws.numel(),
                self.probe_path, sptr), "hg_intersect_into")
            self.ev_free[b].record(s)
            with torch.cuda.stream(s):
                self.h_count[b].copy_(self.count[b], non_blocking=True)
                self.ev_cnt[b].record(s)
            if k >= 1:
                download(k - 1)
        if batches:
            download(len(batches) - 1)
        if end_event is not None:
            self.s_out.wait_stream(self.s_comp)
            end_event.record(self.s_out)
        self.s_out.synchronize()
        return counts
