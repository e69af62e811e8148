"""hashgraph_b200 -- B200 (sm_100a) HashGraph build + intersect.

A HashGraph is a hash table stored as CSR: ``offsets[n_buckets+1]`` and the
keys binned by ``murmur3(low 32 bits of key) % n_buckets`` (optionally with the
input position of every key).  The compute runs in hand-written CUDA kernels
behind the C ABI of ``include/hashgraph_b200.h``; this module binds that ABI
with ctypes and uses torch only to own device memory and streams.  The
reference's C++ class API (SingleHashGraph / MultiHashGraph) is kept by the C++
wrappers in ``include/hashgraph_b200/``.
"""
from __future__ import annotations

import ctypes

from ._capi import (ERR_DEVICE_TIMEOUT, ERR_PAIR_CAPACITY, BatchPair, BatchParams, HGError, build_library,
                    check, lib, status_str)

__all__ = [
    "HGError", "Table", "build_library", "lib", "hash_keys", "intersect", "device_error",
    "gen_uniform", "gen_overlap", "gen_zipf", "zipf_cdf", "PATH_AUTO", "PATH_DIRECT",
    "PATH_PARTITIONED", "PATH_COARSE", "ERR_PAIR_CAPACITY", "ERR_DEVICE_TIMEOUT", "status_str",
    "profile_enable", "profile_read", "launch_count", "Batch",
]

PATH_AUTO, PATH_DIRECT, PATH_PARTITIONED = -1, 0, 1
PATH_COARSE = 2  # probes only: queries grouped by L2-sized bucket ranges, probed from L2


def _torch():
    import torch
    return torch


def _key_bytes(t) -> int:
    torch = _torch()
    if t.dtype in (torch.int32, torch.uint32):
        return 4
    if t.dtype in (torch.int64, torch.uint64):
        return 8
    raise TypeError(f"keys must be a 32- or 64-bit integer tensor, got {t.dtype}")


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _check_cuda(t, name):
    if t is not None and not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t is not None and not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def hash_keys(keys) -> list:
    """Host murmur3 (low 32 bits, seed 0) of python ints, via the C ABI."""
    return [int(lib().hg_hash(int(k) & 0xFFFFFFFFFFFFFFFF)) for k in keys]


def device_error(stream=None) -> int:
    """Synchronise the stream and read/clear the device error word."""
    code = ctypes.c_int32(0)
    check(lib().hg_device_error(_stream(stream), ctypes.byref(code)), "hg_device_error")
    return int(code.value)


def profile_enable(on: bool = True) -> None:
    """Per-phase CUDA-event timing inside the library (stream-ordered)."""
    check(lib().hg_profile_enable(int(on)), "hg_profile_enable")


def profile_read(cap: int = 4096) -> list:
    """[(phase name, ms)] recorded since the last read, in launch order."""
    names = (ctypes.c_char_p * cap)()
    ms = (ctypes.c_float * cap)()
    n = ctypes.c_int(0)
    check(lib().hg_profile_read(cap, ctypes.byref(n), names, ms), "hg_profile_read")
    return [(names[i].decode(), float(ms[i])) for i in range(min(n.value, cap))]


def launch_count() -> int:
    return int(lib().hg_launch_count())


def build_workspace_bytes(n: int, key_bytes: int, n_buckets: int, with_index: bool,
                          path: int = PATH_AUTO) -> int:
    out = ctypes.c_size_t(0)
    check(lib().hg_build_workspace_size_path(n, key_bytes, n_buckets, int(with_index), path,
                                             ctypes.byref(out)), "workspace size")
    return int(out.value)


class Table:
    """A built HashGraph whose arrays are torch CUDA tensors.

    ``offsets`` (int32 storage of uint32 values, n_buckets+1), ``keys``
    (int32/int64 storage of uint32/uint64 keys in CSR order) and ``idx``
    (int32 storage of uint32 input positions, or None).
    """

    def __init__(self, n_buckets: int, key_bytes: int, with_index: bool, capacity: int,
                 device=None, path: int = PATH_AUTO, workspace: bool = True):
        torch = _torch()
        self.device = torch.device(device or "cuda")
        self.n_buckets = int(n_buckets)
        self.key_bytes = int(key_bytes)
        self.with_index = bool(with_index)
        self.capacity = int(capacity)
        self.path = path
        self.n = 0
        kdt = torch.int32 if key_bytes == 4 else torch.int64
        self.offsets = torch.empty(self.n_buckets + 1, dtype=torch.int32, device=self.device)
        self.keys = torch.empty(max(self.capacity, 1), dtype=kdt, device=self.device)
        self.idx = (torch.empty(max(self.capacity, 1), dtype=torch.int32, device=self.device)
                    if with_index else None)
        # workspace=False: arrays only (the caller builds with its own workspace)
        ws = build_workspace_bytes(self.capacity, key_bytes, n_buckets, with_index, path) if workspace else 0
        self.workspace = torch.empty(max(ws, 1), dtype=torch.uint8, device=self.device)

    @classmethod
    def build(cls, keys, n_buckets: int, with_index: bool = False, path: int = PATH_AUTO,
              stream=None) -> "Table":
        _check_cuda(keys, "keys")
        t = cls(n_buckets, _key_bytes(keys), with_index, keys.numel(), keys.device, path)
        t.rebuild(keys, stream)
        return t

    def rebuild(self, keys, stream=None) -> "Table":
        """Rebuild in place from `keys` (numel <= capacity), stream-ordered."""
        _check_cuda(keys, "keys")
        if _key_bytes(keys) != self.key_bytes:
            raise HGError(-8, "key width differs from the table's")
        n = keys.numel()
        if n > self.capacity:
            raise HGError(-6, f"{n} keys exceed capacity {self.capacity}")
        check(lib().hg_build_into_path(
            _ptr(keys), n, self.key_bytes, self.n_buckets, _ptr(self.offsets), _ptr(self.keys),
            _ptr(self.idx), _ptr(self.workspace), self.workspace.numel(), self.path,
            _stream(stream)), "hg_build_into")
        self.n = n
        return self

    def save(self, path: str, stream=None) -> None:
        """Writes the built table to a table file (hg_table_save_arrays)."""
        check(lib().hg_table_save_arrays(str(path).encode(), _ptr(self.offsets), _ptr(self.keys),
                                         _ptr(self.idx), self.n, self.n_buckets, self.key_bytes,
                                         _stream(stream)), "hg_table_save")

    @classmethod
    def load(cls, path: str, device=None, stream=None) -> "Table":
        """Reads a table file onto `device` (hg_table_load_arrays)."""
        n, nb = ctypes.c_uint64(0), ctypes.c_uint64(0)
        kb, wi = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().hg_table_file_info(str(path).encode(), ctypes.byref(n), ctypes.byref(nb), ctypes.byref(kb),
                                       ctypes.byref(wi)), "hg_table_file_info")
        t = cls(nb.value, kb.value, bool(wi.value), n.value, device)
        check(lib().hg_table_load_arrays(str(path).encode(), _ptr(t.offsets), _ptr(t.keys), _ptr(t.idx),
                                         n.value, nb.value, kb.value, _stream(stream)), "hg_table_load")
        t.n = n.value
        return t

    def view_keys(self):
        return self.keys[: self.n]

    def view_idx(self):
        return None if self.idx is None else self.idx[: self.n]

    def intersect(self, queries, query_idx=None, emit: bool = True, pair_cap: int | None = None,
                  stream=None, path: int = PATH_AUTO):
        return intersect(self, queries, query_idx, emit, pair_cap, stream, path)


def intersect_workspace_bytes(a: "Table", nq: int, emit: bool, path: int = PATH_AUTO) -> int:
    out = ctypes.c_size_t(0)
    check(lib().hg_intersect_workspace_size_path(a.n, int(a.with_index), a.n_buckets, nq, a.key_bytes,
                                                 int(emit), path, ctypes.byref(out)), "intersect workspace")
    return int(out.value)


def intersect(a: Table, queries, query_idx=None, emit: bool = True, pair_cap: int | None = None,
              stream=None, path: int = PATH_AUTO):
    """Probe `queries` against table `a`.

    Returns (count, pairs): `count` a 1-element int64 CUDA tensor holding the
    exact number of matches; `pairs` an int32 CUDA tensor [pair_cap, 2] of
    (a_ref, q_ref) or None when emit is False.  Only min(count, pair_cap)
    rows are meaningful.
    """
    torch = _torch()
    _check_cuda(queries, "queries")
    if _key_bytes(queries) != a.key_bytes:
        raise HGError(-8, "query key width differs from the table's")
    nq = queries.numel()
    if pair_cap is None:
        pair_cap = nq
    ws = torch.empty(max(intersect_workspace_bytes(a, nq, emit, path), 1), dtype=torch.uint8,
                     device=a.device)
    count = torch.empty(1, dtype=torch.int64, device=a.device)
    pairs = torch.empty((max(int(pair_cap), 1), 2), dtype=torch.int32, device=a.device) if emit else None
    check(lib().hg_intersect_into_path(
        _ptr(a.offsets), _ptr(a.keys), _ptr(a.idx), a.n, a.n_buckets, a.key_bytes, _ptr(queries),
        nq, _ptr(query_idx), _ptr(pairs), int(pair_cap) if emit else 0, _ptr(count), _ptr(ws),
        ws.numel(), path, _stream(stream)), "hg_intersect_into")
    return count, pairs


class Batch:
    """Batched build + intersect of many (table, queries) pairs (hg_batch_*).

    ``keys[i]`` is built into a table of ``n_buckets[i]`` buckets (with the
    input positions when ``with_index[i]``) and ``queries[i]`` are probed
    against it.  The output tensors are allocated here and kept on the object:
    ``offsets[i]``, ``table_keys[i]``, ``table_idx[i]`` (or None),
    ``pairs[i]`` ([pair_caps[i], 2] int32, or None when emit is False) and
    ``counts`` (int64, one exact match count per pair).  ``run()`` launches
    the whole batch (a fixed sequence of kernels, capturable into a CUDA
    graph); the input tensors must stay alive and may be refilled between
    runs.  All pairs share one key width.
    """

    def __init__(self, keys, queries, n_buckets, with_index=False, pair_caps=None, emit=True,
                 stream=None, params=None):
        torch = _torch()
        n_pairs = len(keys)
        if len(queries) != n_pairs or len(n_buckets) != n_pairs:
            raise ValueError("keys, queries and n_buckets must have one entry per pair")
        if isinstance(with_index, bool):
            with_index = [with_index] * n_pairs
        if pair_caps is None:
            pair_caps = [q.numel() for q in queries]
        kb = _key_bytes(keys[0]) if n_pairs else 8
        self.key_bytes = kb
        self.keys, self.queries = list(keys), list(queries)
        dev = keys[0].device if n_pairs else torch.device("cuda")
        self.counts = torch.zeros(max(n_pairs, 1), dtype=torch.int64, device=dev)
        self.offsets, self.table_keys, self.table_idx, self.pairs = [], [], [], []
        descs = (BatchPair * max(n_pairs, 1))()
        for i in range(n_pairs):
            k, q = keys[i], queries[i]
            _check_cuda(k, "keys")
            _check_cuda(q, "queries")
            if _key_bytes(k) != kb or _key_bytes(q) != kb:
                raise HGError(-8, "all keys and queries of a batch share one width")
            B = int(n_buckets[i])
            off = torch.empty(B + 1, dtype=torch.int32, device=dev)
            tk = torch.empty(max(k.numel(), 1), dtype=k.dtype, device=dev)
            ti = torch.empty(max(k.numel(), 1), dtype=torch.int32, device=dev) if with_index[i] else None
            pr = torch.empty((max(int(pair_caps[i]), 1), 2), dtype=torch.int32, device=dev) if emit else None
            self.offsets.append(off)
            self.table_keys.append(tk)
            self.table_idx.append(ti)
            self.pairs.append(pr)
            d = descs[i]
            d.d_keys, d.n, d.n_buckets = k.data_ptr() if k.numel() else None, k.numel(), B
            d.d_query, d.nq = q.data_ptr() if q.numel() else None, q.numel()
            d.d_offsets, d.d_keys_out = off.data_ptr(), tk.data_ptr()
            d.d_idx_out = ti.data_ptr() if ti is not None else None
            d.d_pairs = pr.data_ptr() if pr is not None else None
            d.pair_cap = int(pair_caps[i]) if emit else 0
            d.d_count = self.counts.data_ptr() + 8 * i
        self.n_pairs = n_pairs
        self._descs = descs
        self._h = ctypes.c_void_p()
        self.params = dict(params) if params else None
        self._create(stream)

    def _create(self, stream=None):
        prm = None
        if self.params is not None:
            prm = BatchParams(int(self.params["part_min"]), int(self.params["l2_table_bytes"]))
        check(lib().hg_batch_create_params(self._descs, self.n_pairs, self.key_bytes,
                                           ctypes.byref(prm) if prm is not None else None, _stream(stream),
                                           ctypes.byref(self._h)), "hg_batch_create")

    def autotune(self, stream=None) -> tuple[dict, float]:
        """Times candidate size classes on this batch (hg_batch_autotune; the
        outputs then hold the batch's results), re-plans the batch with the
        fastest and returns (params, ms per run)."""
        best = BatchParams()
        ms = ctypes.c_float(0.0)
        check(lib().hg_batch_autotune(self._descs, self.n_pairs, self.key_bytes, _stream(stream),
                                      ctypes.byref(best), ctypes.byref(ms)), "hg_batch_autotune")
        self.free(stream)
        self.params = {"part_min": best.part_min, "l2_table_bytes": best.l2_table_bytes}
        self._create(stream)
        return dict(self.params), float(ms.value)

    def run(self, stream=None) -> "Batch":
        check(lib().hg_batch_run(self._h, _stream(stream)), "hg_batch_run")
        return self

    def device_bytes(self) -> int:
        out = ctypes.c_size_t(0)
        check(lib().hg_batch_device_bytes(self._h, ctypes.byref(out)), "hg_batch_device_bytes")
        return int(out.value)

    def free(self, stream=None) -> None:
        if self._h:
            lib().hg_batch_free(self._h, _stream(stream))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Workload generators (device)
# ---------------------------------------------------------------------------
def _empty_keys(n, key_bytes, device):
    torch = _torch()
    return torch.empty(max(n, 1), dtype=torch.int32 if key_bytes == 4 else torch.int64,
                       device=device)[:n]


def gen_uniform(n: int, key_bytes: int, seed: int, device="cuda", stream=None):
    out = _empty_keys(n, key_bytes, device)
    check(lib().hg_gen_uniform(_ptr(out), n, key_bytes, seed, _stream(stream)), "hg_gen_uniform")
    return out


def overlap_count(n: int, n_a: int, frac: float) -> int:
    """Number of keys drawn from A: round-half-away(frac * n), capped at n and n_a."""
    import math
    x = frac * n
    m = int(math.floor(x + 0.5)) if x >= 0 else 0
    return max(0, min(m, n, n_a))


def gen_overlap(n: int, a_keys, frac: float, seed: int, stream=None):
    kb = _key_bytes(a_keys)
    out = _empty_keys(n, kb, a_keys.device)
    m = overlap_count(n, a_keys.numel(), frac)
    check(lib().hg_gen_overlap(_ptr(out), n, kb, _ptr(a_keys), a_keys.numel(), m, seed,
                               _stream(stream)), "hg_gen_overlap")
    return out


def zipf_cdf(universe: int, s: float, device="cuda"):
    import numpy as np
    torch = _torch()
    cdf = np.empty(universe, dtype=np.uint64)
    check(lib().hg_zipf_cdf(cdf.ctypes.data_as(ctypes.c_void_p), universe, float(s)), "hg_zipf_cdf")
    return torch.from_numpy(cdf.view(np.int64)).to(device)


def gen_zipf(n: int, key_bytes: int, cdf, seed: int, stream=None):
    out = _empty_keys(n, key_bytes, cdf.device)
    check(lib().hg_gen_zipf(_ptr(out), n, key_bytes, _ptr(cdf), cdf.numel(), seed,
                            _stream(stream)), "hg_gen_zipf")
    return out
