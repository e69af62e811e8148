"""CPU oracle for the HashGraph build + intersect path.

TEST INFRASTRUCTURE ONLY: this is the checker.  It wraps ``liboracle.so`` (a
plain-C restatement of the reference's algorithm, ``oracle/hg_oracle.c``) for
numpy arrays.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` import it; the product package never does.

Parity is pinned by ``tests/golden/``: murmur known answers produced by the
reference's own ``hash_murmur`` (include/SingleHashGraphOperators.cuh:31-69)
and CSR / intersect results produced by the reference's ``MultiHashGraph`` run
on a B200 (``oracle/ref_multi_driver.cu``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None

_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_p = ctypes.c_void_p


def build_lib(force: bool = False) -> str:
    """Compile liboracle.so with gcc (oracle/Makefile, target ``oracle``)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build_lib()
        L = ctypes.CDLL(LIB_PATH)
        L.or_murmur3_low32.restype = _u32
        L.or_murmur3_low32.argtypes = [_u64]
        L.or_bucket.restype = _u64
        L.or_bucket.argtypes = [_u64, _u64]
        L.or_buckets.restype = None
        L.or_buckets.argtypes = [_p, _u64, ctypes.c_int, _u64, _p]
        L.or_fastmod_magic.restype = _u64
        L.or_fastmod_magic.argtypes = [_u32]
        L.or_fastmod.restype = _u32
        L.or_fastmod.argtypes = [_u32, _u64, _u32]
        L.or_mix64.restype = _u64
        L.or_mix64.argtypes = [_u64]
        L.or_rand64.restype = _u64
        L.or_rand64.argtypes = [_u64, _u64, _u64]
        L.or_perm.restype = _u64
        L.or_perm.argtypes = [_u64, _u64, _u64]
        L.or_gen_uniform.restype = None
        L.or_gen_uniform.argtypes = [_p, _u64, ctypes.c_int, _u64]
        L.or_gen_overlap.restype = None
        L.or_gen_overlap.argtypes = [_p, _u64, ctypes.c_int, _p, _u64, ctypes.c_double, _u64]
        L.or_zipf_cdf.restype = ctypes.c_int
        L.or_zipf_cdf.argtypes = [_p, _u64, ctypes.c_double]
        L.or_gen_zipf.restype = None
        L.or_gen_zipf.argtypes = [_p, _u64, ctypes.c_int, _p, _u64, _u64]
        L.or_build.restype = ctypes.c_int
        L.or_build.argtypes = [_p, _u64, ctypes.c_int, _u64, _p, _p, _p]
        L.or_build_mt.restype = ctypes.c_int
        L.or_build_mt.argtypes = [_p, _u64, ctypes.c_int, _u64, _p, _p, _p, ctypes.c_int]
        L.or_canonicalize.restype = None
        L.or_canonicalize.argtypes = [_p, _u64, _p, ctypes.c_int, _p]
        L.or_intersect.restype = _u64
        L.or_intersect.argtypes = [_p, _u64, _p, _p, ctypes.c_int, _p, _u64, _p, _p, _u64]
        L.or_intersect_mt.restype = _u64
        L.or_intersect_mt.argtypes = [_p, _u64, _p, _p, ctypes.c_int, _p, _u64, _p, _u64, ctypes.c_int]
        L.or_join_count_sorted.restype = _u64
        L.or_join_count_sorted.argtypes = [_p, _u64, _p, _u64, ctypes.c_int]
        L.or_join_count_hashed.restype = _u64
        L.or_join_count_hashed.argtypes = [_p, _u64, _p, _u64, ctypes.c_int, _u64, ctypes.c_int]
        L.or_max_threads.restype = ctypes.c_int
        L.or_max_threads.argtypes = []
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _kb(dtype) -> int:
    dt = np.dtype(dtype)
    if dt not in (np.dtype(np.uint32), np.dtype(np.uint64)):
        raise TypeError(f"keys must be uint32 or uint64, got {dt}")
    return dt.itemsize


def key_dtype(key_bytes: int):
    return np.uint32 if key_bytes == 4 else np.uint64


def murmur(keys: np.ndarray) -> np.ndarray:
    """murmur3_x86_32 of the low 32 bits of each key, seed 0."""
    keys = np.ascontiguousarray(keys)
    out = np.empty(keys.size, dtype=np.uint64)
    lib().or_buckets(_ptr(keys), keys.size, _kb(keys.dtype), 1 << 32, _ptr(out))
    return out.astype(np.uint32)


def buckets(keys: np.ndarray, n_buckets: int) -> np.ndarray:
    keys = np.ascontiguousarray(keys)
    out = np.empty(keys.size, dtype=np.uint64)
    lib().or_buckets(_ptr(keys), keys.size, _kb(keys.dtype), int(n_buckets), _ptr(out))
    return out


def gen_uniform(n: int, key_bytes: int, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=key_dtype(key_bytes))
    lib().or_gen_uniform(_ptr(out), n, key_bytes, seed)
    return out


def gen_overlap(n: int, a_keys: np.ndarray, frac: float, seed: int) -> np.ndarray:
    a_keys = np.ascontiguousarray(a_keys)
    out = np.empty(n, dtype=a_keys.dtype)
    lib().or_gen_overlap(_ptr(out), n, a_keys.dtype.itemsize, _ptr(a_keys), a_keys.size,
                         float(frac), seed)
    return out


def zipf_cdf(universe: int, s: float) -> np.ndarray:
    cdf = np.empty(universe, dtype=np.uint64)
    if lib().or_zipf_cdf(_ptr(cdf), universe, float(s)) != 0:
        raise ValueError("bad zipf universe")
    return cdf


def gen_zipf(n: int, key_bytes: int, cdf: np.ndarray, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=key_dtype(key_bytes))
    lib().or_gen_zipf(_ptr(out), n, key_bytes, _ptr(cdf), cdf.size, seed)
    return out


def build(keys: np.ndarray, n_buckets: int, with_index: bool = True, threads: int | None = None):
    """Stable CSR build -> (offsets[u32, B+1], keys_out, idx_out or None)."""
    keys = np.ascontiguousarray(keys)
    kb = _kb(keys.dtype)
    offsets = np.empty(int(n_buckets) + 1, dtype=np.uint32)
    keys_out = np.empty_like(keys)
    idx = np.empty(keys.size, dtype=np.uint32) if with_index else None
    if threads is None:
        rc = lib().or_build(_ptr(keys), keys.size, kb, int(n_buckets), _ptr(offsets),
                            _ptr(keys_out), _ptr(idx))
    else:
        rc = lib().or_build_mt(_ptr(keys), keys.size, kb, int(n_buckets), _ptr(offsets),
                               _ptr(keys_out), _ptr(idx), int(threads))
    if rc != 0:
        raise ValueError(f"oracle build failed ({rc})")
    return offsets, keys_out, idx


def canonicalize(offsets: np.ndarray, keys: np.ndarray, idx: np.ndarray | None = None):
    """Sort each bucket by (key, idx) in place; returns (keys, idx)."""
    keys = np.ascontiguousarray(keys)
    if idx is not None:
        idx = np.ascontiguousarray(idx)
    lib().or_canonicalize(_ptr(offsets), offsets.size - 1, _ptr(keys), keys.dtype.itemsize,
                          _ptr(idx))
    return keys, idx


def intersect(offsets, a_keys, a_idx, q_keys, pair_cap: int = 0, q_idx=None, threads=None):
    """Probe intersect -> (count, pairs[min(count, cap), 2] as uint32)."""
    q_keys = np.ascontiguousarray(q_keys)
    kb = _kb(q_keys.dtype)
    if a_keys.dtype != q_keys.dtype:
        raise TypeError("key dtype mismatch")
    pairs = np.zeros((max(int(pair_cap), 0), 2), dtype=np.uint32) if pair_cap else None
    if threads is None:
        c = lib().or_intersect(_ptr(offsets), offsets.size - 1, _ptr(a_keys), _ptr(a_idx), kb,
                               _ptr(q_keys), q_keys.size, _ptr(q_idx), _ptr(pairs),
                               int(pair_cap))
    else:
        c = lib().or_intersect_mt(_ptr(offsets), offsets.size - 1, _ptr(a_keys), _ptr(a_idx), kb,
                                  _ptr(q_keys), q_keys.size, _ptr(pairs), int(pair_cap),
                                  int(threads))
    if pairs is not None:
        pairs = pairs[: min(int(c), int(pair_cap))]
    return int(c), pairs


def join_count(a_keys: np.ndarray, b_keys: np.ndarray) -> int:
    """sum over keys of multA(k) * multB(k), by sort + merge-join."""
    a = np.sort(a_keys)
    b = np.sort(b_keys)
    return int(lib().or_join_count_sorted(_ptr(a), a.size, _ptr(b), b.size, a.dtype.itemsize))


def join_count_hashed(a_keys: np.ndarray, b_keys: np.ndarray, max_distinct: int | None = None,
                      threads: int = 0) -> int:
    """sum over keys of multA(k) * multB(k) through a hash map of A's
    distinct keys (linear time; for skewed sets of hundreds of millions)."""
    a_keys = np.ascontiguousarray(a_keys)
    b_keys = np.ascontiguousarray(b_keys)
    if a_keys.dtype != b_keys.dtype:
        raise TypeError("key dtype mismatch")
    md = a_keys.size if max_distinct is None else int(max_distinct)
    c = int(lib().or_join_count_hashed(_ptr(a_keys), a_keys.size, _ptr(b_keys), b_keys.size,
                                       _kb(a_keys.dtype), md, int(threads)))
    if c == (1 << 64) - 1:
        raise MemoryError("join-count map could not be allocated or filled up")
    return c


def max_threads() -> int:
    return int(lib().or_max_threads())


def ref_binary(name: str) -> str | None:
    """Path of a reference driver built into oracle/_ref, or None."""
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) else None
