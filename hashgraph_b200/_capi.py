"""ctypes binding of the C ABI in include/hashgraph_b200.h.

The shared library is built in-tree (hashgraph_b200/_lib/libhashgraph_b200.so,
``hashgraph_b200/csrc/Makefile``).  There is no fallback: if the library is
missing or cannot load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libhashgraph_b200.so")
CSRC = os.path.join(HERE, "csrc")

HG_OK = 0
STATUS_NAMES = {
    0: "HG_OK",
    -1: "HG_ERR_INVALID_ARGUMENT",
    -2: "HG_ERR_CUDA",
    -3: "HG_ERR_OUT_OF_MEMORY",
    -4: "HG_ERR_PAIR_CAPACITY",
    -5: "HG_ERR_DEVICE_TIMEOUT",
    -6: "HG_ERR_TOO_LARGE",
    -7: "HG_ERR_NO_DEVICE",
    -8: "HG_ERR_KEY_WIDTH",
    -9: "HG_ERR_BUCKET_MISMATCH",
    -10: "HG_ERR_DEVICE_STATE",
}
ERR_PAIR_CAPACITY = -4
ERR_DEVICE_TIMEOUT = -5

# Every symbol include/hashgraph_b200.h declares: (restype, argtypes).
_p = ctypes.c_void_p
_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_i32 = ctypes.c_int32
_int = ctypes.c_int
_sz = ctypes.c_size_t
_pp = ctypes.POINTER(ctypes.c_void_p)
class BatchParams(ctypes.Structure):
    """hg_batch_params of include/hashgraph_b200.h."""
    _fields_ = [("part_min", ctypes.c_uint64), ("l2_table_bytes", ctypes.c_uint64)]


class BatchPair(ctypes.Structure):
    """hg_batch_pair of include/hashgraph_b200.h."""
    _fields_ = [
        ("d_keys", ctypes.c_void_p), ("n", ctypes.c_uint64), ("n_buckets", ctypes.c_uint64),
        ("d_query", ctypes.c_void_p), ("nq", ctypes.c_uint64), ("d_offsets", ctypes.c_void_p),
        ("d_keys_out", ctypes.c_void_p), ("d_idx_out", ctypes.c_void_p), ("d_pairs", ctypes.c_void_p),
        ("pair_cap", ctypes.c_uint64), ("d_count", ctypes.c_void_p),
    ]


class ServerRequest(ctypes.Structure):
    """hg_server_request of include/hashgraph_b200.h."""
    _fields_ = [("kind", ctypes.c_int), ("with_index", ctypes.c_int), ("table_id", ctypes.c_uint64),
                ("d_data", ctypes.c_void_p), ("n", ctypes.c_uint64), ("n_buckets", ctypes.c_uint64),
                ("d_pairs", ctypes.c_void_p), ("pair_cap", ctypes.c_uint64), ("arrival_s", ctypes.c_double)]


class ServerDone(ctypes.Structure):
    """hg_server_done of include/hashgraph_b200.h."""
    _fields_ = [("ticket", ctypes.c_uint64), ("kind", ctypes.c_int), ("missed", ctypes.c_int),
                ("count", ctypes.c_ulonglong), ("latency_s", ctypes.c_double)]


SIGNATURES = {
    "hg_status_str": (ctypes.c_char_p, [_i32]),
    "hg_version": (ctypes.c_char_p, []),
    "hg_last_error": (ctypes.c_char_p, []),
    "hg_hash": (ctypes.c_uint32, [_u64]),
    "hg_device_error": (_i32, [_p, ctypes.POINTER(_i32)]),
    "hg_debug_set_wait_limit": (_i32, [ctypes.c_uint32, _p]),
    "hg_build_workspace_size": (_i32, [_u64, _int, _u64, _int, ctypes.POINTER(_sz)]),
    "hg_build_into": (_i32, [_p, _u64, _int, _u64, _p, _p, _p, _p, _sz, _p]),
    "hg_build_workspace_size_path": (_i32, [_u64, _int, _u64, _int, _int, ctypes.POINTER(_sz)]),
    "hg_build_into_path": (_i32, [_p, _u64, _int, _u64, _p, _p, _p, _p, _sz, _int, _p]),
    "hg_build_into_noalloc": (_i32, [_p, _u64, _int, _u64, _p, _p, _p, _p]),
    "hg_table_create": (_i32, [_u64, _int, _u64, _int, _pp]),
    "hg_table_build": (_i32, [_p, _p, _u64, _p]),
    "hg_build": (_i32, [_p, _u64, _int, _u64, _int, _pp, _p]),
    "hg_table_view": (_i32, [_p, _pp, _pp, _pp, ctypes.POINTER(_u64), ctypes.POINTER(_u64),
                             ctypes.POINTER(_int)]),
    "hg_table_device_bytes": (_i32, [_p, ctypes.POINTER(_sz)]),
    "hg_table_free": (None, [_p]),
    "hg_intersect_workspace_size": (_i32, [_u64, _int, _u64, _u64, _int, _int, ctypes.POINTER(_sz)]),
    "hg_intersect_workspace_size_path": (_i32, [_u64, _int, _u64, _u64, _int, _int, _int,
                                                ctypes.POINTER(_sz)]),
    "hg_intersect_into_path": (_i32, [_p, _p, _p, _u64, _u64, _int, _p, _u64, _p, _p, _u64, _p, _p,
                                      _sz, _int, _p]),
    "hg_intersect_into": (_i32, [_p, _p, _p, _u64, _u64, _int, _p, _u64, _p, _p, _u64, _p, _p,
                                 _sz, _p]),
    "hg_intersect": (_i32, [_p, _p, _u64, _p, _p, _u64, _p, _p]),
    "hg_intersect_tables": (_i32, [_p, _p, _p, _u64, _p, _p]),
    "hg_gen_uniform": (_i32, [_p, _u64, _int, _u64, _p]),
    "hg_gen_overlap": (_i32, [_p, _u64, _int, _p, _u64, _u64, _u64, _p]),
    "hg_gen_zipf": (_i32, [_p, _u64, _int, _p, _u64, _u64, _p]),
    "hg_zipf_cdf": (_i32, [_p, _u64, ctypes.c_double]),
    "hg_gen_bounded": (_i32, [_p, _u64, _int, _u64, _u64, _p]),
    "hg_gather_pair_keys": (_i32, [_p, _int, _p, _u64, _int, _p, _p]),
    "hg_export_reference_layout": (_i32, [_p, _p, _p, _u64, _u64, _int, _p, _p, _p]),
    "hg_batch_create": (_i32, [ctypes.POINTER(BatchPair), _int, _int, _p, _pp]),
    "hg_batch_run": (_i32, [_p, _p]),
    "hg_batch_device_bytes": (_i32, [_p, ctypes.POINTER(_sz)]),
    "hg_batch_free": (None, [_p, _p]),
    "hg_batch_params_default": (_i32, [ctypes.POINTER(BatchParams)]),
    "hg_batch_create_params": (_i32, [ctypes.POINTER(BatchPair), _int, _int, ctypes.POINTER(BatchParams), _p, _pp]),
    "hg_batch_autotune": (_i32, [ctypes.POINTER(BatchPair), _int, _int, _p, ctypes.POINTER(BatchParams),
                                 ctypes.POINTER(ctypes.c_float)]),
    "hg_batch_build_intersect": (_i32, [ctypes.POINTER(BatchPair), _int, _int, _p]),
    "hg_table_save": (_i32, [_p, ctypes.c_char_p, _p]),
    "hg_table_load": (_i32, [ctypes.c_char_p, _pp, _p]),
    "hg_table_save_arrays": (_i32, [ctypes.c_char_p, _p, _p, _p, _u64, _u64, _int, _p]),
    "hg_table_file_info": (_i32, [ctypes.c_char_p, ctypes.POINTER(_u64), ctypes.POINTER(_u64),
                                  ctypes.POINTER(_int), ctypes.POINTER(_int)]),
    "hg_table_load_arrays": (_i32, [ctypes.c_char_p, _p, _p, _p, _u64, _u64, _int, _p]),
    "hg_server_now": (ctypes.c_double, []),
    "hg_server_create": (_i32, [_sz, _int, _int, _u64, _int, _pp]),
    "hg_server_reserve": (_i32, [_p, _sz]),
    "hg_server_build": (_i32, [_p, _u64, _p, _u64, _u64, _int, ctypes.c_double, ctypes.POINTER(_u64)]),
    "hg_server_intersect": (_i32, [_p, _u64, _p, _u64, _p, _u64, ctypes.c_double, ctypes.POINTER(_u64)]),
    "hg_server_submit": (_i32, [_p, ctypes.POINTER(ServerRequest), _int, ctypes.POINTER(_u64), ctypes.POINTER(_int)]),
    "hg_server_poll": (_i32, [_p, _int, ctypes.POINTER(ServerDone), _int, ctypes.POINTER(_int)]),
    "hg_server_set_batching": (_i32, [_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double]),
    "hg_server_batch_stats": (_i32, [_p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "hg_server_stats": (_i32, [_p, ctypes.POINTER(_u64), ctypes.POINTER(_sz), ctypes.POINTER(_u64),
                               ctypes.POINTER(_u64)]),
    "hg_server_free": (None, [_p]),
    "hg_shard_histogram": (_i32, [_p, _u64, _int, _u64, _u32, _p, _p]),
    "hg_shard_splits": (_i32, [_p, _u32, _u64, _int, _p]),
    "hg_shard_route_workspace_size": (_i32, [_u64, _int, ctypes.POINTER(_sz)]),
    "hg_shard_route": (_i32, [_p, _u64, _int, _u64, _p, _int, _u32, _p, _p, _p, _p, _sz, _p]),
    "hg_shard_build_into": (_i32, [_p, _p, _u64, _int, _u64, _u64, _u64, _p, _p, _p, _p, _sz, _p]),
    "hg_shard_build_into_path": (_i32, [_p, _p, _u64, _int, _u64, _u64, _u64, _p, _p, _p, _p, _sz, _int, _p]),
    "hg_shard_intersect_into": (_i32, [_p, _p, _p, _u64, _u64, _u64, _u64, _int, _p, _u64, _p, _p, _u64, _p, _p,
                                       _sz, _p]),
    "hg_shard_intersect_into_path": (_i32, [_p, _p, _p, _u64, _u64, _u64, _u64, _int, _p, _u64, _p, _p, _u64, _p,
                                            _p, _sz, _int, _p]),
    "hg_profile_enable": (_i32, [_int]),
    "hg_profile_read": (_i32, [_int, ctypes.POINTER(_int), ctypes.POINTER(ctypes.c_char_p),
                               ctypes.POINTER(ctypes.c_float)]),
    "hg_launch_count": (ctypes.c_ulonglong, []),
}


class HGError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{what}: {name}" if what else name)


_lib = None


def build_library(force: bool = False) -> str:
    """Compile the sm_100a library in-tree with nvcc (csrc/Makefile)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", CSRC], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C {CSRC}` "
                "(or __graft_entry__.build()); there is no fallback path")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, what: str = "") -> None:
    if status != HG_OK:
        detail = ""
        try:
            detail = lib().hg_last_error().decode()
        except Exception:
            pass
        raise HGError(status, f"{what} [{detail}]" if detail else what)


def status_str(status: int) -> str:
    return lib().hg_status_str(status).decode()
