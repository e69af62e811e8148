"""Shared test set-up: the `gpu` marker, repo root on sys.path, helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the sm_100a library")
    config.addinivalue_line("markers", "slow: full-size checks (minutes)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def hg():
    """The product package with its CUDA library loaded; fails loudly if the
    library is missing on a GPU machine."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    import hashgraph_b200
    hashgraph_b200.lib()
    return hashgraph_b200


def to_np_u(t, key_bytes):
    """torch int32/int64 tensor holding unsigned values -> numpy uint32/uint64."""
    a = t.detach().cpu().numpy()
    return a.view(np.uint32 if key_bytes == 4 else np.uint64)


def from_np_u(a, device="cuda"):
    import torch
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).to(device)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64).copy()).to(device)
    raise TypeError(a.dtype)


def device_array(ptr: int, count: int, np_dtype):
    """Copy `count` elements at device address `ptr` to a numpy array (via
    __cuda_array_interface__, so torch never owns the memory)."""
    import torch

    class _View:
        pass

    v = _View()
    v.__cuda_array_interface__ = {"shape": (count,), "typestr": np.dtype(np_dtype).str,
                                  "data": (int(ptr), False), "version": 2}
    return torch.as_tensor(v, device="cuda").cpu().numpy().copy()
