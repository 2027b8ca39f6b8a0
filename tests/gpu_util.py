"""Shared helpers of the GPU parity tests."""
from __future__ import annotations

import functools

import numpy as np


@functools.lru_cache(maxsize=None)
def problems(nx, ny, nz, keep=True):
    import rochpcg_b200 as R
    from oracle.oracle import ColoredProblem

    return R.Problem(nx, ny, nz, keep_generated=keep), ColoredProblem(nx, ny, nz)


def to_dev(a: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def sync(P):
    import torch

    torch.cuda.ExternalStream(P.stream_handle).synchronize()
    torch.cuda.synchronize()


def host(t) -> np.ndarray:
    return t.cpu().numpy()


class _DeviceArray:
    """A raw device allocation of the library, seen by torch through the CUDA
    array interface (no copy)."""

    def __init__(self, ptr: int, n: int, dtype):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str, "data": (ptr, False),
                                         "version": 3}


def dev_field(P, name: str, level: int, dtype):
    """Torch view of a problem's DEVICE array (compared on the GPU, so the
    full-size tests need no host copy of the library's arrays)."""
    import ctypes

    import torch

    from rochpcg_b200 import check

    nbytes = ctypes.c_size_t()
    check(P.L, P.L.hpcgb200_problem_field_bytes(P.h, level, name.encode(), ctypes.byref(nbytes)))
    n = nbytes.value // np.dtype(dtype).itemsize
    sync(P)
    return torch.as_tensor(_DeviceArray(P.device_ptr(name, level), n, dtype), device="cuda")
