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
