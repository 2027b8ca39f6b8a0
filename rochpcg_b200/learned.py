"""Learned smoother for the coarse MG levels: a 3-layer 3x3x3 conv net
(1 -> 16 -> 16 -> 1 channels, ReLU, BF16 weights, FP32 accumulation) whose
forward pass, backward pass and Adam update all run in libhpcgb200's tcgen05
kernels.  No reference counterpart.

Device buffers are torch CUDA tensors (plumbing only); every computation is a
call into the library.  Weight files are ``.npz`` with the FP32 weights
(``w``: layers 1..3, each ``w[tap][ci][co]``) and the training record.
"""
from __future__ import annotations

import ctypes
import dataclasses
import hashlib
import json
import os

import numpy as np

from ._lib import check, load

WEIGHTS = 3 * 27 * 16 * 16
PLAIN, ODD, TIED = 0, 1, 2
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "smoother_l23.npz")


def _torch():
    import torch

    return torch


def _vp(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream() -> ctypes.c_void_p:
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def jacobi_weights(omega: float = 1.0, noise: float = 0.0, seed: int = 0, twin: int = 1) -> np.ndarray:
    """Weights whose network computes omega * r / 26 (a damped Jacobi step)
    plus seeded uniform noise on the other used weights; `twin` is the hidden
    channel carrying relu(-r) (8 for the tied odd form)."""
    L = load()
    w = np.zeros(WEIGHTS, np.float32)
    check(L, L.hpcgb200_smoother_init_jacobi(w.ctypes.data_as(ctypes.c_void_p), omega, noise, seed, twin))
    return w


@dataclasses.dataclass
class PairSet:
    """`count` (residual, error) pairs on an nz x ny x nx grid (device)."""
    r: object
    e: object
    inv_ee: object
    count: int
    dims: tuple
    batch: int = 1


class _CPairSet(ctypes.Structure):
    _fields_ = [("r", ctypes.c_void_p), ("e", ctypes.c_void_p), ("inv_ee", ctypes.c_void_p), ("count", ctypes.c_int),
                ("nz", ctypes.c_int), ("ny", ctypes.c_int), ("nx", ctypes.c_int), ("batch", ctypes.c_int)]


def make_pairs(fine_n: int, level: int, first_seed: int, count: int, tol: float = 1e-8, batch: int = 1) -> PairSet:
    """Training pairs of the plain FP32 V-cycle on fine_n^3 grids: the residual
    handed to MG level `level` for b ~ N(0,1) seeds first_seed.., and the
    level's exact correction (hpcgb200_make_training_pairs)."""
    torch = _torch()
    L = load()
    n = fine_n >> level
    per = n ** 3
    r = torch.empty(count * per, dtype=torch.float32, device="cuda")
    e = torch.empty(count * per, dtype=torch.float32, device="cuda")
    inv = torch.empty(count, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    check(L, L.hpcgb200_make_training_pairs(fine_n, level, first_seed, count, _vp(r), _vp(e), _vp(inv), tol))
    return PairSet(r, e, inv, count, (n, n, n), batch)


class Smoother:
    """Device state of the conv-net smoother (weights, tiles, activations, Adam)."""

    def __init__(self, weights: np.ndarray | None = None, symmetry: int = PLAIN):
        self.L = load()
        h = ctypes.c_void_p()
        check(self.L, self.L.hpcgb200_smoother_create(ctypes.byref(h)))
        self.h = h
        self.meta: dict = {}
        self.symmetry = PLAIN
        self.configure(symmetry)
        if weights is not None:
            self.set_weights(weights)

    def configure(self, symmetry: int):
        """PLAIN: N(r); ODD: (N(r) - N(-r)) / 2; TIED: weights kept in the tied
        odd form, so one evaluation is odd."""
        check(self.L, self.L.hpcgb200_smoother_configure(self.h, int(symmetry)))
        self.symmetry = int(symmetry)

    def close(self):
        if getattr(self, "h", None):
            self.L.hpcgb200_smoother_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == WEIGHTS
        check(self.L, self.L.hpcgb200_smoother_set_weights(self.h, w.ctypes.data_as(ctypes.c_void_p)))

    def get_weights(self) -> np.ndarray:
        w = np.empty(WEIGHTS, np.float32)
        check(self.L, self.L.hpcgb200_smoother_get_weights(self.h, w.ctypes.data_as(ctypes.c_void_p)))
        return w

    def forward(self, r, dims, nb: int = 1):
        torch = _torch()
        nz, ny, nx = dims
        y = torch.empty(nb * nz * ny * nx, dtype=torch.float32, device="cuda")
        check(self.L, self.L.hpcgb200_smoother_forward(self.h, nb, nz, ny, nx, _vp(r), _vp(y), _stream()))
        return y

    def loss_grad(self, r, e, inv_norm, dims, nb: int = 1, scale: float = 1.0, kind: int = 0):
        torch = _torch()
        nz, ny, nx = dims
        dw = torch.empty(WEIGHTS, dtype=torch.float32, device="cuda")
        loss = ctypes.c_double()
        check(self.L, self.L.hpcgb200_smoother_loss_grad(self.h, nb, nz, ny, nx, _vp(r), _vp(e), _vp(inv_norm),
                                                         scale, kind, _vp(dw), ctypes.byref(loss), _stream()))
        return loss.value, dw

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        check(self.L, self.L.hpcgb200_smoother_adam_step(self.h, lr, beta1, beta2, eps, _stream()))

    def train(self, sets: list, epochs: int, lr0: float = 2e-3, lr1: float = 2e-4, seed: int = 0, kind: int = 0):
        """Adam over the pair sets on the device; returns the mean loss of each epoch."""
        torch = _torch()
        cs = (_CPairSet * len(sets))()
        for i, s in enumerate(sets):
            nz, ny, nx = s.dims
            cs[i] = _CPairSet(s.r.data_ptr(), s.e.data_ptr(), s.inv_ee.data_ptr(), s.count, nz, ny, nx, s.batch)
        hist = np.zeros(epochs)
        torch.cuda.synchronize()
        check(self.L, self.L.hpcgb200_smoother_train(self.h, cs, len(sets), epochs, lr0, lr1, kind, seed,
                                                     hist.ctypes.data_as(ctypes.c_void_p), None))
        return hist

    # -- weight files -------------------------------------------------------
    def save(self, path: str, **meta):
        w = self.get_weights()
        meta = dict(meta, symmetry=self.symmetry, sha256=hashlib.sha256(w.tobytes()).hexdigest())
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, w=w, meta=np.array(json.dumps(meta)))

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS) -> "Smoother":
        w, meta = read_weights(path)
        s = cls(w, symmetry=int(meta.get("symmetry", PLAIN)))
        s.meta = meta
        return s


def read_weights(path: str = DEFAULT_WEIGHTS):
    """(weights, training record) of a weight file, checksum verified."""
    with np.load(path) as f:
        w = np.array(f["w"], np.float32)
        meta = json.loads(str(f["meta"]))
    if w.size != WEIGHTS or hashlib.sha256(w.tobytes()).hexdigest() != meta.get("sha256"):
        raise ValueError(f"{path}: not a smoother weight file (size or checksum mismatch)")
    return w, meta


def sample_norms(e, dims, nb: int, kind: int = 0):
    """1/(e.e) (kind 0) or 1/(e.Ae) (kind 1) per sample, on the device."""
    torch = _torch()
    L = load()
    nz, ny, nx = dims
    out = torch.empty(nb, dtype=torch.float32, device="cuda")
    check(L, L.hpcgb200_sample_norms(nb, nz, ny, nx, _vp(e), kind, _vp(out), _stream()))
    return out
