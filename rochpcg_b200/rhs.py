"""Seeded right-hand sides.

``normal_rhs(m, seed)`` gives b ~ N(0,1) i.i.d. indexed by the NATURAL row id,
from a counter-based generator written out here (SplitMix64 finalizer over
(key + 2i, key + 2i + 1), then Box-Muller), so the same b is reproducible on
any machine and independent of how rows are later permuted.
(std::normal_distribution is implementation-defined, so the generator is
specified by this code, not by a library.)
"""
from __future__ import annotations

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    z = z + _GAMMA
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def normal_rhs(m: int, seed: int, chunk: int = 1 << 22) -> np.ndarray:
    out = np.empty(m, np.float64)
    with np.errstate(over="ignore"):
        key = _mix(np.array([seed], np.uint64))[0]
        for s in range(0, m, chunk):
            e = min(m, s + chunk)
            i = np.arange(s, e, dtype=np.uint64)
            a = _mix(key + np.uint64(2) * i)
            b = _mix(key + np.uint64(2) * i + np.uint64(1))
            u1 = ((a >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
            u2 = (b >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
            out[s:e] = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    return out
