"""The multi-rank restatement of the reference's natural-order path
(oracle/distributed_ref.c), pinned to the reference's own compiled `_ref`
code, and the optimized multi-rank restatement held to the reference's
multi-rank iteration bounds.

* one rank: its CG_ref equals the reference's CG_ref (oracle/_ref, one OpenMP
  thread so that the dot products sum in index order) bit for bit, with and
  without the preconditioner;
* several ranks: its decomposed SpMV equals the reference's SpMV of the global
  grid bit for bit (every row sums its neighbours in the same order), and its
  unpreconditioned CG follows the global one to rounding (only the dot
  products' summation order differs);
* the optimized restatement (oracle/distributed.c) reaches the tolerance that
  50 CG_ref iterations fix within src/test_rochpcg.cpp's bound for that rank
  count and brick -- the same check the GPU test makes of the CUDA path.
"""
import ctypes
import ctypes.util
import os

import numpy as np
import pytest

from niter_bounds import check_niter


def _omp():
    name = ctypes.util.find_library("gomp") or "libgomp.so.1"
    return ctypes.CDLL(name)


class one_thread:
    """OpenMP's thread count for the calling thread set to 1 for the block."""

    def __enter__(self):
        self.L = _omp()
        self.L.omp_get_max_threads.restype = ctypes.c_int
        self.prev = self.L.omp_get_max_threads()
        self.L.omp_set_num_threads(1)

    def __exit__(self, *a):
        self.L.omp_set_num_threads(self.prev)


def _need_ref(O):
    if not os.path.exists(O.REF_SO):
        pytest.skip("oracle/_ref not built (needs the reference sources)")


def _concat_to_global(size, n, grid):
    """Index of every concatenated (rank, natural row) in the global grid."""
    npx, npy, npz = grid
    m = n ** 3
    i = np.arange(m)
    ix, iy, iz = i % n, (i // n) % n, i // (n * n)
    out = np.empty(size * m, np.int64)
    for q in range(size):
        ipz, ipy, ipx = q // (npx * npy), (q % (npx * npy)) // npx, q % npx
        out[q * m:(q + 1) * m] = ((ipz * n + iz) * npy * n + ipy * n + iy) * npx * n + ipx * n + ix
    return out


@pytest.mark.parametrize("dims", [(16, 16, 16), (24, 16, 8)])
@pytest.mark.parametrize("precond", [True, False])
def test_one_rank_is_the_reference_cg_ref(oracle_libs, dims, precond):
    O = oracle_libs
    _need_ref(O)
    d = O.DistRefOracle(1, *dims).cg(30, 0.0, precond=precond)
    R = O.RefProblem(*dims)
    with one_thread():
        r = R.cg(30, 0.0, precond=precond)
    assert d["niters"] == r["niters"] == 30
    assert d["normr0"] == r["normr0"] and d["normr"] == r["normr"]


@pytest.mark.parametrize("size,n", [(2, 16), (4, 8), (3, 8), (8, 8)])
def test_decomposed_reference_operator_is_the_global_one(oracle_libs, size, n):
    O = oracle_libs
    _need_ref(O)
    grid = O.od_shape(size)
    D = O.DistRefOracle(size, n, n, n)
    G = O.RefProblem(grid[0] * n, grid[1] * n, grid[2] * n)
    idx = _concat_to_global(size, n, grid)
    xg = np.random.default_rng(size).uniform(-1, 1, idx.size)
    assert np.array_equal(D.spmv(0, xg[idx]), G.spmv(0, xg)[idx])
    d = D.cg(25, 0.0, precond=False)
    with one_thread():
        g = G.cg(25, 0.0, precond=False)
    assert d["normr0"] == g["normr0"]
    np.testing.assert_allclose(d["normr"], g["normr"], rtol=1e-9)


def test_decomposed_gauss_seidel_freezes_the_external_columns(oracle_libs):
    """ComputeSYMGS_ref after ExchangeHalo on two ranks, restated here in
    Python loops on a 2 x (4x4x4) problem: each rank sweeps its own rows
    forward and back, reading the other rank's rows at the values they had
    when the sweep began.  A sequential sweep over the global rows would read
    rank 0's new values in rank 1's sweep and differ."""
    O = oracle_libs
    n, size = 4, 2
    grid = O.od_shape(size)
    D = O.DistRefOracle(size, n, n, n, nlevels=1)
    m = n ** 3
    idx = _concat_to_global(size, n, grid)
    gdims = (grid[0] * n, grid[1] * n, grid[2] * n)
    where = np.empty(size * m, np.int64)
    where[idx] = np.arange(size * m)  # global natural id -> concatenated index
    rng = np.random.default_rng(3)
    r, x0 = rng.uniform(-1, 1, size * m), rng.uniform(-1, 1, size * m)
    want = x0.copy()
    for q in range(size):
        rows = range(q * m, (q + 1) * m)
        for order in (rows, reversed(rows)):
            for g in order:
                gid = idx[g]
                gx, gy, gz = gid % gdims[0], (gid // gdims[0]) % gdims[1], gid // (gdims[0] * gdims[1])
                s = r[g]
                for dz in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dx in (-1, 0, 1):
                            X, Y, Z = gx + dx, gy + dy, gz + dz
                            if not (0 <= X < gdims[0] and 0 <= Y < gdims[1] and 0 <= Z < gdims[2]):
                                continue
                            c = where[(Z * gdims[1] + Y) * gdims[0] + X]
                            v = want[c] if c // m == q else x0[c]
                            s -= (26.0 if c == g else -1.0) * v
                s += want[g] * 26.0
                want[g] = s / 26.0
    got = D.symgs(0, r, x0)
    assert np.array_equal(got, want)
    if os.path.exists(O.REF_SO):
        G = O.RefProblem(*gdims, nlevels=1)
        xg, rg = np.empty_like(x0), np.empty_like(r)
        xg[idx], rg[idx] = x0, r
        assert not np.array_equal(G.symgs(0, rg, xg)[idx], got)


@pytest.mark.parametrize("size,n", [(2, 16), (4, 16)])
def test_optimized_restatement_meets_the_reference_bounds(oracle_libs, size, n):
    O = oracle_libs
    ref = O.DistRefOracle(size, n, n, n).cg(50, 0.0)
    tol = ref["normr"] / ref["normr0"]
    got = O.DistOracle(size, n, n, n).cg(500, tol)
    assert got["normr0"] == pytest.approx(ref["normr0"], rel=1e-14)
    assert got["normr"] / got["normr0"] <= tol
    assert got["niters"] <= check_niter(size, (n, n, n))
