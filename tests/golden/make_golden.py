"""Generate the golden fixtures in tests/golden/ from the reference's own CPU
path (oracle/_ref/libhpcg_ref.so, compiled unmodified from rocHPCG 0.8.9
src/*_ref.cpp by oracle/Makefile) and from the colored restatement.

Run from the repository root where the reference tree exists:

    make -C oracle ref && python tests/golden/make_golden.py

Fixtures (small, committed):
  ref_<nx>x<ny>x<nz>.npz  -- reference CG_ref / SpMV / SymGS results (natural order)
  colored_<...>.npz       -- colored restatement index arrays (regression pins)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import ColoredProblem, RefProblem  # noqa: E402

GRIDS = [(16, 16, 16), (32, 32, 32), (16, 24, 32), (64, 64, 64)]


def seeded(n: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


def make_ref(nx, ny, nz):
    R = RefProblem(nx, ny, nz)
    R.check_problem()
    out = {}
    r50 = R.cg(50, 0.0)
    out["cg50_normr0"] = r50["normr0"]
    out["cg50_normr"] = r50["normr"]
    r9 = R.cg(500, 1e-9)
    out["cg1e9_niters"] = r9["niters"]
    out["cg1e9_normr"] = r9["normr"]
    m = R.nrows[0]
    if m > 16 * 16 * 16:
        # large grids: scalars only (keeps the fixtures small)
        out["nnz"] = np.array(R.nnz, np.int64)
        out["rows"] = np.array(R.nrows, np.int64)
        np.savez_compressed(os.path.join(HERE, f"ref_{nx}x{ny}x{nz}.npz"), **out)
        return out
    out["cg1e9_x"] = r9["x"]
    b, xe = R.rhs()
    out["b"] = b
    x = seeded(m, 1)
    out["spmv_x"] = x
    out["spmv_y"] = R.spmv(0, x)
    r = seeded(m, 2)
    out["symgs_r"] = r
    out["symgs_x"] = R.symgs(0, r, np.zeros(m))
    out["nnz"] = np.array(R.nnz, np.int64)
    out["rows"] = np.array(R.nrows, np.int64)
    cols, vals, nnz = R.matrix(0)
    out["nnz_in_row"] = nnz
    out["cols_checksum"] = np.array([int(cols.astype(np.int64).sum()), int((cols >= 0).sum())], np.int64)
    np.savez_compressed(os.path.join(HERE, f"ref_{nx}x{ny}x{nz}.npz"), **out)
    return out


def make_colored(nx, ny, nz):
    P = ColoredProblem(nx, ny, nz)
    out = {}
    for l, L in enumerate(P.levels):
        out[f"L{l}_colors"] = L.colors
        out[f"L{l}_perm"] = L.perm
        out[f"L{l}_sizes"] = L.sizes
        out[f"L{l}_round_colors"] = L.round_colors
        out[f"L{l}_round_sizes"] = L.round_sizes
    np.savez_compressed(os.path.join(HERE, f"colored_{nx}x{ny}x{nz}.npz"), **out)


def make_big(n):
    """Scalars of the reference CPU path at a full benchmark size (minutes)."""
    R = RefProblem(n, n, n)
    r50 = R.cg(50, 0.0)
    r9 = R.cg(1000, 1e-9)
    np.savez_compressed(os.path.join(HERE, f"ref_{n}x{n}x{n}.npz"), cg50_normr0=r50["normr0"],
                        cg50_normr=r50["normr"], cg50_seconds=r50["seconds"], cg1e9_niters=r9["niters"],
                        cg1e9_normr=r9["normr"], nnz=np.array(R.nnz, np.int64), rows=np.array(R.nrows, np.int64))
    print(n, r50, {k: v for k, v in r9.items() if k != "x"})


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--big":
        make_big(int(sys.argv[2]))
        sys.exit(0)
    for g in GRIDS:
        o = make_ref(*g)
        if g[0] * g[1] * g[2] <= 32 ** 3:
            make_colored(*g)
        print(g, "normr0", o["cg50_normr0"], "iters to 1e-9", o["cg1e9_niters"])
