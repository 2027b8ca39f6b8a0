"""B200-native HPCG multigrid-preconditioned CG.

Python mirror of the reference's operator API over ``libhpcgb200.so`` (C ABI
declared in ``include/hpcg_b200.h``).  The library is CUDA-only: importing
works without a GPU, but every compute call needs the built extension and a
visible device -- there is no CPU fallback.

``Problem`` follows the reference benchmark's set-up sequence
(``src/main.cpp:198-210`` GenerateProblem + 3x GenerateCoarseProblem,
``src/main.cpp:355`` OptimizeProblem) and exposes ``CG`` (``src/CG.cpp:104``),
``TestCG`` (``src/TestCG.cpp:111``), ``TestSymmetry``
(``src/TestSymmetry.cpp:88``) and the per-operator calls.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._lib import LIB_PATH, load, HpcgError, check  # noqa: F401

MODE_FP64 = 0
MODE_MIXED = 1
MODE_LEARNED = 2
MODE_FP64_STENCIL = 3  # FP64 results of MODE_FP64 bit for bit, V-cycle and SpMV on the implicit stencil
FLAG_KEEP_GENERATED = 1
ERR_NONFINITE = 8  # a solve ended with a non-finite residual (HPCGB200_ERR_NONFINITE)

_FIELD_DTYPES = {
    "perm": np.int32, "colors": np.int32, "ell_col": np.int32, "ell_val": np.float64, "diag_idx": np.int32,
    "inv_diag": np.float64, "diag": np.float64, "diag32": np.float32, "inv_diag32": np.float32, "f2c": np.int32,
    "inj_f": np.int32, "inj_c": np.int32, "mtx_ind": np.int32, "values": np.float64, "nnz_in_row": np.int8,
    "hash": np.int32, "diag_slot": np.int32, "l2g": np.int64, "sizes": np.int32, "offsets": np.int32,
    "round_sizes": np.int32, "b": np.float64, "xexact": np.float64, "x": np.float64,
}


def hpcg_model(dims_per_level, nnz_per_level):
    """HPCG flop and memory-traffic model per CG iteration
    (``src/ReportResults.cpp:134-195`` with one CG set and optMaxIters = 1;
    8-byte values, 4-byte indices)."""
    rows = [d[0] * d[1] * d[2] for d in dims_per_level]
    nnz = list(nnz_per_level)
    n0, z0 = rows[0], nnz[0]
    flops = 12.0 * n0 + 2.0 * z0
    rd = 12.0 * n0 * 8 + z0 * 12.0 + n0 * 8
    wr = 3 * 8.0 + 4.0 * n0 * 8
    for lv in range(len(rows) - 1):
        z, n = nnz[lv], rows[lv]
        flops += 4 * z + 2 * z + 4 * z
        rd += (2 * z * 12.0 + n * 8) + (z * 12.0 + n * 8) + (2 * z * 12.0 + n * 8)
        wr += n * 8 + z * 8.0 + z * 8.0
    z, n = nnz[-1], rows[-1]
    flops += 4 * z
    rd += 2 * z * 12.0 + n * 8
    wr += n * 8
    return flops, rd + wr


class Problem:
    """A generated and optimized HPCG hierarchy on the current CUDA device."""

    def __init__(self, nx: int, ny: int | None = None, nz: int | None = None, nlevels: int = 4,
                 keep_generated: bool = False):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.L = load()
        h = ctypes.c_void_p()
        check(self.L, self.L.hpcgb200_problem_create_ex(nx, ny, nz, nlevels,
                                                         FLAG_KEEP_GENERATED if keep_generated else 0,
                                                         ctypes.byref(h)))
        self.h = h
        nl = ctypes.c_int()
        dims = np.zeros(3 * nlevels, np.int32)
        rows = np.zeros(nlevels, np.int32)
        nnz = np.zeros(nlevels, np.int64)
        nb = np.zeros(nlevels, np.int32)
        check(self.L, self.L.hpcgb200_problem_info(self.h, ctypes.byref(nl), _p(dims), _p(rows), _p(nnz), _p(nb)))
        self.nlevels = nl.value
        self.dims = [tuple(int(v) for v in dims[3 * l:3 * l + 3]) for l in range(self.nlevels)]
        self.rows = [int(v) for v in rows]
        self.nnz = [int(v) for v in nnz]
        self.nblocks = [int(v) for v in nb]
        s, o = ctypes.c_double(), ctypes.c_double()
        check(self.L, self.L.hpcgb200_problem_setup_times(self.h, ctypes.byref(s), ctypes.byref(o)))
        self.setup_seconds, self.optimize_seconds = s.value, o.value
        st = ctypes.c_void_p()
        check(self.L, self.L.hpcgb200_problem_stream(self.h, ctypes.byref(st)))
        self.stream_handle = st.value

    def close(self):
        if getattr(self, "h", None):
            self.L.hpcgb200_problem_destroy(self.h)
            self.h = None
            self._smoother = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- data access -------------------------------------------------------
    def field(self, name: str, level: int = 0) -> np.ndarray:
        """Host copy of a level array (device arrays are synchronised first)."""
        dt = np.dtype(_FIELD_DTYPES[name])
        nbytes = ctypes.c_size_t()
        check(self.L, self.L.hpcgb200_problem_field_bytes(self.h, level, name.encode(), ctypes.byref(nbytes)))
        out = np.empty(nbytes.value // dt.itemsize, dt)
        check(self.L, self.L.hpcgb200_problem_copy_field(self.h, level, name.encode(), _p(out), out.nbytes))
        m = self.rows[level]
        if name in ("ell_col", "ell_val"):
            out = out.reshape(27, m)
        elif name in ("mtx_ind", "values"):
            out = out.reshape(m, 27)
        return out

    def device_ptr(self, name: str, level: int = 0) -> int:
        d = ctypes.c_void_p()
        check(self.L, self.L.hpcgb200_problem_device_field(self.h, level, name.encode(), ctypes.byref(d)))
        return d.value

    def stencil_ok(self, level: int = 0) -> bool:
        ok = ctypes.c_int()
        check(self.L, self.L.hpcgb200_problem_stencil_ok(self.h, level, ctypes.byref(ok)))
        return bool(ok.value)

    def set_rhs(self, b_natural: np.ndarray | None):
        if b_natural is None:
            check(self.L, self.L.hpcgb200_problem_set_rhs(self.h, None))
        else:
            b = np.ascontiguousarray(b_natural, np.float64)
            check(self.L, self.L.hpcgb200_problem_set_rhs(self.h, _p(b)))

    def get_x(self) -> np.ndarray:
        x = np.empty(self.rows[0])
        check(self.L, self.L.hpcgb200_problem_get_x(self.h, _p(x)))
        return x

    # -- solver ------------------------------------------------------------
    def cg(self, max_iter: int, tol: float, mode: int = MODE_FP64, precond: bool = True) -> dict:
        it = ctypes.c_int()
        nr, nr0, sec = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        hist = np.zeros(max_iter + 1)
        rc = self.L.hpcgb200_problem_cg(self.h, mode, max_iter, tol, int(precond), ctypes.byref(it), ctypes.byref(nr),
                                        ctypes.byref(nr0), _p(hist), ctypes.byref(sec))
        out = dict(niters=it.value, normr=nr.value, normr0=nr0.value, hist=hist[: it.value + 1], seconds=sec.value)
        if rc != 0:
            err = HpcgError(self.L, rc)
            err.result = out if rc == ERR_NONFINITE else None  # a non-finite end still fills the outputs
            raise err
        return out

    def solve_host(self, b_natural: np.ndarray, x_out: np.ndarray, max_iter: int, tol: float,
                   mode: int = MODE_FP64) -> dict:
        """End-to-end solve from HOST memory (the H2D/D2H copies are inside)."""
        it = ctypes.c_int()
        nr, nr0, sec = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(self.L, self.L.hpcgb200_problem_solve_host(self.h, mode, ctypes.c_void_p(_addr(b_natural)),
                                                         ctypes.c_void_p(_addr(x_out)), max_iter, tol,
                                                         ctypes.byref(it), ctypes.byref(nr), ctypes.byref(nr0),
                                                         ctypes.byref(sec)))
        return dict(niters=it.value, normr=nr.value, normr0=nr0.value, seconds=sec.value)

    def cg_ref(self, max_iter: int, tol: float, precond: bool = True) -> dict:
        """The benchmark's reference CG (src/CG_ref.cpp) in natural order on the
        device; needs a problem created with keep_generated=True.  Leaves x in
        natural order."""
        it = ctypes.c_int()
        nr, nr0, sec = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(self.L, self.L.hpcgb200_problem_cg_ref(self.h, max_iter, tol, int(precond), ctypes.byref(it),
                                                     ctypes.byref(nr), ctypes.byref(nr0), ctypes.byref(sec)))
        return dict(niters=it.value, normr=nr.value, normr0=nr0.value, seconds=sec.value)

    def mg_ref(self, r_ptr: int, z_ptr: int) -> None:
        """z = M^-1 r with the reference V-cycle (src/ComputeMG_ref.cpp), natural
        order, device pointers; needs keep_generated=True."""
        check(self.L, self.L.hpcgb200_problem_mg_ref(self.h, ctypes.c_void_p(r_ptr), ctypes.c_void_p(z_ptr)))

    def true_residual(self) -> float:
        """||b - A x|| / ||b|| of the current solution, computed in FP64."""
        rel = ctypes.c_double()
        check(self.L, self.L.hpcgb200_problem_true_residual(self.h, ctypes.byref(rel)))
        return rel.value

    def kernels_per_iteration(self, mode: int = MODE_FP64, precond: bool = True) -> int:
        k = ctypes.c_int()
        check(self.L, self.L.hpcgb200_problem_kernels_per_iteration(self.h, mode, int(precond), ctypes.byref(k)))
        return k.value

    def test_cg(self, mode: int = MODE_FP64) -> dict:
        n = np.zeros(4, np.int32)
        cp, cf = ctypes.c_int(), ctypes.c_int()
        check(self.L, self.L.hpcgb200_problem_test_cg(self.h, mode, _p(n), ctypes.byref(cp), ctypes.byref(cf)))
        return dict(niters=[int(v) for v in n], count_pass=cp.value, count_fail=cf.value)

    def test_symmetry(self, mode: int = MODE_FP64) -> dict:
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(self.L, self.L.hpcgb200_problem_test_symmetry(self.h, mode, ctypes.byref(a), ctypes.byref(b),
                                                            ctypes.byref(c)))
        return dict(depsym_spmv=a.value, depsym_mg=b.value, residual_inf=c.value)

    # -- per-operator calls on device pointers (permuted order) -------------
    def spmv(self, level: int, x_ptr: int, y_ptr: int):
        check(self.L, self.L.hpcgb200_problem_spmv(self.h, level, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr)))

    def spmv_stencil(self, level: int, x_ptr: int, y_ptr: int):
        check(self.L, self.L.hpcgb200_problem_spmv_stencil(self.h, level, ctypes.c_void_p(x_ptr),
                                                           ctypes.c_void_p(y_ptr)))

    def spmv_mixed(self, level: int, x_ptr: int, y_ptr: int):
        """The mixed path's outer FP64 operator (separable sum; equal to the ELL
        product to rounding)."""
        check(self.L, self.L.hpcgb200_problem_spmv_mixed(self.h, level, ctypes.c_void_p(x_ptr),
                                                         ctypes.c_void_p(y_ptr)))

    def symgs(self, level: int, r_ptr: int, x_ptr: int):
        check(self.L, self.L.hpcgb200_problem_symgs(self.h, level, ctypes.c_void_p(r_ptr), ctypes.c_void_p(x_ptr)))

    def symgs_zero(self, level: int, r_ptr: int, x_ptr: int):
        check(self.L, self.L.hpcgb200_problem_symgs_zero(self.h, level, ctypes.c_void_p(r_ptr),
                                                         ctypes.c_void_p(x_ptr)))

    def mg(self, r_ptr: int, x_ptr: int, mode: int = MODE_FP64):
        check(self.L, self.L.hpcgb200_problem_mg(self.h, mode, ctypes.c_void_p(r_ptr), ctypes.c_void_p(x_ptr)))

    def restrict(self, level: int, rf_ptr: int, xf_ptr: int, rc_ptr: int):
        check(self.L, self.L.hpcgb200_problem_restrict(self.h, level, ctypes.c_void_p(rf_ptr), ctypes.c_void_p(xf_ptr),
                                                       ctypes.c_void_p(rc_ptr)))

    def prolong(self, level: int, xc_ptr: int, xf_ptr: int):
        check(self.L, self.L.hpcgb200_problem_prolong(self.h, level, ctypes.c_void_p(xc_ptr), ctypes.c_void_p(xf_ptr)))

    # -- learned smoother --------------------------------------------------
    def set_smoother(self, smoother, first_level: int = 2, coarse_steps: int = 1):
        """Attach a ``rochpcg_b200.learned.Smoother`` to levels >= first_level
        for MODE_LEARNED (None detaches); coarse_steps learned Richardson steps
        replace the coarsest level's SymGS."""
        if smoother is None:
            check(self.L, self.L.hpcgb200_problem_set_smoother(self.h, None, 0, 0))
            self._smoother = None
        else:
            check(self.L, self.L.hpcgb200_problem_set_smoother(self.h, smoother.h, first_level, coarse_steps))
            self._smoother = smoother  # kept alive while attached

    def set_fallback(self, jump: float = 2.0, stall: int = 16, window: int = 16, rate: float = 0.8):
        """Failure rule of the learned solve (see hpcgb200_problem_set_fallback)."""
        check(self.L, self.L.hpcgb200_problem_set_fallback(self.h, jump, stall, window, rate))

    # named failure rules of the learned solve: "first-increase" falls back at
    # the first iteration that does not reduce the FP64 residual norm (the
    # literal rule); "default" on a jump (x2), a 16-iteration stall without a
    # new minimum, or less than 20 % reduction over 16 iterations (PCG's
    # residual norm is not monotone, so single small increases are tolerated)
    FALLBACK_RULES = {"first-increase": (1.0, 10 ** 6, 16, 0.0), "default": (2.0, 16, 16, 0.8)}

    def set_fallback_rule(self, name: str):
        """Select a named failure rule of the learned solve (FALLBACK_RULES)."""
        self.set_fallback(*self.FALLBACK_RULES[name])

    def last_fallback(self) -> int:
        """Iteration at which the last MODE_LEARNED solve fell back to SymGS (0: never)."""
        it = ctypes.c_int()
        check(self.L, self.L.hpcgb200_problem_last_fallback(self.h, ctypes.byref(it)))
        return it.value

    def time_op(self, op: str, n: int) -> float:
        ms = ctypes.c_double()
        check(self.L, self.L.hpcgb200_problem_time_op(self.h, op.encode(), n, ctypes.byref(ms)))
        return ms.value

    def model(self):
        return hpcg_model(self.dims, self.nnz)


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _addr(a) -> int:
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())  # torch tensor (e.g. pinned host memory)
