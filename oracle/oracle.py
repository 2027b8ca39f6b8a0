"""Python access to the two CPU oracles.  TEST INFRASTRUCTURE ONLY.

* :class:`RefProblem` drives ``oracle/_ref/libhpcg_ref.so`` -- the reference's
  own CPU path (``CG_ref``, ``ComputeMG_ref``, ``ComputeSYMGS_ref`` ...)
  compiled unmodified from rocHPCG 0.8.9 ``src/*_ref.cpp`` by
  ``oracle/Makefile``.
* :class:`ColoredProblem` drives ``oracle/liboracle.so`` -- our C restatement
  of the reference's *optimized* path (JPL multicoloring, permutation,
  column-major ELL, colored SymGS; see ``oracle/colored.h`` for the per-kernel
  citations).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libhpcg_ref.so")
# the same reference sources built without HPCG_CONTIGUOUS_ARRAYS (per-row
# arrays) and with NDEBUG: the contiguous build computes rows * 27 in 32-bit
# int (src/GenerateProblem_ref.cpp:115-117), and the int nonzero count's
# overflow check (:204) aborts above 2^31 nonzeros; this build serves the grids
# past those limits (560 x 560 x 280), where only ComputeSPMV_ref is called
REF_ROWS_SO = os.path.join(HERE, "_ref", "libhpcg_ref_rows.so")
INT_MAX = 0x7FFFFFFF
COLORED_SO = os.path.join(HERE, "liboracle.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)


def reference_tree() -> str | None:
    """The rocHPCG source tree the reference oracle is compiled from:
    $HPCG_REFERENCE_DIR, else a directory named ``reference`` beside the
    repository; None when neither holds ``src/CG_ref.cpp``."""
    cands = [os.environ.get("HPCG_REFERENCE_DIR"),
             os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")]
    for c in cands:
        if c and os.path.isfile(os.path.join(c, "src", "CG_ref.cpp")):
            return os.path.abspath(c)
    return None


def build(ref: bool = True) -> None:
    """Compile the oracle libraries (the reference one only where its source tree exists)."""
    subprocess.check_call(["make", "-s", "-C", HERE])
    tree = reference_tree() if ref else None
    if tree:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", "REF=" + tree])


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------
# reference CPU path


_ref_libs: dict = {}


def ref_lib(rows: bool = False):
    """The reference CPU library: contiguous arrays (the reference build's
    setting), or per-row arrays for grids whose 27 * rows exceeds INT_MAX."""
    so = REF_ROWS_SO if rows else REF_SO
    if so not in _ref_libs:
        if not os.path.exists(so):
            raise FileNotFoundError(f"{so} missing: run `make -C oracle ref` where the reference tree exists")
        L = ctypes.CDLL(so)
        L.hpcgref_create.restype = ctypes.c_void_p
        L.hpcgref_create.argtypes = [ctypes.c_int] * 4
        L.hpcgref_destroy.argtypes = [ctypes.c_void_p]
        L.hpcgref_num_levels.argtypes = [ctypes.c_void_p]
        L.hpcgref_level_info.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, _c_int_p,
                                         ctypes.POINTER(ctypes.c_longlong)]
        L.hpcgref_get_matrix.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 3
        L.hpcgref_get_f2c.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.hpcgref_get_rhs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.hpcgref_check_problem.argtypes = [ctypes.c_void_p]
        L.hpcgref_cg.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_int, _c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]
        for name in ("hpcgref_spmv", "hpcgref_symgs", "hpcgref_mg"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.hpcgref_restriction.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 3
        L.hpcgref_prolongation.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 2
        L.hpcgref_dot.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, _c_dbl_p]
        L.hpcgref_waxpby.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_double,
                                     ctypes.c_void_p, ctypes.c_void_p]
        L.hpcgref_residual.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, _c_dbl_p]
        L.hpcgref_test_norms.argtypes = [ctypes.c_void_p, ctypes.c_int, _c_dbl_p, _c_dbl_p, _c_int_p]
        L.hpcgref_optimal_shape.argtypes = [ctypes.c_int, _c_int_p, _c_int_p, _c_int_p]
        L.hpcgref_optimal_shape.restype = None
        L.hpcgref_rank_problem.argtypes = [ctypes.c_int] * 5 + [ctypes.c_void_p] * 5
        L.hpcgref_geometry.argtypes = [ctypes.c_int] * 11 + [ctypes.c_void_p]
        L.hpcgref_geometry.restype = None
        _ref_libs[so] = L
    return _ref_libs[so]


def ref_optimal_shape(size: int) -> tuple[int, int, int]:
    """The reference's own process grid (src/ComputeOptimalShapeXYZ.cpp)."""
    L = ref_lib()
    x, y, z = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.hpcgref_optimal_shape(size, ctypes.byref(x), ctypes.byref(y), ctypes.byref(z))
    return x.value, y.value, z.value


def ref_geometry(size, rank, pz, zl, zu, nx, ny, nz, npx=0, npy=0, npz=0) -> list[int]:
    """The reference's GenerateGeometry (src/GenerateGeometry.cpp)."""
    out = np.zeros(13, np.int64)
    ref_lib().hpcgref_geometry(size, rank, pz, zl, zu, nx, ny, nz, npx, npy, npz, _ptr(out))
    return [int(v) for v in out]


def ref_rank_problem(size: int, rank: int, nx: int, ny: int, nz: int) -> dict:
    """Rank `rank` of a `size`-rank run as the reference generates it
    (src/GenerateGeometry.cpp + src/GenerateProblem_ref.cpp): per natural row
    the GLOBAL column ids (-1 padded), values, nonzero count and b."""
    L = ref_lib()
    m = nx * ny * nz
    gcols = np.empty((m, 27), np.int64)
    vals = np.empty((m, 27), np.float64)
    nnz = np.empty(m, np.int8)
    b = np.empty(m, np.float64)
    grid = np.zeros(6, np.int32)
    assert L.hpcgref_rank_problem(size, rank, nx, ny, nz, _ptr(gcols), _ptr(vals), _ptr(nnz), _ptr(b), _ptr(grid)) == 0
    return {"gcols": gcols, "vals": vals, "nnz": nnz, "b": b, "grid": tuple(int(v) for v in grid)}


class RefProblem:
    """The reference CPU problem (natural ordering): GenerateProblem_ref +
    SetupHalo_ref + 3 coarse levels, solved by CG_ref."""

    def __init__(self, nx: int, ny: int, nz: int, nlevels: int = 4):
        self.L = ref_lib(rows=27 * nx * ny * nz > INT_MAX)
        self.h = self.L.hpcgref_create(nx, ny, nz, nlevels)
        if not self.h:
            raise ValueError("hpcgref_create failed")
        self.nlevels = self.L.hpcgref_num_levels(self.h)
        self.dims, self.nrows, self.nnz = [], [], []
        for l in range(self.nlevels):
            d = np.zeros(3, np.int32)
            m = ctypes.c_int()
            nnz = ctypes.c_longlong()
            self.L.hpcgref_level_info(self.h, l, _ptr(d), ctypes.byref(m), ctypes.byref(nnz))
            self.dims.append(tuple(int(v) for v in d))
            self.nrows.append(m.value)
            self.nnz.append(nnz.value)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.hpcgref_destroy(self.h)
            self.h = None

    def matrix(self, level: int = 0):
        m = self.nrows[level]
        cols = np.empty((m, 27), np.int32)
        vals = np.empty((m, 27), np.float64)
        nnz = np.empty(m, np.int8)
        self.L.hpcgref_get_matrix(self.h, level, _ptr(cols), _ptr(vals), _ptr(nnz))
        return cols, vals, nnz

    def f2c(self, level: int):
        out = np.empty(self.nrows[level + 1], np.int32)
        assert self.L.hpcgref_get_f2c(self.h, level, _ptr(out)) == 0
        return out

    def rhs(self):
        b = np.empty(self.nrows[0])
        xe = np.empty(self.nrows[0])
        self.L.hpcgref_get_rhs(self.h, _ptr(b), _ptr(xe))
        return b, xe

    def check_problem(self):
        self.L.hpcgref_check_problem(self.h)

    def cg(self, max_iter: int, tol: float, b: np.ndarray | None = None, precond: bool = True):
        x = np.empty(self.nrows[0])
        it = ctypes.c_int()
        nr, nr0, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        bb = None if b is None else np.ascontiguousarray(b, np.float64)
        self.L.hpcgref_cg(self.h, max_iter, tol, None if bb is None else _ptr(bb), _ptr(x), int(precond),
                          ctypes.byref(it), ctypes.byref(nr), ctypes.byref(nr0), ctypes.byref(t))
        return dict(x=x, niters=it.value, normr=nr.value, normr0=nr0.value, seconds=t.value)

    def spmv(self, level: int, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.nrows[level])
        self.L.hpcgref_spmv(self.h, level, _ptr(x), _ptr(y))
        return y

    def symgs(self, level: int, r: np.ndarray, x: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float64)
        x = np.array(x, np.float64, copy=True)
        self.L.hpcgref_symgs(self.h, level, _ptr(r), _ptr(x))
        return x

    def mg(self, r: np.ndarray, level: int = 0) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float64)
        x = np.zeros(self.nrows[level])
        self.L.hpcgref_mg(self.h, level, _ptr(r), _ptr(x))
        return x

    def restriction(self, level: int, rf: np.ndarray, xf: np.ndarray) -> np.ndarray:
        rf = np.ascontiguousarray(rf, np.float64)
        xf = np.ascontiguousarray(xf, np.float64)
        rc = np.empty(self.nrows[level + 1])
        assert self.L.hpcgref_restriction(self.h, level, _ptr(rf), _ptr(xf), _ptr(rc)) == 0
        return rc

    def prolongation(self, level: int, xc: np.ndarray, xf: np.ndarray) -> np.ndarray:
        xc = np.ascontiguousarray(xc, np.float64)
        xf = np.array(xf, np.float64, copy=True)
        assert self.L.hpcgref_prolongation(self.h, level, _ptr(xc), _ptr(xf)) == 0
        return xf


def ref_test_norms(values) -> dict:
    v = np.ascontiguousarray(values, np.float64)
    mean, var, ok = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    ref_lib().hpcgref_test_norms(_ptr(v), len(v), ctypes.byref(mean), ctypes.byref(var), ctypes.byref(ok))
    return dict(mean=mean.value, variance=var.value, pass_=bool(ok.value))


# --------------------------------------------------------------------------
# colored (optimized-path) restatement


class _OcLevel(ctypes.Structure):
    _fields_ = [
        ("m", ctypes.c_int), ("nblocks", ctypes.c_int), ("ublocks", ctypes.c_int),
        ("sizes", ctypes.c_void_p), ("offsets", ctypes.c_void_p), ("ell_col", ctypes.c_void_p),
        ("ell_val", ctypes.c_void_p), ("diag_idx", ctypes.c_void_p), ("inv_diag", ctypes.c_void_p),
        ("nc", ctypes.c_int), ("f2c", ctypes.c_void_p), ("perm", ctypes.c_void_p), ("perm_c", ctypes.c_void_p),
        ("rc", ctypes.c_void_p), ("xc", ctypes.c_void_p),
    ]


_oc_lib = None


def colored_lib():
    global _oc_lib
    if _oc_lib is None:
        if not os.path.exists(COLORED_SO):
            build(ref=False)
        L = ctypes.CDLL(COLORED_SO)
        vp = ctypes.c_void_p
        L.oc_generate.argtypes = [ctypes.c_int] * 3 + [vp] * 6
        L.oc_f2c.argtypes = [ctypes.c_int] * 3 + [vp]
        L.oc_jpl_coloring.argtypes = [ctypes.c_int] + [vp] * 6
        L.oc_jpl_coloring.restype = ctypes.c_int
        L.oc_color_perm.argtypes = [ctypes.c_int, vp, ctypes.c_int, vp, vp, vp]
        L.oc_build_ell.argtypes = [ctypes.c_int] + [vp] * 7
        L.oc_permute_vector.argtypes = [ctypes.c_int, vp, vp, vp]
        L.oc_spmv.argtypes = [ctypes.c_int, vp, vp, vp, vp]
        L.oc_symgs.argtypes = [ctypes.c_int] * 3 + [vp] * 7
        L.oc_symgs_zero.argtypes = [ctypes.c_int] * 3 + [vp] * 7
        L.oc_restrict_fused.argtypes = [ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp, vp]
        L.oc_prolong.argtypes = [ctypes.c_int] + [vp] * 5
        L.oc_dot.argtypes = [ctypes.c_int, vp, vp]
        L.oc_dot.restype = ctypes.c_double
        L.oc_mg.argtypes = [vp, ctypes.c_int, vp, vp]
        L.oc_mg_f32.argtypes = [vp, ctypes.c_int, vp, vp]
        L.oc_cg.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                            _c_int_p, _c_dbl_p, _c_dbl_p, vp]
        L.oc_bf16.argtypes = [ctypes.c_float]
        L.oc_bf16.restype = ctypes.c_float
        L.oc_conv16.argtypes = [ctypes.c_int] * 3 + [vp, vp, vp, ctypes.c_int]
        L.oc_flip_transpose.argtypes = [vp, vp]
        L.oc_conv16_wgrad.argtypes = [ctypes.c_int] * 3 + [vp, vp, vp, ctypes.c_int]
        L.oc_net_forward.argtypes = [ctypes.c_int] * 3 + [vp] * 7 + [ctypes.c_int]
        L.oc_net_loss_grad.argtypes = [ctypes.c_int] * 3 + [vp] * 8 + [ctypes.c_int]
        L.oc_net_loss_grad.restype = ctypes.c_double
        L.oc_net_loss_grad2.argtypes = [ctypes.c_int] * 3 + [vp] * 8 + [ctypes.c_int] * 3
        L.oc_net_loss_grad2.restype = ctypes.c_double
        L.oc_stencil_apply.argtypes = [ctypes.c_int] * 3 + [vp, vp]
        _oc_lib = L
    return _oc_lib


class ColoredLevel:
    """One level of the optimized data: natural-order generated matrix, JPL
    colors, permutation, column-major ELL and diagonal data."""

    def __init__(self, nx: int, ny: int, nz: int, with_rhs: bool = False):
        L = colored_lib()
        self.dims = (nx, ny, nz)
        m = self.m = nx * ny * nz
        self.cols = np.empty((m, 27), np.int32)
        self.vals = np.empty((m, 27), np.float64)
        self.nnz_in_row = np.empty(m, np.int8)
        self.diag_slot = np.empty(m, np.int32)
        self.hash = np.empty(m, np.int32)
        self.b_nat = np.empty(m) if with_rhs else None
        L.oc_generate(nx, ny, nz, _ptr(self.cols), _ptr(self.vals), _ptr(self.nnz_in_row), _ptr(self.diag_slot),
                      _ptr(self.hash), None if self.b_nat is None else _ptr(self.b_nat))
        self.colors = np.empty(m, np.int32)
        self.round_colors = np.zeros(256, np.int32)
        self.round_sizes = np.zeros(256, np.int32)
        nb = L.oc_jpl_coloring(m, _ptr(self.cols), _ptr(self.nnz_in_row), _ptr(self.hash), _ptr(self.colors),
                               _ptr(self.round_colors), _ptr(self.round_sizes))
        if nb < 0:
            raise RuntimeError("JPL coloring did not terminate")
        self.nblocks = nb
        self.ublocks = nb - 2  # MultiColoring.cpp:316,350-352 (non-reference build)
        self.round_colors = self.round_colors[:nb].copy()
        self.round_sizes = self.round_sizes[:nb].copy()
        self.perm = np.empty(m, np.int32)
        self.sizes = np.zeros(max(nb, int(self.colors.max()) + 1), np.int32)
        self.offsets = np.zeros(len(self.sizes) + 1, np.int32)
        L.oc_color_perm(m, _ptr(self.colors), len(self.sizes), _ptr(self.perm), _ptr(self.sizes), _ptr(self.offsets))
        self.ell_col = np.empty((27, m), np.int32)
        self.ell_val = np.empty((27, m), np.float64)
        self.diag_idx = np.empty(m, np.int32)
        self.inv_diag = np.empty(m, np.float64)
        L.oc_build_ell(m, _ptr(self.cols), _ptr(self.vals), _ptr(self.perm), _ptr(self.ell_col), _ptr(self.ell_val),
                       _ptr(self.diag_idx), _ptr(self.inv_diag))
        self.f2c = None
        self.nc = 0

    def permute(self, v: np.ndarray) -> np.ndarray:
        out = np.empty_like(v)
        out[self.perm] = v
        return out

    def unpermute(self, v: np.ndarray) -> np.ndarray:
        return v[self.perm]

    def spmv(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.m)
        colored_lib().oc_spmv(self.m, _ptr(self.ell_col), _ptr(self.ell_val), _ptr(x), _ptr(y))
        return y

    def symgs(self, r, x):
        r = np.ascontiguousarray(r, np.float64)
        x = np.array(x, np.float64, copy=True)
        colored_lib().oc_symgs(self.m, self.nblocks, self.ublocks, _ptr(self.sizes), _ptr(self.offsets),
                               _ptr(self.ell_col), _ptr(self.ell_val), _ptr(self.inv_diag), _ptr(r), _ptr(x))
        return x

    def symgs_zero(self, r):
        r = np.ascontiguousarray(r, np.float64)
        x = np.zeros(self.m)
        colored_lib().oc_symgs_zero(self.m, self.nblocks, self.ublocks, _ptr(self.sizes), _ptr(self.offsets),
                                    _ptr(self.ell_col), _ptr(self.ell_val), _ptr(self.diag_idx), _ptr(r), _ptr(x))
        return x


class ColoredProblem:
    """4-level optimized hierarchy (all vectors in color-permuted order)."""

    def __init__(self, nx: int, ny: int, nz: int, nlevels: int = 4):
        self.levels = [ColoredLevel(nx, ny, nz, with_rhs=True)]
        for l in range(1, nlevels):
            f = self.levels[-1]
            fx, fy, fz = f.dims
            f.f2c = np.empty((fx // 2) * (fy // 2) * (fz // 2), np.int32)
            colored_lib().oc_f2c(fx, fy, fz, _ptr(f.f2c))
            f.nc = len(f.f2c)
            self.levels.append(ColoredLevel(fx // 2, fy // 2, fz // 2))
        self.nlevels = nlevels
        L0 = self.levels[0]
        self.b = L0.permute(L0.b_nat)
        self.xexact = np.ones(L0.m)
        self._bufs = []
        self._struct = (_OcLevel * nlevels)()
        for l, lev in enumerate(self.levels):
            s = self._struct[l]
            s.m, s.nblocks, s.ublocks = lev.m, lev.nblocks, lev.ublocks
            s.sizes, s.offsets = _ptr(lev.sizes).value, _ptr(lev.offsets).value
            s.ell_col, s.ell_val = _ptr(lev.ell_col).value, _ptr(lev.ell_val).value
            s.diag_idx, s.inv_diag = _ptr(lev.diag_idx).value, _ptr(lev.inv_diag).value
            s.perm = _ptr(lev.perm).value
            if l + 1 < nlevels:
                rc, xc = np.zeros(lev.nc), np.zeros(lev.nc)
                self._bufs += [rc, xc]
                s.nc, s.f2c = lev.nc, _ptr(lev.f2c).value
                s.perm_c = _ptr(self.levels[l + 1].perm).value
                s.rc, s.xc = _ptr(rc).value, _ptr(xc).value

    def restrict_fused(self, level: int, rf, xf):
        A, C = self.levels[level], self.levels[level + 1]
        rf = np.ascontiguousarray(rf, np.float64)
        xf = np.ascontiguousarray(xf, np.float64)
        rc = np.empty(C.m)
        colored_lib().oc_restrict_fused(A.nc, _ptr(A.f2c), _ptr(A.perm), _ptr(C.perm), A.m, _ptr(A.ell_col),
                                        _ptr(A.ell_val), _ptr(rf), _ptr(xf), _ptr(rc))
        return rc

    def prolong(self, level: int, xc, xf):
        A, C = self.levels[level], self.levels[level + 1]
        xc = np.ascontiguousarray(xc, np.float64)
        xf = np.array(xf, np.float64, copy=True)
        colored_lib().oc_prolong(A.nc, _ptr(A.f2c), _ptr(A.perm), _ptr(C.perm), _ptr(xc), _ptr(xf))
        return xf

    def mg(self, r):
        r = np.ascontiguousarray(r, np.float64)
        x = np.zeros(self.levels[0].m)
        colored_lib().oc_mg(ctypes.cast(self._struct, ctypes.c_void_p), self.nlevels, _ptr(r), _ptr(x))
        return x

    def mg_f32(self, r):
        r = np.ascontiguousarray(r, np.float32)
        x = np.zeros(self.levels[0].m, np.float32)
        colored_lib().oc_mg_f32(ctypes.cast(self._struct, ctypes.c_void_p), self.nlevels, _ptr(r), _ptr(x))
        return x

    def cg(self, max_iter: int, tol: float, b=None, precond: bool = True):
        b = self.b if b is None else np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.levels[0].m)
        hist = np.zeros(max_iter + 1)
        it = ctypes.c_int()
        nr, nr0 = ctypes.c_double(), ctypes.c_double()
        colored_lib().oc_cg(ctypes.cast(self._struct, ctypes.c_void_p), self.nlevels, _ptr(b), _ptr(x), max_iter, tol,
                            int(precond), ctypes.byref(it), ctypes.byref(nr), ctypes.byref(nr0), _ptr(hist))
        return dict(x=x, niters=it.value, normr=nr.value, normr0=nr0.value, hist=hist[: it.value + 1])


# --------------------------------------------------------------------------
# learned smoother (conv net) restatement


def _dist_lib():
    L = colored_lib()
    if not getattr(L, "_od_ready", False):
        vp, ci = ctypes.c_void_p, ctypes.c_int
        L.od_shape.argtypes = [ci, _c_int_p, _c_int_p, _c_int_p]
        L.od_create.argtypes = [ci] * 8
        L.od_create.restype = vp
        L.od_destroy.argtypes = [vp]
        L.od_level_info.argtypes = [vp, ci, ci, vp]
        for name in ("od_level_perm", "od_level_ext_gid"):
            getattr(L, name).argtypes = [vp, ci, ci, vp]
        L.od_level_ell.argtypes = [vp, ci, ci, vp, vp]
        L.od_level_b.argtypes = [vp, ci, vp]
        L.od_exchange.argtypes = [vp, ci, vp]
        for name in ("od_spmv", "od_symgs", "od_symgs_zero"):
            getattr(L, name).argtypes = [vp, ci, vp, vp]
        L.od_restrict.argtypes = [vp, ci, vp, vp, vp]
        L.od_mg.argtypes = [vp, vp, vp]
        L.od_cg.argtypes = [vp, ci, ctypes.c_double, ci, vp, vp, _c_int_p, _c_dbl_p, _c_dbl_p, vp]
        for name in ("od_shape", "od_destroy", "od_level_info", "od_level_perm", "od_level_ext_gid", "od_level_ell",
                     "od_level_b", "od_exchange", "od_spmv", "od_symgs", "od_symgs_zero", "od_restrict", "od_mg",
                     "od_cg"):
            getattr(L, name).restype = None
        L._od_ready = True
    return L


def od_shape(size: int) -> tuple[int, int, int]:
    L = _dist_lib()
    x, y, z = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.od_shape(size, ctypes.byref(x), ctypes.byref(y), ctypes.byref(z))
    return x.value, y.value, z.value


def _vec_ptrs(vs):
    return (ctypes.c_void_p * len(vs))(*[v.ctypes.data for v in vs])


class DistOracle:
    """Every rank of a decomposed problem (oracle/distributed.c): per-rank
    level data and the operators over all ranks, vectors as lists of numpy
    arrays in each rank's permuted order (x-type ones with the external tail)."""

    def __init__(self, size: int, nx: int, ny: int, nz: int, nlevels: int = 4, grid=None):
        self.L = _dist_lib()
        npx, npy, npz = grid if grid else (0, 0, 0)
        self.h = self.L.od_create(size, npx, npy, npz, nx, ny, nz, nlevels)
        if not self.h:
            raise ValueError("od_create: process grid does not match size")
        self.size, self.nlevels = size, nlevels
        self.info = []
        for r in range(size):
            per = []
            for l in range(nlevels):
                v = np.zeros(8, np.int32)
                self.L.od_level_info(self.h, r, l, _ptr(v))
                per.append(dict(zip(("m", "next", "nblocks", "ublocks", "nhalo", "nx", "ny", "nz"),
                                    (int(a) for a in v))))
                per[-1]["ncols"] = per[-1]["m"] + per[-1]["next"]
            self.info.append(per)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.od_destroy(self.h)
            self.h = None

    def perm(self, rank: int, level: int = 0) -> np.ndarray:
        out = np.empty(self.info[rank][level]["m"], np.int32)
        self.L.od_level_perm(self.h, rank, level, _ptr(out))
        return out

    def ell(self, rank: int, level: int = 0):
        m = self.info[rank][level]["m"]
        col = np.empty((27, m), np.int32)
        val = np.empty((27, m), np.float64)
        self.L.od_level_ell(self.h, rank, level, _ptr(col), _ptr(val))
        return col, val

    def ext_gid(self, rank: int, level: int = 0) -> np.ndarray:
        out = np.empty(self.info[rank][level]["next"], np.int64)
        self.L.od_level_ext_gid(self.h, rank, level, _ptr(out))
        return out

    def b(self, rank: int) -> np.ndarray:
        out = np.empty(self.info[rank][0]["m"], np.float64)
        self.L.od_level_b(self.h, rank, _ptr(out))
        return out

    def _xs(self, level, xs):
        out = []
        for r, x in enumerate(xs):
            v = np.zeros(self.info[r][level]["ncols"])
            v[:len(x)] = x
            out.append(v)
        return out

    def spmv(self, level: int, xs):
        xs = self._xs(level, xs)
        ys = [np.empty(self.info[r][level]["m"]) for r in range(self.size)]
        self.L.od_spmv(self.h, level, _vec_ptrs(xs), _vec_ptrs(ys))
        return ys

    def symgs(self, level: int, rs, xs):
        rs = [np.ascontiguousarray(r, np.float64) for r in rs]
        xs = self._xs(level, xs)
        self.L.od_symgs(self.h, level, _vec_ptrs(rs), _vec_ptrs(xs))
        return [x[:self.info[r][level]["m"]] for r, x in enumerate(xs)]

    def restrict(self, level: int, rfs, xfs):
        rfs = [np.ascontiguousarray(r, np.float64) for r in rfs]
        xfs = self._xs(level, xfs)
        rcs = [np.empty(self.info[r][level + 1]["m"]) for r in range(self.size)]
        self.L.od_restrict(self.h, level, _vec_ptrs(rfs), _vec_ptrs(xfs), _vec_ptrs(rcs))
        return rcs

    def mg(self, rs):
        rs = [np.ascontiguousarray(r, np.float64) for r in rs]
        xs = [np.zeros(self.info[r][0]["ncols"]) for r in range(self.size)]
        self.L.od_mg(self.h, _vec_ptrs(rs), _vec_ptrs(xs))
        return [x[:self.info[r][0]["m"]] for r, x in enumerate(xs)]

    def cg(self, max_iter: int, tol: float, precond: bool = True, bs=None) -> dict:
        xs = [np.zeros(self.info[r][0]["m"]) for r in range(self.size)]
        hist = np.zeros(max_iter + 1)
        it = ctypes.c_int()
        nr, nr0 = ctypes.c_double(), ctypes.c_double()
        bptr = None
        if bs is not None:
            bs = [np.ascontiguousarray(b, np.float64) for b in bs]
            bptr = _vec_ptrs(bs)
        self.L.od_cg(self.h, max_iter, tol, 1 if precond else 0, bptr, _vec_ptrs(xs), ctypes.byref(it),
                     ctypes.byref(nr), ctypes.byref(nr0), _ptr(hist))
        return {"niters": it.value, "normr": nr.value, "normr0": nr0.value, "hist": hist[:it.value + 1], "x": xs}


def _dist_ref_lib():
    L = _dist_lib()
    if not getattr(L, "_odr_ready", False):
        vp, ci = ctypes.c_void_p, ctypes.c_int
        L.odr_create.argtypes = [ci] * 8
        L.odr_create.restype = vp
        L.odr_destroy.argtypes = [vp]
        L.odr_spmv.argtypes = [vp, ci, vp, vp]
        L.odr_symgs.argtypes = [vp, ci, vp, vp]
        L.odr_mg.argtypes = [vp, vp, vp]
        L.odr_cg.argtypes = [vp, ci, ctypes.c_double, ci, _c_int_p, _c_dbl_p, _c_dbl_p, vp]
        for name in ("odr_destroy", "odr_spmv", "odr_symgs", "odr_mg", "odr_cg"):
            getattr(L, name).restype = None
        L._odr_ready = True
    return L


class DistRefOracle:
    """The reference's natural-order `_ref` path over a decomposition
    (oracle/distributed_ref.c): vectors hold every rank's rows, rank after
    rank, each in natural order.  `cg(50, 0.0)` gives the tolerance that
    src/test_rochpcg.cpp:262-271 fixes before it runs the optimized CG."""

    def __init__(self, size: int, nx: int, ny: int, nz: int, nlevels: int = 4, grid=None):
        self.L = _dist_ref_lib()
        npx, npy, npz = grid if grid else (0, 0, 0)
        self.h = self.L.odr_create(size, npx, npy, npz, nx, ny, nz, nlevels)
        if not self.h:
            raise ValueError("odr_create: process grid does not match size, or a level is empty")
        self.size, self.m = size, nx * ny * nz
        self.dims = [(nx >> l, ny >> l, nz >> l) for l in range(nlevels)]

    def __del__(self):
        if getattr(self, "h", None):
            self.L.odr_destroy(self.h)
            self.h = None

    def rows(self, level: int = 0) -> int:
        nx, ny, nz = self.dims[level]
        return self.size * nx * ny * nz

    def spmv(self, level: int, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.rows(level))
        self.L.odr_spmv(self.h, level, _ptr(x), _ptr(y))
        return y

    def symgs(self, level: int, r: np.ndarray, x: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float64)
        x = np.array(x, np.float64)
        self.L.odr_symgs(self.h, level, _ptr(r), _ptr(x))
        return x

    def mg(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float64)
        x = np.zeros(self.rows(0))
        self.L.odr_mg(self.h, _ptr(r), _ptr(x))
        return x

    def cg(self, max_iter: int, tol: float, precond: bool = True) -> dict:
        hist = np.zeros(max_iter + 1)
        it = ctypes.c_int()
        nr, nr0 = ctypes.c_double(), ctypes.c_double()
        self.L.odr_cg(self.h, max_iter, tol, 1 if precond else 0, ctypes.byref(it), ctypes.byref(nr),
                      ctypes.byref(nr0), _ptr(hist))
        return {"niters": it.value, "normr": nr.value, "normr0": nr0.value, "hist": hist[:it.value + 1]}


def bf16(a: np.ndarray) -> np.ndarray:
    """fp32 -> bf16 (round to nearest even) -> fp32, vectorised like oc_bf16."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def conv16(dims, x, w, round_=True):
    nz, ny, nx = dims
    x = np.ascontiguousarray(x, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    out = np.empty_like(x)
    colored_lib().oc_conv16(nz, ny, nx, _ptr(x), _ptr(w), _ptr(out), int(round_))
    return out


def flip_transpose(w):
    w = np.ascontiguousarray(w, np.float32)
    out = np.empty_like(w)
    colored_lib().oc_flip_transpose(_ptr(w), _ptr(out))
    return out


def conv16_wgrad(dims, x, g, round_=True):
    nz, ny, nx = dims
    x = np.ascontiguousarray(x, np.float32)
    g = np.ascontiguousarray(g, np.float32)
    dw = np.empty(27 * 16 * 16, np.float32)
    colored_lib().oc_conv16_wgrad(nz, ny, nx, _ptr(x), _ptr(g), _ptr(dw), int(round_))
    return dw


def net_forward(dims, w1, w2, w3, r, round_=True):
    nz, ny, nx = dims
    n = nz * ny * nx
    r = np.ascontiguousarray(r, np.float32)
    ws = [np.ascontiguousarray(w, np.float32) for w in (w1, w2, w3)]
    y = np.empty(n, np.float32)
    a1 = np.empty(n * 16, np.float32)
    a2 = np.empty(n * 16, np.float32)
    colored_lib().oc_net_forward(nz, ny, nx, *[_ptr(w) for w in ws], _ptr(r), _ptr(y), _ptr(a1), _ptr(a2), int(round_))
    return y, a1, a2


def net_loss_grad(dims, w1, w2, w3, r, e, round_=True, odd=False, kind=0):
    """Loss and weight gradients; odd: y = (N(r) - N(-r)) / 2; kind 1: energy norm of the stencil."""
    nz, ny, nx = dims
    r = np.ascontiguousarray(r, np.float32)
    e = np.ascontiguousarray(e, np.float32)
    ws = [np.ascontiguousarray(w, np.float32) for w in (w1, w2, w3)]
    d = [np.empty(27 * 256, np.float32) for _ in range(3)]
    loss = colored_lib().oc_net_loss_grad2(nz, ny, nx, *[_ptr(w) for w in ws], _ptr(r), _ptr(e),
                                           *[_ptr(x) for x in d], int(round_), int(odd), int(kind))
    return loss, d


def stencil_apply(dims, v):
    nz, ny, nx = dims
    v = np.ascontiguousarray(v, np.float32)
    out = np.empty_like(v)
    colored_lib().oc_stencil_apply(nz, ny, nx, _ptr(v), _ptr(out))
    return out
