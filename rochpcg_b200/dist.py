"""Domain decomposition of the HPCG problem over ranks (one GPU each).

Python mirror of the reference's multi-rank path: the process grid
(``src/ComputeOptimalShapeXYZ.cpp``, ``src/GenerateGeometry.cpp``), the halo
plan (``src/SetupHalo.cpp``), the halo exchange (``src/ExchangeHalo.cpp``) and
the operators with their halo halves, over ``libhpcgb200.so``:

* :func:`shape` and :class:`HaloPlan` are host computations (no GPU needed);
* :class:`DistProblem` is one rank's sub-brick on the current device;
* :func:`group_cg` and the ``group_*`` operators drive every rank of a
  decomposition from one process on one device (the exchange is a device copy
  per neighbour) -- or one rank alone once :func:`attach_nccl` gave it a
  communicator, one process per GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, load

_INT_FIELDS = ("nbr_rank", "nbr_slot", "recv_len", "recv_off", "send_len", "send_off", "send_rows", "halo_rows",
               "halo_ptr", "halo_cols", "perm", "send_perm", "halo_prow", "halo_col", "halo_pc", "ell_col")
_INFO_KEYS = ("m", "next", "neighbours", "send_entries", "halo_rows", "halo_width", "halo_entries", "npx", "npy",
              "npz", "ipx", "ipy", "ipz", "nx", "ny", "nz")
NCCL_ID_BYTES = 128


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def shape(size: int) -> tuple[int, int, int]:
    """Process grid (npx, npy, npz) for `size` ranks (src/ComputeOptimalShapeXYZ.cpp:94-157)."""
    L = load()
    x, y, z = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(L, L.hpcgb200_dist_shape(size, ctypes.byref(x), ctypes.byref(y), ctypes.byref(z)))
    return x.value, y.value, z.value


def _field_len(info: dict, name: str) -> int:
    n = {"nbr_rank": info["neighbours"], "nbr_slot": info["neighbours"], "recv_len": info["neighbours"],
         "recv_off": info["neighbours"], "send_len": info["neighbours"], "send_off": info["neighbours"],
         "recv_gid": info["next"], "send_rows": info["send_entries"], "halo_rows": info["halo_rows"],
         "halo_ptr": info["halo_rows"] + 1, "halo_cols": info["halo_entries"]}
    return n[name]


class HaloPlan:
    """Host-side halo plan of one rank (src/SetupHalo.cpp:135-651)."""

    def __init__(self, nx: int, ny: int, nz: int, size: int, rank: int, grid: tuple | None = None):
        self.L = load()
        npx, npy, npz = grid if grid else (0, 0, 0)
        h = ctypes.c_void_p()
        check(self.L, self.L.hpcgb200_halo_plan_create(nx, ny, nz, size, rank, npx, npy, npz, ctypes.byref(h)))
        self.h = h
        v = np.zeros(16, np.int32)
        check(self.L, self.L.hpcgb200_halo_plan_info(self.h, _p(v)))
        self.info = dict(zip(_INFO_KEYS, (int(a) for a in v)))

    def field(self, name: str) -> np.ndarray:
        dt = np.int64 if name == "recv_gid" else np.int32
        out = np.empty(_field_len(self.info, name), dt)
        check(self.L, self.L.hpcgb200_halo_plan_copy(self.h, name.encode(), _p(out), out.nbytes))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.L.hpcgb200_halo_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DistProblem:
    """One rank's sub-brick (nx, ny, nz) of a problem split over `size` ranks,
    generated and optimized on the current device with its halo plan on every
    level (src/main.cpp:183-210, src/OptimizeProblem.cpp)."""

    def __init__(self, nx: int, ny: int, nz: int, size: int, rank: int, nlevels: int = 4,
                 grid: tuple | None = None):
        self.L = load()
        npx, npy, npz = grid if grid else (0, 0, 0)
        h = ctypes.c_void_p()
        check(self.L, self.L.hpcgb200_dist_create(nx, ny, nz, nlevels, size, rank, npx, npy, npz, ctypes.byref(h)))
        self.h = h
        self.size, self.rank = size, rank
        self.levels = []
        for l in range(nlevels):
            v = np.zeros(20, np.int32)
            nnz = ctypes.c_longlong()
            check(self.L, self.L.hpcgb200_dist_info(self.h, l, _p(v), ctypes.byref(nnz)))
            d = dict(zip(_INFO_KEYS, (int(a) for a in v[:16])))
            d["nblocks"] = int(v[19])
            d["nnz"] = int(nnz.value)
            d["ncols"] = d["m"] + d["next"]
            self.levels.append(d)
        self.nlevels = nlevels
        self.grid = (self.levels[0]["npx"], self.levels[0]["npy"], self.levels[0]["npz"])

    def field(self, name: str, level: int = 0) -> np.ndarray:
        info = self.levels[level]
        m = info["m"]
        if name in ("ell_col", "ell_val"):
            n = 27 * m
        elif name in ("perm", "b"):
            n = m
        elif name == "x":
            n = info["ncols"]
        elif name == "send_perm":
            n = info["send_entries"]
        elif name in ("halo_prow", "halo_pc"):
            n = info["halo_rows"]
        elif name == "halo_col":
            n = info["halo_rows"] * info["halo_width"]
        else:
            n = _field_len(info, name)
        dt = np.int64 if name == "recv_gid" else (np.int32 if name in _INT_FIELDS else np.float64)
        out = np.empty(n, dt)
        check(self.L, self.L.hpcgb200_dist_copy_field(self.h, level, name.encode(), _p(out), out.nbytes))
        if name in ("ell_col", "ell_val"):
            out = out.reshape(27, m)
        elif name == "halo_col":
            out = out.reshape(info["halo_width"], info["halo_rows"])
        return out

    def set_rhs(self, b_natural: np.ndarray | None):
        if b_natural is None:
            check(self.L, self.L.hpcgb200_dist_set_rhs(self.h, None))
        else:
            b = np.ascontiguousarray(b_natural, np.float64)
            assert b.size == self.levels[0]["m"]
            check(self.L, self.L.hpcgb200_dist_set_rhs(self.h, _p(b)))

    def get_x(self) -> np.ndarray:
        out = np.empty(self.levels[0]["m"], np.float64)
        check(self.L, self.L.hpcgb200_dist_get_x(self.h, _p(out)))
        return out

    def attach_nccl(self, nccl_id: bytes):
        buf = ctypes.create_string_buffer(bytes(nccl_id), NCCL_ID_BYTES)
        check(self.L, self.L.hpcgb200_dist_attach_nccl(self.h, buf, NCCL_ID_BYTES))

    def cg(self, max_iter: int, tol: float, precond: bool = True) -> dict:
        """The solve of this rank alone: with a communicator, or size 1."""
        return group_cg([self], max_iter, tol, precond)

    def close(self):
        if getattr(self, "h", None):
            self.L.hpcgb200_dist_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nccl_available() -> bool:
    return bool(load().hpcgb200_dist_nccl_available())


def nccl_id() -> bytes:
    L = load()
    buf = ctypes.create_string_buffer(NCCL_ID_BYTES)
    check(L, L.hpcgb200_dist_nccl_id(buf, NCCL_ID_BYTES))
    return buf.raw


def attach_nccl(problem: DistProblem, dist) -> None:
    """Give `problem` a communicator over the ranks of the default
    torch.distributed group `dist` (rank 0 makes the id, every rank joins)."""
    obj = [nccl_id() if dist.get_rank() == 0 else None]
    dist.broadcast_object_list(obj, src=0)
    problem.attach_nccl(obj[0])


def _handles(ranks):
    arr = (ctypes.c_void_p * len(ranks))(*[r.h.value for r in ranks])
    return arr, len(ranks)


def _ptrs(vs):
    return (ctypes.c_void_p * len(vs))(*[int(v) for v in vs])


def group_spmv(ranks, level: int, xs, ys) -> None:
    """y = A x on every rank (device pointers, permuted order, x with its external tail)."""
    h, n = _handles(ranks)
    L = ranks[0].L
    check(L, L.hpcgb200_dist_group_spmv(h, n, level, _ptrs(xs), _ptrs(ys)))


def group_symgs(ranks, level: int, rs, xs) -> None:
    h, n = _handles(ranks)
    L = ranks[0].L
    check(L, L.hpcgb200_dist_group_symgs(h, n, level, _ptrs(rs), _ptrs(xs)))


def group_restrict(ranks, level: int, rfs, xfs, rcs) -> None:
    h, n = _handles(ranks)
    L = ranks[0].L
    check(L, L.hpcgb200_dist_group_restrict(h, n, level, _ptrs(rfs), _ptrs(xfs), _ptrs(rcs)))


def group_mg(ranks, rs, xs) -> None:
    h, n = _handles(ranks)
    L = ranks[0].L
    check(L, L.hpcgb200_dist_group_mg(h, n, _ptrs(rs), _ptrs(xs)))


def group_cg(ranks, max_iter: int, tol: float, precond: bool = True) -> dict:
    """CG over the group from x = 0 (src/CG.cpp:104-200)."""
    h, n = _handles(ranks)
    L = ranks[0].L
    it = ctypes.c_int()
    nr, nr0, sec = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    hist = np.zeros(max_iter + 1, np.float64)
    check(L, L.hpcgb200_dist_group_cg(h, n, max_iter, tol, 1 if precond else 0, ctypes.byref(it), ctypes.byref(nr),
                                      ctypes.byref(nr0), _p(hist), ctypes.byref(sec)))
    return {"niters": it.value, "normr": nr.value, "normr0": nr0.value, "hist": hist[:it.value + 1],
            "seconds": sec.value}


def global_nnz(gnx: int, gny: int, gnz: int) -> int:
    """Nonzeros of the 27-point problem on a gnx x gny x gnz grid."""
    return (3 * gnx - 2) * (3 * gny - 2) * (3 * gnz - 2)
