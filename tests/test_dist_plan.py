"""Domain decomposition on the CPU: the process grid and the halo plan (host
code of libhpcgb200, no device needed), the multi-rank oracle pinned to the
reference's own generation, and the exchange protocol over real gloo
processes.

* process grid: the library's and the oracle's restatements of
  src/ComputeOptimalShapeXYZ.cpp equal the reference's compiled function;
* generation: every rank's rows, global columns and b in the multi-rank
  oracle equal src/GenerateProblem_ref.cpp's for that rank of the geometry;
* halo plan (src/SetupHalo.cpp): external columns, halo rows and their
  external entries equal the oracle's; every send list is the partner's
  receive list;
* the oracle's decomposed SpMV is the global operator, its CG starts from the
  global residual and ends within a few iterations of the global problem's
  (each brick is coloured on its own);
* gloo processes exchange halos with the library's send lists and receive
  exactly the values the receive lists name.
"""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

from rochpcg_b200 import dist as D  # noqa: E402

# (bricks whose halved level is not 4x3x2: the reference's colouring loop
# leaves rows of that brick uncoloured, see oracle/distributed.c)
CASES = [(2, (8, 8, 8)), (4, (8, 4, 6)), (8, (6, 8, 4)), (3, (4, 8, 8)), (12, (4, 4, 4)), (6, (8, 4, 6))]


def _ref_available():
    from oracle import oracle as O

    return os.path.exists(O.REF_SO)


def rank_coords(rank, grid):
    npx, npy, _ = grid
    return rank % npx, (rank % (npx * npy)) // npx, rank // (npx * npy)


def natural_gids(loc, rank, grid):
    """Global id of every natural local row of `rank`."""
    nx, ny, nz = loc
    ipx, ipy, ipz = rank_coords(rank, grid)
    gnx, gny = grid[0] * nx, grid[1] * ny
    nat = np.arange(nx * ny * nz)
    gx = ipx * nx + nat % nx
    gy = ipy * ny + (nat // nx) % ny
    gz = ipz * nz + nat // (nx * ny)
    return (gz * gny + gy) * gnx + gx


def row_global_columns(loc, rank, grid, perm, ext_gid, ell_col):
    """Global column ids of every natural row of a rank (sorted per row)."""
    m = loc[0] * loc[1] * loc[2]
    gid_of_nat = natural_gids(loc, rank, grid)
    inv = np.empty(m, np.int64)
    inv[perm] = np.arange(m)  # permuted row -> natural row
    out = []
    for row in range(m):
        cols = ell_col[:, perm[row]]
        cols = cols[cols >= 0]
        g = np.empty(len(cols), np.int64)
        loc_ = cols < m
        g[loc_] = gid_of_nat[inv[cols[loc_]]]
        g[~loc_] = ext_gid[cols[~loc_] - m]
        out.append(np.sort(g))
    return out


@pytest.mark.parametrize("size", list(range(1, 97)) + [128, 256, 360, 512, 1000, 1024, 4096])
def test_process_grid_matches_reference(size, oracle_libs):
    O = oracle_libs
    got = D.shape(size)
    assert got == O.od_shape(size)
    assert got[0] * got[1] * got[2] == size
    if _ref_available():
        assert got == O.ref_optimal_shape(size)


@pytest.mark.parametrize("size,loc", CASES)
def test_oracle_generation_matches_reference_rank_problem(size, loc, oracle_libs):
    if not _ref_available():
        pytest.skip("oracle/_ref not built (needs the reference source tree)")
    O = oracle_libs
    orc = O.DistOracle(size, *loc, nlevels=1)
    grid = D.shape(size)
    for rank in range(size):
        ref = O.ref_rank_problem(size, rank, *loc)
        assert ref["grid"][:3] == grid
        assert ref["grid"][3:] == rank_coords(rank, grid)
        col, _ = orc.ell(rank)
        perm = orc.perm(rank)
        got = row_global_columns(loc, rank, grid, perm, orc.ext_gid(rank), col)
        for row in range(len(got)):
            want = np.sort(ref["gcols"][row, :ref["nnz"][row]])
            assert np.array_equal(got[row], want), (rank, row)
        # b = row sum for x = 1, the reference's value per row
        assert np.array_equal(orc.b(rank)[perm], ref["b"])


@pytest.mark.parametrize("size,loc", CASES)
def test_library_halo_plan_matches_oracle(size, loc, oracle_libs):
    O = oracle_libs
    orc = O.DistOracle(size, *loc, nlevels=2)
    grid = D.shape(size)
    for level in range(2):
        l_loc = tuple(v >> level for v in loc)
        plans = {rank: D.HaloPlan(*l_loc, size, rank) for rank in range(size)}
        for rank, P in plans.items():
            oi = orc.info[rank][level]
            assert P.info["m"] == oi["m"] and P.info["next"] == oi["next"]
            assert np.array_equal(P.field("recv_gid"), orc.ext_gid(rank, level))
            # halo rows: the natural rows with external columns, ascending, and
            # their external columns as the oracle's ELL holds them
            col, _ = orc.ell(rank, level)
            perm = orc.perm(rank, level)
            m = oi["m"]
            ext_rows = [r for r in range(m) if (col[:, perm[r]] >= m).any()]
            assert list(P.field("halo_rows")) == ext_rows
            assert P.info["halo_rows"] == oi["nhalo"]
            ptr, hc = P.field("halo_ptr"), P.field("halo_cols")
            for h, r in enumerate(ext_rows):
                c = col[:, perm[r]]
                assert list(hc[ptr[h]:ptr[h + 1]]) == list(c[c >= m])
        # send list of a to b == receive list of b from a (as global ids)
        for rank, P in plans.items():
            gids = natural_gids(l_loc, rank, grid)
            nbr, soff, slen = P.field("nbr_rank"), P.field("send_off"), P.field("send_len")
            rows = P.field("send_rows")
            for j, q in enumerate(nbr):
                Q = plans[int(q)]
                k = list(Q.field("nbr_rank")).index(rank)
                got = rows[soff[j]:soff[j] + slen[j]]
                roff, rlen = Q.field("recv_off"), Q.field("recv_len")
                assert np.array_equal(gids[got], Q.field("recv_gid")[roff[k]:roff[k] + rlen[k]])
                assert np.all(np.diff(got) > 0)


def test_single_rank_plan_is_empty():
    P = D.HaloPlan(8, 8, 8, 1, 0)
    assert P.info["next"] == 0 and P.info["neighbours"] == 0 and P.info["halo_rows"] == 0


def test_plan_rejects_bad_geometry():
    from rochpcg_b200 import HpcgError

    with pytest.raises(HpcgError):
        D.HaloPlan(8, 8, 8, 4, 0, grid=(3, 1, 1))
    with pytest.raises(HpcgError):
        D.HaloPlan(8, 8, 8, 2, 2)


@pytest.mark.parametrize("size,loc,glob", [(2, (8, 8, 8), (16, 8, 8)), (4, (8, 8, 8), (16, 16, 8)),
                                           (8, (8, 8, 8), (16, 16, 16))])
def test_oracle_decomposed_operator_is_the_global_one(size, loc, glob, oracle_libs):
    O = oracle_libs
    orc = O.DistOracle(size, *loc, nlevels=4)
    G = O.ColoredProblem(*glob)
    grid = D.shape(size)
    assert (grid[0] * loc[0], grid[1] * loc[1], grid[2] * loc[2]) == glob
    rng = np.random.default_rng(3)
    xg = rng.uniform(-1, 1, glob[0] * glob[1] * glob[2])
    L0 = G.levels[0]
    yg = L0.unpermute(L0.spmv(L0.permute(xg)))
    xs, maps = [], []
    for rank in range(size):
        gid = natural_gids(loc, rank, grid)
        perm = orc.perm(rank)
        v = np.empty(len(gid))
        v[perm] = xg[gid]
        xs.append(v)
        maps.append((perm, gid))
    ys = orc.spmv(0, xs)
    for rank, (perm, gid) in enumerate(maps):
        np.testing.assert_allclose(ys[rank][perm], yg[gid], rtol=1e-13, atol=1e-13)
    # the same right-hand side and initial residual; the colouring of the
    # bricks (each coloured on its own) changes the count by a few iterations
    r, g = orc.cg(200, 1e-9), G.cg(200, 1e-9)
    assert r["normr0"] == g["normr0"]
    assert abs(r["niters"] - g["niters"]) <= 3


# ------------------------------------------------------------ gloo processes

def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_rank(rank, world, port, loc, q):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from rochpcg_b200 import dist as Dm

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        P = Dm.HaloPlan(*loc, world, rank)
        grid = Dm.shape(world)
        m = loc[0] * loc[1] * loc[2]
        # x holds each row's global id; the halo tail must receive the ids it names
        x = np.concatenate([natural_gids(loc, rank, grid).astype(np.float64), np.full(P.info["next"], -1.0)])
        rows = P.field("send_rows")
        buf = torch.from_numpy(x[rows].copy())
        nbr, soff, slen = P.field("nbr_rank"), P.field("send_off"), P.field("send_len")
        roff, rlen = P.field("recv_off"), P.field("recv_len")
        reqs, recv_bufs = [], []
        for j, peer in enumerate(nbr):
            rb = torch.empty(int(rlen[j]), dtype=torch.float64)
            recv_bufs.append(rb)
            reqs.append(dist.irecv(rb, int(peer)))
        for j, peer in enumerate(nbr):
            reqs.append(dist.isend(buf[soff[j]:soff[j] + slen[j]].clone(), int(peer)))
        for rq in reqs:
            rq.wait()
        for j in range(len(nbr)):
            x[m + roff[j]:m + roff[j] + rlen[j]] = recv_bufs[j].numpy()
        ok = bool(np.array_equal(x[m:], P.field("recv_gid").astype(np.float64)))
        dist.barrier()
        q.put((rank, ok, int(P.info["next"])))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,loc", [(2, (8, 6, 4)), (4, (6, 4, 8))])
def test_gloo_ranks_exchange_halos_with_the_library_plan(world, loc):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_exchange_rank, args=(r, world, port, loc, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert all(ok for _, ok, _ in res), res
    assert all(n > 0 for _, _, n in res)


@pytest.mark.parametrize("size", [1, 2, 3, 4, 6, 8, 12, 16, 27, 30])
def test_cpp_geometry_matches_reference(size, oracle_libs):
    """The C++ GenerateGeometry (process grid, coordinates, global offsets,
    the two-zone z split) against the reference's own, every rank."""
    import ctypes

    if not _ref_available():
        pytest.skip("oracle/_ref not built (needs the reference source tree)")
    from rochpcg_b200 import load

    L = load()
    # process grids of exactly `size` ranks (the given one, the computed one, a
    # row of ranks); a z split (pz > 0) needs more than pz process planes
    grids = [(0, 0, 0), D.shape(size), (size, 1, 1), (1, 1, size)]
    for grid in grids:
        npz = grid[2] if grid[0] else D.shape(size)[2]
        for pz, zl, zu in [(0, 0, 0)] + ([(1, 6, 10)] if npz > 1 else []):
            for rank in range(size):
                out = np.zeros(13, np.int64)
                assert L.hpcgb200_geometry(size, rank, pz, zl, zu, 8, 6, 4, *grid,
                                           out.ctypes.data_as(ctypes.c_void_p)) == 0
                want = oracle_libs.ref_geometry(size, rank, pz, zl, zu, 8, 6, 4, *grid)
                assert list(out) == want, (size, rank, pz, grid)
