"""Device problem generation and optimization vs the CPU restatement:
every index array bit-exact, values exact."""
import numpy as np
import pytest

from gpu_util import problems

pytestmark = pytest.mark.gpu

GRIDS = [(16, 16, 16), (32, 32, 32), (16, 24, 32)]


@pytest.mark.parametrize("dims", GRIDS)
def test_generated_problem(dims):
    P, O = problems(*dims)
    for l in range(4):
        L = O.levels[l]
        assert np.array_equal(P.field("mtx_ind", l), L.cols)
        assert np.array_equal(P.field("values", l), L.vals)
        assert np.array_equal(P.field("nnz_in_row", l), L.nnz_in_row)
        assert np.array_equal(P.field("diag_slot", l), L.diag_slot)
        assert np.array_equal(P.field("hash", l), L.hash)
        assert np.array_equal(P.field("l2g", l), np.arange(L.m, dtype=np.int64))
    assert np.array_equal(P.field("b"), O.b)  # permuted generated b
    assert np.all(P.field("xexact") == 1.0)
    m = O.levels[0].m
    assert P.nnz[0] == int((O.levels[0].nnz_in_row.astype(np.int64)).sum())


@pytest.mark.parametrize("dims", GRIDS)
def test_coloring_and_permutation(dims):
    P, O = problems(*dims)
    for l in range(4):
        L = O.levels[l]
        assert np.array_equal(P.field("colors", l), L.colors)
        assert np.array_equal(P.field("perm", l), L.perm)
        assert np.array_equal(P.field("round_sizes", l), L.round_sizes)
        sz = P.field("sizes", l)
        assert np.array_equal(sz[: len(L.sizes)], L.sizes)
        assert P.nblocks[l] == 8


@pytest.mark.parametrize("dims", GRIDS)
def test_ell_and_diagonal(dims):
    P, O = problems(*dims)
    for l in range(4):
        L = O.levels[l]
        ec = P.field("ell_col", l)
        assert np.array_equal(ec, L.ell_col)
        ev = P.field("ell_val", l)
        valid = L.ell_col >= 0
        assert np.array_equal(ev[valid], L.ell_val[valid])
        assert np.array_equal(P.field("diag_idx", l), L.diag_idx)
        assert np.array_equal(P.field("inv_diag", l), L.inv_diag)
        if l < 3:
            assert np.array_equal(P.field("f2c", l), L.f2c)
            C = O.levels[l + 1]
            assert np.array_equal(P.field("inj_f", l), L.perm[L.f2c])
            assert np.array_equal(P.field("inj_c", l), C.perm)


def test_odd_coarse_level_two_levels():
    """6x10x14 with 2 levels: the coarse grid 3x5x7 has unequal parity
    classes; colors/perm still match the restatement bit for bit and the
    by-value colour blocks tile the permutation."""
    import rochpcg_b200 as R
    from oracle.oracle import ColoredLevel

    P = R.Problem(6, 10, 14, nlevels=2, keep_generated=True)
    L = ColoredLevel(3, 5, 7)
    assert np.array_equal(P.field("colors", 1), L.colors)
    assert np.array_equal(P.field("perm", 1), L.perm)
    assert np.array_equal(P.field("ell_col", 1), L.ell_col)
    sz = P.field("sizes", 1)
    assert sz.sum() == L.m
    P.close()


def test_stencil_verified():
    P, _ = problems(16, 16, 16)
    assert all(P.stencil_ok(l) for l in range(4))
