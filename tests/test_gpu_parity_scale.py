"""Parity at the benchmarked sizes.

* Every index array the device set-up builds -- colours, permutation, colour
  sizes, JPL round sizes, ELL columns, ELL values, diagonal index, 1/a_ii and
  the multigrid transfer indices -- equals the CPU restatement of the
  reference's optimized set-up (oracle/colored.c: src/MultiColoring.cpp:
  151-353, src/Permute.cpp:95-218, src/SparseMatrix.cpp:166-407) BIT FOR BIT
  on all four levels of the 256^3 and 320^3 problems the bench solves.  The
  comparison runs on the GPU against device views of the library's arrays.
* At 128^3: the FP64 V-cycle, the FP64 implicit-stencil V-cycle and the FP32
  (mixed) V-cycle equal the restatement bit for bit, and the FP64 CG's
  residual history and its iteration count to 1e-9 match the restatement's
  optimized CG (src/CG.cpp:104-200) within the dot-product summation order.
"""
import numpy as np
import pytest
import torch

from gpu_util import dev_field, host, problems, sync, to_dev

pytestmark = pytest.mark.gpu


def _oracle_f2c(fx, fy, fz):
    from oracle.oracle import _ptr, colored_lib

    out = np.empty((fx // 2) * (fy // 2) * (fz // 2), np.int32)
    colored_lib().oc_f2c(fx, fy, fz, _ptr(out))
    return out


def _eq(dev, arr):
    return torch.equal(dev, torch.from_numpy(np.ascontiguousarray(arr).reshape(-1)).cuda())


@pytest.mark.parametrize("n", [256, 320])
def test_index_arrays_bit_exact_at_benchmark_size(n):
    import rochpcg_b200 as R
    from oracle.oracle import ColoredLevel

    P = R.Problem(n)  # the product configuration (generated arrays freed)
    prev = None  # (perm, f2c) of the finer level
    for l in range(4):
        d = (n >> l, n >> l, n >> l)
        L = ColoredLevel(*d)
        m = L.m
        assert P.rows[l] == m
        del L.cols, L.vals  # natural-order generated arrays: not needed below
        assert _eq(dev_field(P, "colors", l, np.int32), L.colors), ("colors", l)
        assert _eq(dev_field(P, "perm", l, np.int32), L.perm), ("perm", l)
        assert np.array_equal(P.field("round_sizes", l), L.round_sizes), l
        assert np.array_equal(P.field("sizes", l)[: len(L.sizes)], L.sizes), l
        assert P.nblocks[l] == L.nblocks == 8
        assert _eq(dev_field(P, "ell_col", l, np.int32), L.ell_col), ("ell_col", l)
        ev = dev_field(P, "ell_val", l, np.float64)
        valid = torch.from_numpy(L.ell_col.reshape(-1) >= 0).cuda()
        assert torch.equal(ev[valid], torch.from_numpy(L.ell_val.reshape(-1)).cuda()[valid]), ("ell_val", l)
        del ev, valid
        assert _eq(dev_field(P, "diag_idx", l, np.int32), L.diag_idx), ("diag_idx", l)
        assert _eq(dev_field(P, "inv_diag", l, np.float64), L.inv_diag), ("inv_diag", l)
        if prev is not None:
            pperm, pf2c = prev
            assert _eq(dev_field(P, "f2c", l - 1, np.int32), pf2c), ("f2c", l - 1)
            assert _eq(dev_field(P, "inj_f", l - 1, np.int32), pperm[pf2c]), ("inj_f", l - 1)
            assert _eq(dev_field(P, "inj_c", l - 1, np.int32), L.perm), ("inj_c", l - 1)
        prev = (L.perm, _oracle_f2c(*d) if l < 3 else None)
        del L
        torch.cuda.empty_cache()
    P.close()


def test_fp64_vcycles_bitwise_128():
    import rochpcg_b200 as R

    P, O = problems(128, 128, 128)
    r = np.random.default_rng(81).uniform(-1, 1, O.levels[0].m)
    want = O.mg(r)
    for mode in (R.MODE_FP64, R.MODE_FP64_STENCIL):
        rd, zd = to_dev(r), torch.empty(O.levels[0].m, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        P.mg(rd.data_ptr(), zd.data_ptr(), mode=mode)
        sync(P)
        assert np.array_equal(host(zd), want), mode


def test_mixed_vcycle_bitwise_128():
    import rochpcg_b200 as R

    P, O = problems(128, 128, 128)
    r = np.random.default_rng(82).normal(size=O.levels[0].m)
    rd, zd = to_dev(r), torch.empty(O.levels[0].m, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    P.mg(rd.data_ptr(), zd.data_ptr(), mode=R.MODE_MIXED)
    sync(P)
    assert np.array_equal(host(zd), O.mg_f32(r.astype(np.float32)).astype(np.float64))


def test_cg_iterations_match_oracle_128():
    """FP64 MG-PCG at 128^3 to 1e-9 from the generated b: the same iteration
    count as the restatement (+-1 allowed for the summation order of the dot
    products), histories equal to 1e-6 while above roundoff."""
    P, O = problems(128, 128, 128)
    r = P.cg(1000, 1e-9)
    o = O.cg(1000, 1e-9)
    assert r["normr0"] == o["normr0"]
    assert abs(r["niters"] - o["niters"]) <= 1, (r["niters"], o["niters"])
    k = min(len(r["hist"]), len(o["hist"]))
    rel_r, rel_o = r["hist"][:k] / r["normr0"], o["hist"][:k] / o["normr0"]
    live = rel_o > 1e-11
    assert np.allclose(rel_r[live], rel_o[live], rtol=1e-6, atol=0)
    assert r["normr"] / r["normr0"] <= 1e-9
