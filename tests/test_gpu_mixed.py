"""Mixed precision: FP64 outer CG with the FP32 V-cycle on the implicit
stencil.  The V-cycle must equal the CPU FP32 restatement of the ELL kernels
bit for bit; the solve must reach 1e-9 verified by an FP64 true residual."""
import numpy as np
import pytest
import torch

from gpu_util import host, problems, sync, to_dev

pytestmark = pytest.mark.gpu

FLT_OVER_DBL = np.finfo(np.float32).eps / np.finfo(np.float64).eps


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 32, 32), (16, 24, 32), (64, 64, 64), (24, 40, 56), (56, 56, 40)])
def test_mixed_vcycle_bitwise(dims):
    import rochpcg_b200 as R

    P, O = problems(*dims)
    r = np.random.default_rng(3).normal(size=O.levels[0].m)
    rd, zd = to_dev(r), torch.empty(O.levels[0].m, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    P.mg(rd.data_ptr(), zd.data_ptr(), mode=R.MODE_MIXED)
    sync(P)
    z_oracle = O.mg_f32(r.astype(np.float32)).astype(np.float64)
    assert np.array_equal(host(zd), z_oracle)


@pytest.mark.parametrize("n", [32, 64])
def test_mixed_cg_converges_fp64_verified(n):
    import rochpcg_b200 as R
    from rochpcg_b200.rhs import normal_rhs

    P = R.Problem(n)
    fp = P.cg(1000, 1e-9)
    mx = P.cg(1000, 1e-9, mode=R.MODE_MIXED)
    assert mx["normr"] / mx["normr0"] <= 1e-9
    assert P.true_residual() <= 2e-9
    assert mx["niters"] <= fp["niters"] + 3
    P.set_rhs(normal_rhs(P.rows[0], 0))
    fp = P.cg(1000, 1e-9)
    mx = P.cg(1000, 1e-9, mode=R.MODE_MIXED)
    assert P.true_residual() <= 2e-9
    assert mx["niters"] <= fp["niters"] + 3
    P.close()


def test_mixed_test_symmetry_and_test_cg():
    import rochpcg_b200 as R

    P, _ = problems(32, 32, 32)
    s = P.test_symmetry(mode=R.MODE_MIXED)
    assert s["depsym_spmv"] <= 1.0
    # the FP32 V-cycle is symmetric to single-precision rounding: the
    # reference's DBL_EPSILON-scaled departure, rescaled to FLT_EPSILON
    assert s["depsym_mg"] / FLT_OVER_DBL <= 1.0
    t = P.test_cg(mode=R.MODE_MIXED)
    assert t["count_fail"] == 0, t


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 32, 32), (16, 24, 32), (24, 40, 56), (72, 40, 48)])
def test_stencil_spmv_equals_ell_spmv_bitwise(dims):
    """The mixed path's implicit FP64 operator is the ELL operator, bit for bit."""
    P, O = problems(*dims)
    for l in range(4):
        m = O.levels[l].m
        x = np.random.default_rng(40 + l).uniform(-1, 1, m)
        xd = to_dev(x)
        y1 = torch.empty(m, dtype=torch.float64, device="cuda")
        y2 = torch.empty_like(y1)
        torch.cuda.synchronize()
        P.spmv(l, xd.data_ptr(), y1.data_ptr())
        P.spmv_stencil(l, xd.data_ptr(), y2.data_ptr())
        sync(P)
        assert torch.equal(y1, y2)
        assert np.array_equal(host(y2), O.levels[l].spmv(x))


@pytest.mark.parametrize("dims", [(16, 16, 16), (16, 24, 32), (24, 40, 56), (72, 40, 48), (56, 56, 40),
                                  (136, 12, 66)])
def test_mixed_outer_spmv_equals_ell_to_rounding(dims):
    """The mixed path's outer operator sums the 27 terms as a separable box
    (x, y, then z sums) instead of the ELL slot order: per row it must equal
    the ELL product to FP64 rounding, |y - y_ell| <= 64 eps (a_ii |x_i| +
    sum_j |x_j|), on grids whose sizes are not multiples of the kernel's
    64 x 4 x 32 blocks, on every level (coarse levels without the canonical
    colouring take the ELL-ordered stencil kernel)."""
    if dims == (136, 12, 66):
        import rochpcg_b200 as R

        P = R.Problem(*dims, nlevels=2)
        nl = 2
    else:
        P, _ = problems(*dims)
        nl = 4
    eps = np.finfo(np.float64).eps
    for l in range(nl):
        m = P.rows[l]
        x = np.random.default_rng(90 + l).uniform(-1, 1, m)
        xd = to_dev(x)
        y1 = torch.empty(m, dtype=torch.float64, device="cuda")
        y2 = torch.empty_like(y1)
        ya = torch.empty_like(y1)
        xa = xd.abs()
        torch.cuda.synchronize()
        P.spmv(l, xd.data_ptr(), y1.data_ptr())
        P.spmv_mixed(l, xd.data_ptr(), y2.data_ptr())
        P.spmv(l, xa.data_ptr(), ya.data_ptr())  # a_ii |x_i| - sum |x_j|
        sync(P)
        d = torch.from_numpy(P.field("diag", l)).cuda()
        bound = 64 * eps * (2 * d * xa - ya)  # a_ii |x_i| + sum_j |x_j|
        assert torch.all((y1 - y2).abs() <= bound), l
    if dims == (136, 12, 66):
        P.close()


@pytest.mark.parametrize("mode_name", ["MODE_MIXED", "MODE_FP64_STENCIL"])
def test_direct_launches_equal_graph(mode_name, monkeypatch):
    """The solve as one graph (kernels back to back, no programmatic launch)
    and as direct launches (the 4-row kernels with programmatic dependent
    launch, a host check per iteration) give the same residual history bit
    for bit; the graph form of the V-cycle times like the direct one."""
    import rochpcg_b200 as R

    mode = getattr(R, mode_name)
    P = R.Problem(48, 40, 56)
    g = P.cg(40, 0.0, mode=mode)
    monkeypatch.setenv("HPCGB200_GRAPH", "0")
    d = P.cg(40, 0.0, mode=mode)
    monkeypatch.delenv("HPCGB200_GRAPH")
    assert g["niters"] == d["niters"] == 40
    assert np.array_equal(g["hist"], d["hist"])
    op = "mg_mixed" if mode == R.MODE_MIXED else "mg_stencil"
    assert P.time_op("graph:" + op, 2) > 0 and P.time_op(op, 2) > 0
    with pytest.raises(R.HpcgError):
        P.time_op("graph:no_such_op", 1)
    P.close()
