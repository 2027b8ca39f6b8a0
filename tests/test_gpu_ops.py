"""Operator parity on the device vs the CPU restatement of the reference's
optimized kernels.  Row-wise operators keep the reference's fma order, so
they must agree BIT FOR BIT; only reductions get a tolerance."""
import numpy as np
import pytest
import torch

from gpu_util import host, problems, sync, to_dev

pytestmark = pytest.mark.gpu

GRIDS = [(16, 16, 16), (32, 32, 32), (16, 24, 32)]


def rand(n, seed):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


@pytest.mark.parametrize("dims", GRIDS)
def test_spmv_bitwise(dims):
    P, O = problems(*dims)
    for l in range(4):
        L = O.levels[l]
        x = rand(L.m, 10 + l)
        xd, yd = to_dev(x), torch.empty(L.m, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        P.spmv(l, xd.data_ptr(), yd.data_ptr())
        sync(P)
        assert np.array_equal(host(yd), L.spmv(x))


@pytest.mark.parametrize("dims", GRIDS)
def test_symgs_bitwise(dims):
    P, O = problems(*dims)
    for l in range(4):
        L = O.levels[l]
        r, x0 = rand(L.m, 20 + l), rand(L.m, 30 + l)
        rd, xd = to_dev(r), to_dev(x0)
        torch.cuda.synchronize()
        P.symgs(l, rd.data_ptr(), xd.data_ptr())
        sync(P)
        assert np.array_equal(host(xd), L.symgs(r, x0))


@pytest.mark.parametrize("dims", GRIDS)
def test_symgs_zero_guess_bitwise(dims):
    P, O = problems(*dims)
    for l in range(4):
        L = O.levels[l]
        r = rand(L.m, 40 + l)
        rd = to_dev(r)
        xd = torch.full((L.m,), 123.0, dtype=torch.float64, device="cuda")  # must be ignored
        torch.cuda.synchronize()
        P.symgs_zero(l, rd.data_ptr(), xd.data_ptr())
        sync(P)
        assert np.array_equal(host(xd), L.symgs_zero(r))


@pytest.mark.parametrize("dims", GRIDS)
def test_restriction_prolongation_bitwise(dims):
    P, O = problems(*dims)
    for l in range(3):
        L, C = O.levels[l], O.levels[l + 1]
        rf, xf, xc = rand(L.m, 50 + l), rand(L.m, 60 + l), rand(C.m, 70 + l)
        rfd, xfd, rcd, xcd = to_dev(rf), to_dev(xf), torch.zeros(C.m, dtype=torch.float64, device="cuda"), to_dev(xc)
        torch.cuda.synchronize()
        P.restrict(l, rfd.data_ptr(), xfd.data_ptr(), rcd.data_ptr())
        P.prolong(l, xcd.data_ptr(), xfd.data_ptr())
        sync(P)
        assert np.array_equal(host(rcd), O.restrict_fused(l, rf, xf))
        assert np.array_equal(host(xfd), O.prolong(l, xc, xf))


@pytest.mark.parametrize("dims", GRIDS)
def test_restriction_reference_form(dims):
    """ComputeRestriction in its HPCG_REFERENCE form
    (src/ComputeRestriction.cpp:59-79,182-197): Axf = A xf by the SpMV, then
    rc = rf - Axf at the injected points, through hpcgb200_restrict.  Bit for
    bit against the restatement (rf - A xf of the ELL product at inj_f), and to
    rounding against the reference's own ComputeSPMV_ref +
    ComputeRestriction_ref in natural order (another summation order)."""
    import ctypes

    import rochpcg_b200 as R
    from oracle.oracle import RefProblem

    P, O = problems(*dims)
    lib = R.load()
    ref = RefProblem(*dims)
    for l in range(3):
        F, C = O.levels[l], O.levels[l + 1]
        rf, xf = rand(F.m, 90 + l), rand(F.m, 95 + l)
        rfd, xfd = to_dev(rf), to_dev(xf)
        axf = torch.empty_like(xfd)
        rcd = torch.full((C.m,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        P.spmv(l, xfd.data_ptr(), axf.data_ptr())
        vp = ctypes.c_void_p
        assert lib.hpcgb200_restrict(C.m, vp(P.device_ptr("inj_f", l)), vp(P.device_ptr("inj_c", l)),
                                     vp(rfd.data_ptr()), vp(axf.data_ptr()), vp(rcd.data_ptr()),
                                     vp(P.stream_handle)) == 0
        sync(P)
        inj_f = F.perm[F.f2c]
        want = np.empty(C.m)
        want[C.perm] = rf[inj_f] - F.spmv(xf)[inj_f]
        got = host(rcd)
        assert np.array_equal(got, want)
        nat = ref.restriction(l, F.unpermute(rf), F.unpermute(xf))
        assert np.allclose(C.unpermute(got), nat, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("dims", GRIDS)
def test_mg_vcycle_bitwise(dims):
    """The whole 4-level V-cycle has no reduction: bit-exact."""
    P, O = problems(*dims)
    r = rand(O.levels[0].m, 80)
    rd, zd = to_dev(r), torch.empty(O.levels[0].m, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    P.mg(rd.data_ptr(), zd.data_ptr())
    sync(P)
    assert np.array_equal(host(zd), O.mg(r))


def test_spmv_matches_reference_natural_order():
    """Against the reference's own ComputeSPMV_ref golden output (natural
    order, different summation order): equal to rounding."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_16x16x16.npz"))
    P, O = problems(16, 16, 16)
    L = O.levels[0]
    x = g["spmv_x"]
    xd, yd = to_dev(L.permute(x)), torch.empty(L.m, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    P.spmv(0, xd.data_ptr(), yd.data_ptr())
    sync(P)
    y = L.unpermute(host(yd))
    assert np.allclose(y, g["spmv_y"], rtol=1e-13, atol=1e-13)


def test_spmv_axpy_identities_256():
    """Full-size (256^3) size-independent properties of the FP64 operators:
    A 1 = b (the generator's b), SpMV linearity A(x + 2y) = Ax + 2Ay to
    rounding, and symmetry x'Ay = y'Ax to rounding."""
    import rochpcg_b200 as R

    P = R.Problem(256)
    m = P.rows[0]
    ones = torch.ones(m, dtype=torch.float64, device="cuda")
    y = torch.empty_like(ones)
    torch.cuda.synchronize()
    P.spmv(0, ones.data_ptr(), y.data_ptr())
    sync(P)
    b = torch.from_numpy(P.field("b")).cuda()
    assert torch.equal(y, b)
    g = torch.Generator(device="cuda").manual_seed(1)
    x1 = torch.rand(m, dtype=torch.float64, device="cuda", generator=g)
    x2 = torch.rand(m, dtype=torch.float64, device="cuda", generator=g)
    a1, a2, a3 = torch.empty_like(x1), torch.empty_like(x1), torch.empty_like(x1)
    s = x1 + 2 * x2
    torch.cuda.synchronize()
    P.spmv(0, x1.data_ptr(), a1.data_ptr())
    P.spmv(0, x2.data_ptr(), a2.data_ptr())
    P.spmv(0, s.data_ptr(), a3.data_ptr())
    sync(P)
    assert torch.allclose(a3, a1 + 2 * a2, rtol=1e-12, atol=1e-11)
    xay, yax = float(x1 @ a2), float(x2 @ a1)
    assert abs(xay - yax) / abs(xay) < 1e-12
    P.close()
