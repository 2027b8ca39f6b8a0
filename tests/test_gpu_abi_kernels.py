"""The plain-pointer C ABI kernel entry points, called with torch device
buffers on torch's stream, against numpy / the CPU restatement."""
import ctypes

import numpy as np
import pytest
import torch

import rochpcg_b200 as R
from gpu_util import problems

pytestmark = pytest.mark.gpu


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ws():
    n = R.load().hpcgb200_reduction_workspace_bytes()
    return torch.zeros(n, dtype=torch.uint8, device="cuda"), n


@pytest.mark.parametrize("n", [1, 255, 4096, 1 << 20, 3_000_001])
def test_dot_waxpby_residual(n):
    L = R.load()
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5
    y = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    w, nb = ws()
    assert L.hpcgb200_dot(n, vp(x), vp(y), vp(res), vp(w), nb, stream()) == 0
    torch.cuda.synchronize()
    ref = float(np.dot(x.cpu().numpy(), y.cpu().numpy()))
    assert abs(res.item() - ref) <= 1e-12 * max(1.0, float((x.abs() * y.abs()).sum()))
    # waxpby: alpha == 1, beta == 1 and general forms
    out = torch.empty_like(x)
    for a, b in ((1.0, -2.5), (3.0, 1.0), (0.25, -0.5)):
        assert L.hpcgb200_waxpby(n, a, vp(x), b, vp(y), vp(out), stream()) == 0
        torch.cuda.synchronize()
        assert torch.allclose(out, a * x + b * y, rtol=1e-15, atol=1e-15)
    # fused y += alpha x, ||y||^2
    yy = y.clone()
    assert L.hpcgb200_waxpby_dot(n, -0.75, vp(x), vp(yy), vp(res), vp(w), nb, stream()) == 0
    torch.cuda.synchronize()
    assert torch.allclose(yy, y - 0.75 * x, rtol=1e-15, atol=1e-15)
    assert abs(res.item() - float((yy * yy).sum())) <= 1e-10 * res.item() + 1e-300
    assert L.hpcgb200_residual_inf(n, vp(x), vp(y), vp(res), vp(w), nb, stream()) == 0
    torch.cuda.synchronize()
    assert res.item() == float((x - y).abs().max())


def test_dot_empty_and_workspace_errors():
    L = R.load()
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    res = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    w, nb = ws()
    assert L.hpcgb200_dot(0, vp(x), vp(x), vp(res), vp(w), nb, stream()) == 0
    torch.cuda.synchronize()
    assert res.item() == 0.0
    assert L.hpcgb200_dot(4, vp(x), vp(x), vp(res), vp(w), 16, stream()) == 4  # workspace too small


def test_raw_kernels_on_oracle_data():
    """spmv / symgs / symgs_zero / restrict / prolong entry points fed with
    the CPU restatement's level arrays."""
    L = R.load()
    _, O = problems(16, 16, 16)
    A, C = O.levels[0], O.levels[1]
    m = A.m
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    col, val, inv, dg, didx = d(A.ell_col), d(A.ell_val), d(A.inv_diag), d(A.ell_val[A.diag_idx, np.arange(m)]), d(A.diag_idx)
    sizes = (ctypes.c_int * 8)(*A.sizes[:8].tolist())
    offs = (ctypes.c_int * 9)(*A.offsets[:9].tolist())
    x = np.random.default_rng(0).uniform(-1, 1, m)
    xd, yd = d(x), torch.empty(m, dtype=torch.float64, device="cuda")
    assert L.hpcgb200_spmv(m, vp(col), vp(val), vp(xd), vp(yd), stream()) == 0
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), A.spmv(x))
    xs = xd.clone()
    assert L.hpcgb200_symgs(m, 8, 6, sizes, offs, vp(col), vp(val), vp(inv), vp(yd), vp(xs), stream()) == 0
    torch.cuda.synchronize()
    assert np.array_equal(xs.cpu().numpy(), A.symgs(A.spmv(x), x))
    assert L.hpcgb200_symgs_zero(m, 8, 6, sizes, offs, vp(col), vp(val), vp(didx), vp(dg), vp(inv), vp(yd), vp(xs),
                                 stream()) == 0
    torch.cuda.synchronize()
    assert np.array_equal(xs.cpu().numpy(), A.symgs_zero(A.spmv(x)))
    injf, injc = d(A.perm[A.f2c]), d(C.perm)
    rc = torch.empty(C.m, dtype=torch.float64, device="cuda")
    assert L.hpcgb200_restrict_fused(C.m, vp(injf), vp(injc), m, vp(col), vp(val), vp(yd), vp(xd), vp(rc),
                                     stream()) == 0
    torch.cuda.synchronize()
    assert np.array_equal(rc.cpu().numpy(), O.restrict_fused(0, A.spmv(x), x))
    # bad colour layout is rejected
    bad = (ctypes.c_int * 8)(*([1] * 8))
    assert L.hpcgb200_symgs(m, 8, 6, bad, offs, vp(col), vp(val), vp(inv), vp(yd), vp(xs), stream()) == 1
