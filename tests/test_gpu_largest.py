"""The largest configuration, 560 x 560 x 280 (87.8M rows; 27 x 87.8M ELL
slots exceed 2^31, so slot offsets are 64-bit; the coarsest level is
70 x 70 x 35, odd), through size-independent properties: level sizes and
nonzero counts of the 27-point stencil, the implicit-stencil SpMV equal to the
ELL SpMV bit for bit on every level, the FP64 stencil solve's residual history
equal to the FP64 ELL solve's, and the mixed solve's FP64 true residual; the
index arrays of its two coarsest levels (140 x 140 x 70 and the odd
70 x 70 x 35) and the transfer indices between them bit for bit against the
CPU restatement of the optimized set-up."""
import numpy as np
import pytest
import torch

import rochpcg_b200 as R
from rochpcg_b200.rhs import normal_rhs
from gpu_util import dev_field, sync, to_dev

pytestmark = pytest.mark.gpu


def _coarse_levels_bit_exact(P, dims):
    from oracle.oracle import ColoredLevel, _ptr, colored_lib

    def eq(dev, arr):
        return torch.equal(dev, torch.from_numpy(np.ascontiguousarray(arr).reshape(-1)).cuda())

    lv = {l: ColoredLevel(*dims[l]) for l in (2, 3)}
    for l, L in lv.items():
        assert eq(dev_field(P, "colors", l, np.int32), L.colors), l
        assert eq(dev_field(P, "perm", l, np.int32), L.perm), l
        assert np.array_equal(P.field("round_sizes", l), L.round_sizes), l
        sz = P.field("sizes", l)
        assert np.array_equal(sz[: len(L.sizes)], L.sizes), l  # by value: 70x70x35 has unequal classes
        assert eq(dev_field(P, "ell_col", l, np.int32), L.ell_col), l
        assert eq(dev_field(P, "diag_idx", l, np.int32), L.diag_idx), l
        assert eq(dev_field(P, "inv_diag", l, np.float64), L.inv_diag), l
    f2c = np.empty(lv[3].m, np.int32)
    colored_lib().oc_f2c(*dims[2], _ptr(f2c))
    assert eq(dev_field(P, "f2c", 2, np.int32), f2c)
    assert eq(dev_field(P, "inj_f", 2, np.int32), lv[2].perm[f2c])
    assert eq(dev_field(P, "inj_c", 2, np.int32), lv[3].perm)


def test_largest_config_properties():
    P = R.Problem(560, 560, 280)
    dims = [(560 >> l, 560 >> l, 280 >> l) for l in range(4)]
    assert P.dims == dims
    assert P.rows == [a * b * c for a, b, c in dims]
    assert P.nnz == [(3 * a - 2) * (3 * b - 2) * (3 * c - 2) for a, b, c in dims]
    assert 27 * P.rows[0] > 2 ** 31
    assert all(P.stencil_ok(l) for l in range(4))
    _coarse_levels_bit_exact(P, dims)
    for l in (0, 3):
        x = np.random.default_rng(l).uniform(-1, 1, P.rows[l])
        xd = to_dev(x)
        y1 = torch.empty_like(xd)
        y2 = torch.empty_like(xd)
        torch.cuda.synchronize()
        P.spmv(l, xd.data_ptr(), y1.data_ptr())
        P.spmv_stencil(l, xd.data_ptr(), y2.data_ptr())
        sync(P)
        assert torch.equal(y1, y2), l
        del xd, y1, y2
    P.set_rhs(normal_rhs(P.rows[0], 7))
    a = P.cg(12, 0.0, mode=R.MODE_FP64)
    b = P.cg(12, 0.0, mode=R.MODE_FP64_STENCIL)
    assert a["niters"] == b["niters"] == 12
    assert np.array_equal(a["hist"], b["hist"])
    m = P.cg(1000, 1e-9, mode=R.MODE_MIXED)
    assert m["normr"] / m["normr0"] <= 1e-9
    assert P.true_residual() <= 2e-9
    P.close()
