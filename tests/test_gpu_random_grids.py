"""Parity on a fixed set of pseudo-random grids (dimensions multiples of 8
from 16, the reference's smallest local dimension, to 64; seed 2024): every
index array of the set-up, the FP64 V-cycle, the FP32 mixed V-cycle and the
FP64 stencil V-cycle bit for bit against the CPU restatement, and the FP64 CG residual history against the restatement's to
the dot products' rounding (rtol 1e-8, as the smoke test)."""
import numpy as np
import pytest
import torch

import rochpcg_b200 as R
from gpu_util import host, problems, sync, to_dev

pytestmark = pytest.mark.gpu

_rng = np.random.default_rng(2024)
GRIDS = [tuple(int(v) for v in 8 * _rng.integers(2, 9, 3)) for _ in range(6)]


@pytest.mark.parametrize("dims", GRIDS)
def test_random_grid_setup_and_vcycles(dims):
    P, O = problems(*dims)
    for l in range(4):
        L = O.levels[l]
        assert np.array_equal(P.field("perm", l), L.perm), l
        assert np.array_equal(P.field("ell_col", l), L.ell_col), l
        assert np.array_equal(P.field("diag_idx", l), L.diag_idx), l
    m = O.levels[0].m
    r = np.random.default_rng(sum(dims)).normal(size=m)
    rd = to_dev(r)
    # thin coarse levels (2 points across) may colour into other than one parity
    # class per colour: the FP32 V-cycle then refuses, the FP64 stencil V-cycle
    # takes the ELL kernels there
    all_stencil = all(P.stencil_ok(l) for l in range(4))
    modes = (R.MODE_FP64, R.MODE_FP64_STENCIL) + ((R.MODE_MIXED,) if all_stencil else ())
    z = {mode: torch.empty(m, dtype=torch.float64, device="cuda") for mode in modes}
    torch.cuda.synchronize()
    for mode, zd in z.items():
        P.mg(rd.data_ptr(), zd.data_ptr(), mode=mode)
    sync(P)
    assert np.array_equal(host(z[R.MODE_FP64]), O.mg(r))
    assert torch.equal(z[R.MODE_FP64_STENCIL], z[R.MODE_FP64])
    if all_stencil:
        assert np.array_equal(host(z[R.MODE_MIXED]), O.mg_f32(r.astype(np.float32)).astype(np.float64))
    else:
        zd = torch.empty(m, dtype=torch.float64, device="cuda")
        with pytest.raises(R.HpcgError) as ei:
            P.mg(rd.data_ptr(), zd.data_ptr(), mode=R.MODE_MIXED)
        assert ei.value.code == 5  # HPCGB200_ERR_NOT_STENCIL
        # the FP64 stencil solve still runs and keeps the FP64 history
        a = P.cg(20, 0.0, mode=R.MODE_FP64)
        b = P.cg(20, 0.0, mode=R.MODE_FP64_STENCIL)
        assert np.array_equal(a["hist"], b["hist"])


@pytest.mark.parametrize("dims", GRIDS[:3])
def test_random_grid_cg_history(dims):
    P, O = problems(*dims)
    got = P.cg(30, 0.0)
    ref = O.cg(30, 0.0)
    n = min(len(got["hist"]), len(ref["hist"]))
    h, hr = np.asarray(got["hist"][:n]), np.asarray(ref["hist"][:n])
    keep = hr > 1e-12 * hr[0]  # while above rounding
    assert np.allclose(h[keep], hr[keep], rtol=1e-8)
