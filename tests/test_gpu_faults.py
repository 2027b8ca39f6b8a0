"""Failures injected from the host, on a healthy GPU (no device fault, trap or
hang is ever provoked).  A NaN planted in the right-hand side, in the FP32
V-cycle's operator data or in the learned smoother's weights must end or
redirect the solve within its iteration bound, be reported through the C ABI
status, and leave the problem and the context usable: the next solve on the
repaired data reproduces the healthy one bit for bit."""
import numpy as np
import pytest
import torch

import rochpcg_b200 as R
from gpu_util import dev_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode_name", ["MODE_FP64", "MODE_FP64_STENCIL", "MODE_MIXED"])
def test_nan_in_rhs_ends_solve_with_status(mode_name):
    mode = getattr(R, mode_name)
    P = R.Problem(32)
    healthy = P.cg(500, 1e-9, mode=mode)
    b = np.full(P.rows[0], 1.0)
    b[1234] = np.nan
    P.set_rhs(b)
    with pytest.raises(R.HpcgError) as ei:
        P.cg(500, 1e-9, mode=mode)
    assert ei.value.code == R.ERR_NONFINITE
    res = ei.value.result
    assert res["niters"] == 0 and np.isnan(res["normr0"])  # the preamble already sees it
    P.set_rhs(None)  # the generated b again
    again = P.cg(500, 1e-9, mode=mode)
    assert again["niters"] == healthy["niters"]
    assert np.array_equal(again["hist"], healthy["hist"])
    P.close()


def test_nan_in_fp32_vcycle_data_ends_solve_with_status():
    """A NaN in the level-1 1/a_ii of the FP32 V-cycle: the first
    preconditioner application poisons z, the loop control ends the WHILE node
    after that iteration, and the status says so."""
    P = R.Problem(32)
    healthy = P.cg(500, 1e-9, mode=R.MODE_MIXED)
    inv = dev_field(P, "inv_diag32", 1, np.float32)
    saved = inv.clone()
    inv[77] = float("nan")
    torch.cuda.synchronize()
    with pytest.raises(R.HpcgError) as ei:
        P.cg(500, 1e-9, mode=R.MODE_MIXED)
    assert ei.value.code == R.ERR_NONFINITE
    assert ei.value.result["niters"] == 1
    assert np.isfinite(ei.value.result["normr0"])
    inv.copy_(saved)
    torch.cuda.synchronize()
    again = P.cg(500, 1e-9, mode=R.MODE_MIXED)
    assert np.array_equal(again["hist"], healthy["hist"])
    P.close()


def test_nan_in_learned_weights_falls_back_and_restarts():
    """A NaN in the network's weights makes the learned V-cycle's first output
    non-finite: the learned solve counts that as a smoother failure, restarts
    from x = 0 with the plain FP32 V-cycle and still reaches 1e-9 (FP64 true
    residual); the abandoned iteration is counted and reported."""
    from rochpcg_b200 import learned as LS

    P = R.Problem(64)
    mixed = P.cg(1000, 1e-9, mode=R.MODE_MIXED)
    S = LS.Smoother.load()
    w = S.get_weights()
    # one layer-3 weight (tap 13, input channel 3, output channel 0): no ReLU
    # follows layer 3, so the NaN reaches the output (a ReLU, max(z, 0), would
    # turn a NaN pre-activation into 0)
    w[2 * 27 * 256 + 13 * 256 + 3 * 16 + 0] = np.nan
    S.set_weights(w)
    P.set_smoother(S, 2)
    r = P.cg(1000, 1e-9, mode=R.MODE_LEARNED)
    assert P.last_fallback() == 1
    assert r["niters"] == 1 + mixed["niters"]
    assert not np.isfinite(r["hist"][1])
    assert np.array_equal(r["hist"][2:], mixed["hist"][1:])  # the restarted solve is the mixed one
    assert r["normr"] / r["normr0"] <= 1e-9
    assert P.true_residual() <= 2e-9
    P.set_smoother(None)
    P.close()


def test_grid_barrier_wait_runs_out_and_reports():
    """The persistent CG step's grid barrier waits at most about a second: when
    one block never arrives (a flag that nothing sets), the others give up,
    the status word says so, and the context stays usable (a full barrier then
    passes).  No GPU fault, trap or hang is involved."""
    import ctypes
    import time

    L = R.load()
    st, passed, blocks = ctypes.c_int(-1), ctypes.c_int(-1), ctypes.c_int(0)
    t0 = time.perf_counter()
    assert L.hpcgb200_selftest_grid_barrier(0, ctypes.byref(st), ctypes.byref(passed), ctypes.byref(blocks)) == 0
    elapsed = time.perf_counter() - t0
    assert blocks.value > 1
    assert st.value == 1 and passed.value == 0
    assert elapsed < 10.0
    assert L.hpcgb200_selftest_grid_barrier(-1, ctypes.byref(st), ctypes.byref(passed), ctypes.byref(blocks)) == 0
    assert st.value == 0 and passed.value == blocks.value
    P = R.Problem(16)  # the context is fine
    assert P.cg(50, 1e-9)["normr"] / P.cg(50, 1e-9)["normr0"] <= 1e-9
    P.close()
