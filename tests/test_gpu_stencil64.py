"""FP64 V-cycle and CG on the implicit stencil (HPCGB200_MODE_FP64_STENCIL):
the V-cycle must equal the FP64 ELL V-cycle bit for bit on every level shape
(4-aligned colour bricks use the stencil kernels, the others the ELL
kernels), and whole solves must reproduce the FP64 residual history bit for
bit (the p.Ap reduction follows the ELL kernel's partition)."""
import numpy as np
import pytest
import torch

import rochpcg_b200 as R
from rochpcg_b200 import benchmark as B
from rochpcg_b200.rhs import normal_rhs
from gpu_util import host, sync, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 32, 32), (16, 24, 32), (64, 64, 64), (24, 40, 56),
                                  (56, 56, 40), (128, 128, 128)])
def test_stencil_vcycle_equals_ell_vcycle(dims):
    P = R.Problem(*dims)
    r = np.random.default_rng(11).normal(size=P.rows[0])
    rd = to_dev(r)
    z1 = torch.empty_like(rd)
    z2 = torch.full_like(rd, 7.0)
    torch.cuda.synchronize()
    P.mg(rd.data_ptr(), z1.data_ptr(), mode=R.MODE_FP64)
    P.mg(rd.data_ptr(), z2.data_ptr(), mode=R.MODE_FP64_STENCIL)
    sync(P)
    assert torch.equal(z1, z2)
    assert np.isfinite(host(z2)).all()
    P.close()


@pytest.mark.parametrize("dims,rhs", [((32, 32, 32), None), ((64, 64, 64), 0), ((24, 40, 56), 3),
                                      ((128, 128, 128), 9999)])
def test_stencil_cg_history_equals_fp64(dims, rhs):
    P = R.Problem(*dims)
    if rhs is not None:
        P.set_rhs(normal_rhs(P.rows[0], rhs))
    a = P.cg(500, 1e-9, mode=R.MODE_FP64)
    b = P.cg(500, 1e-9, mode=R.MODE_FP64_STENCIL)
    assert a["niters"] == b["niters"]
    assert np.array_equal(a["hist"], b["hist"])
    assert b["normr"] / b["normr0"] <= 1e-9 and P.true_residual() <= 2e-9
    # a second solve reuses the cached graph and gives the same bits
    c = P.cg(500, 1e-9, mode=R.MODE_FP64_STENCIL)
    assert np.array_equal(b["hist"], c["hist"])
    P.close()


def test_stencil_mode_validation_tests():
    P = R.Problem(32, 32, 32)
    t = P.test_cg(mode=R.MODE_FP64_STENCIL)
    assert t["count_fail"] == 0, t
    assert t == P.test_cg(mode=R.MODE_FP64)
    s = P.test_symmetry(mode=R.MODE_FP64_STENCIL)
    assert s["depsym_spmv"] <= 1.0 and s["depsym_mg"] <= 1.0
    P.close()


def test_stencil_mode_benchmark_protocol():
    res, rep = B.run(32, 32, 32, running_time=0, verify=True, mode=R.MODE_FP64_STENCIL)
    assert res["valid"] == 1 and res["opt_setup_niters"] <= 53
    assert "implicit stencil" in rep["Implementation"]["Precision"]
