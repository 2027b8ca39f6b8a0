"""The reference-operator residual checker (oracle/residual_check.py) that
bench.py uses to verify every solve's final x on the host: its worker
rebuilds the reference's own problem and right-hand sides, so the residual of
the exact solution (all ones, generated b) is exactly zero, and the residual
of a CG_ref solution equals the one CG_ref reports (the reference's
ComputeSPMV_ref and norms on both sides)."""
import numpy as np

from oracle.oracle import RefProblem
from oracle.residual_check import RefResidualChecker
from rochpcg_b200.rhs import normal_rhs


def test_checker_matches_reference_cg_residuals():
    grid = (16, 16, 24)
    P = RefProblem(*grid)
    m = P.nrows[0]
    r1 = P.cg(8, 0.0)  # generated b
    bn = normal_rhs(m, 5)
    r2 = P.cg(8, 0.0, b=bn)
    C = RefResidualChecker(threads=2)
    try:
        C.prepare(grid)
        C.submit("ones", grid, ("generated",), np.ones(m))
        C.submit("cg_generated", grid, ("generated",), r1["x"])
        C.submit("cg_normal", grid, ("normal", 5), r2["x"])
        C.submit("bad_grid", (3, 3, 0), ("generated",), np.ones(1))
        v = C.results(timeout_s=120)
    finally:
        C.close()
    assert v["ones"] == 0.0
    # CG_ref's normr is the recurrence residual; after 8 iterations it equals
    # the true residual to many digits
    assert abs(v["cg_generated"] - r1["normr"] / r1["normr0"]) <= 1e-6 * v["cg_generated"]
    b_norm = np.linalg.norm(bn)
    assert abs(v["cg_normal"] - r2["normr"] / b_norm) <= 1e-6 * v["cg_normal"]
    assert v["bad_grid"] is None and "bad_grid" in C.errors
