"""The solver CLI (python -m rochpcg_b200.solve) on the B200: every precision,
both smoothers and both right-hand sides reach the tolerance, verified by the
FP64 true residual."""
import json

import pytest

from rochpcg_b200 import solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("argv", [
    ["32", "--precision=fp64"],
    ["40", "24", "16", "--precision=fp64_stencil", "--rhs=normal:3"],
    ["64", "--precision=mixed", "--rhs=normal:0"],
    ["64", "--precision=mixed", "--smoother=learned", "--rhs=normal:9999"],
])
def test_solve_cli(argv, tmp_path, capsys):
    out = tmp_path / "r.json"
    assert solve.main(argv + ["--tol=1e-9", f"--out={out}"]) == 0
    r = json.loads(out.read_text())
    assert r == json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert r["rel_residual_recurrence"] <= 1e-9
    assert r["rel_residual_fp64_true"] <= 2e-9
    assert r["iterations"] > 0 and r["gflops_hpcg_model"] > 0


def test_solve_cli_reports_a_coloring_that_does_not_end():
    """32x24x16 has a 4x3x2 coarsest level, where the JPL loop's stop rule
    (colored == m, MultiColoring.cpp:281) is never met: a round that draws a
    colour value drawn before counts its rows twice.  The reference loops
    there; the library ends after 64 rounds with HPCGB200_ERR_COLORING."""
    from rochpcg_b200 import HpcgError

    with pytest.raises(HpcgError, match="JPL coloring did not finish"):
        solve.main(["32", "24", "16", "--tol=1e-9"])
