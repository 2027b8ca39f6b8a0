"""The solver CLI (python -m rochpcg_b200.solve) on the B200: every precision,
both smoothers and both right-hand sides reach the tolerance, verified by the
FP64 true residual."""
import json

import pytest

from rochpcg_b200 import solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("argv", [
    ["32", "--precision=fp64"],
    ["32", "24", "16", "--precision=fp64_stencil", "--rhs=normal:3"],
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
