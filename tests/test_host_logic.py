"""Host-side logic that needs no device: the HPCG flop / byte model, the
seeded right-hand side generator, and bench.py's result assembly."""
import json
import os
import subprocess
import sys

import numpy as np

import rochpcg_b200 as R
from rochpcg_b200.rhs import normal_rhs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def level_dims(n):
    return [(n >> l, n >> l, n >> l) for l in range(4)]


def stencil_nnz(d):
    return (3 * d[0] - 2) * (3 * d[1] - 2) * (3 * d[2] - 2)


def test_hpcg_model_256():
    dims = level_dims(256)
    flops, bytes_ = R.hpcg_model(dims, [stencil_nnz(d) for d in dims])
    # src/ReportResults.cpp:140-195 evaluated for one iteration at 256^3
    assert abs(flops - 6.2241e9) / 6.2241e9 < 1e-4
    assert abs(bytes_ - 4.7224e10) / 4.7224e10 < 1e-4


def test_hpcg_model_matches_reference_formula_small():
    dims = level_dims(32)
    nnz = [stencil_nnz(d) for d in dims]
    flops, _ = R.hpcg_model(dims, nnz)
    assert abs(flops - 1.1444e7) / 1.1444e7 < 1e-3


def test_normal_rhs_deterministic_and_normal():
    a = normal_rhs(1 << 16, 0)
    b = normal_rhs(1 << 16, 0)
    c = normal_rhs(1 << 16, 1)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    assert abs(a.mean()) < 0.02 and abs(a.std() - 1) < 0.02
    # chunking does not change values
    assert np.array_equal(normal_rhs(1000, 7, chunk=64), normal_rhs(1000, 7))


def test_bench_reference_arm_schema():
    """bench.py --impl reference prints one JSON line with the contract's keys
    (tiny sample so it runs in seconds on CPU)."""
    env = dict(os.environ, HPCG_BENCH_REF_SAMPLE="16", OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "1"], capture_output=True, text=True, env=env, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    if "unavailable" in d:
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "impl",
              "cpu_baseline", "e2e", "config"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "reference"


def test_solve_cli_arguments():
    """python -m rochpcg_b200.solve: the reference's grid arguments plus the
    solver flags (host-only parsing)."""
    import pytest
    from rochpcg_b200.solve import parse_args

    a = parse_args(["64", "32", "16", "--precision=mixed", "--rhs=normal:9999", "--tol=1e-8"])
    assert a["dims"] == (64, 32, 16) and a["precision"] == "mixed" and a["rhs"] == ("normal", 9999)
    assert a["tol"] == 1e-8 and a["smoother"] == "symgs"
    a = parse_args(["--nx=96", "--smoother=learned"])
    assert a["dims"] == (96, 96, 96) and a["smoother"] == "learned" and a["rhs"] == ("ones", None)
    assert parse_args([])["dims"] == (128, 128, 128)
    for bad in (["--precision=fp16"], ["--rhs=uniform"], ["--smoother=jacobi"], ["--bogus=1"],
                ["--precision=fp64_stencil", "--smoother=learned"]):
        with pytest.raises(ValueError):
            parse_args(bad)
