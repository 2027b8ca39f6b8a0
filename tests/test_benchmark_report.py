"""The benchmark report on the CPU: the library's report arithmetic (FLOP and
traffic models, ratings with convergence and optimisation overhead, validity,
JSON layout) against the restatement of src/ReportResults.cpp in
oracle/report.py, and the driver's argument rules (src/init.cpp)."""
import ctypes
import math
import os

import numpy as np
import pytest

from oracle import report as OR
from rochpcg_b200 import MODE_FP64, MODE_MIXED
from rochpcg_b200 import benchmark as B


def grid_counts(nx, ny, nz, levels=4):
    """Rows and nonzeros of the generated 27-point hierarchy."""
    rows, nnz = [], []
    for _ in range(levels):
        rows.append(nx * ny * nz)
        nnz.append((3 * nx - 2) * (3 * ny - 2) * (3 * nz - 2))
        nx, ny, nz = nx // 2, ny // 2, nz // 2
    return rows, nnz


def filled(nx=256, ny=256, nz=256, sets=3, opt_iters=51, times=None, **kw):
    r = B.Result()
    r.nx, r.ny, r.nz, r.levels = nx, ny, nz, 4
    rows, nnz = grid_counts(nx, ny, nz)
    for i in range(4):
        r.rows[i], r.nonzeros[i] = rows[i], nnz[i]
    r.presmoother_steps = r.postsmoother_steps = 1
    t = times or {0: 2.1, 1: 0.0, 2: 0.0, 3: 0.0, 5: 0.0, 7: 0.9, 8: 0.004, 9: 0.35}
    for k, v in t.items():
        r.times[k] = v
    r.ref_max_iters, r.opt_max_iters, r.cg_sets = 50, opt_iters, sets
    r.norms_pass = 1
    r.optimize_problem_bytes = 1.0e9
    for k, v in kw.items():
        setattr(r, k, v)
    return r, rows, nnz


def test_report_matches_reference_formulas():
    r, rows, nnz = filled()
    rep = B.report(r)
    ref = OR.model(rows, nnz, r.cg_sets, 50, r.opt_max_iters, list(r.times))
    fl = rep["Floating Point Operations Summary"]
    for k in ("Raw DDOT", "Raw WAXPBY", "Raw SpMV", "Raw MG", "Total", "Total with convergence overhead"):
        assert fl[k] == pytest.approx(ref[k], rel=1e-15), k
    g = rep["GFLOP/s Summary"]
    assert g["Raw Total"] == pytest.approx(ref["raw_gflops"], rel=1e-14)
    assert g["Total with convergence overhead"] == pytest.approx(ref["convergence_gflops"], rel=1e-14)
    assert g["Total with convergence and optimization phase overhead"] == pytest.approx(ref["final_gflops"], rel=1e-14)
    # a phase whose time is 0 has no rate: null, not infinity
    assert g["Raw DDOT"] is None and g["Raw MG"] is None
    bw = rep["GB/s Summary"]
    assert bw["Raw Total B/W"] == pytest.approx(ref["raw_gbs"], rel=1e-14)
    assert bw["Total with convergence and optimization phase overhead"] == pytest.approx(ref["final_gbs"], rel=1e-14)
    fs = rep["Final Summary"]
    assert fs["HPCG result is VALID with a GFLOP/s rating of"] == pytest.approx(ref["final_gflops"], rel=1e-14)
    assert fs["HPCG 2.4 rating for historical reasons is"] == pytest.approx(ref["gflops24"], rel=1e-14)
    assert rep["User Optimization Overheads"]["Optimization phase time vs reference SpMV+MG time"] == \
        pytest.approx(ref["opt_vs_ref"], rel=1e-14)
    assert r.valid == 1 and r.gflops_final == pytest.approx(ref["final_gflops"], rel=1e-14)
    # the model figures per iteration at 256^3 (6.2241e9 flop per iteration)
    per_it = (fl["Total"] - r.cg_sets * (2 * rows[0] + 2 * rows[0] + 2 * nnz[0])) / (r.cg_sets * r.opt_max_iters)
    assert per_it == pytest.approx(6.2241e9, rel=1e-4)


def test_report_layout_and_coarse_grids():
    r, rows, nnz = filled(nx=64, ny=32, nz=48, sets=1, opt_iters=50)
    rep = B.report(r)
    assert rep["HPCG-Benchmark version"] == "3.1"
    assert rep["Global Problem Dimensions"] == {"Global nx": 64, "Global ny": 32, "Global nz": 48}
    mg = rep["Multigrid Information"]
    assert mg["Number of coarse grid levels"] == 3
    assert [c["Number of Equations"] for c in mg["Coarse Grids"]] == rows[1:]
    assert [c["Number of Nonzero Terms"] for c in mg["Coarse Grids"]] == nnz[1:]
    assert rep["Linear System Information"] == {"Number of Equations": rows[0], "Number of Nonzero Terms": nnz[0]}
    it = rep["Iteration Count Information"]
    assert it["Total number of reference iterations"] == 50 and it["Total number of optimized iterations"] == 50
    mem = rep["Memory Use Information"]
    assert mem["Memory used for OptimizeProblem data (Gbytes)"] == pytest.approx(1.0)
    assert mem["Total memory used for data (Gbytes)"] > mem["Memory used for linear system and CG (Gbytes)"]


@pytest.mark.parametrize("field,value", [("testcg_count_fail", 1), ("symmetry_count_fail", 1), ("norms_pass", 0),
                                         ("global_failure", 1), ("check_problem_errors", 3)])
def test_report_invalid_when_a_check_fails(field, value):
    r, _, _ = filled(**{field: value})
    rep = B.report(r)
    assert r.valid == 0
    assert rep["Final Summary"] == {"HPCG result is": "INVALID."}


def test_report_mixed_mode_is_labelled():
    r, _, _ = filled(mode=MODE_MIXED)
    rep = B.report(r)
    assert "FP32" in rep["Implementation"]["Precision"]
    assert "Mixed precision" in rep["Final Summary"]


def test_report_buffer_too_small_reports_length():
    from rochpcg_b200 import load

    L = load()
    r, _, _ = filled()
    n = ctypes.c_size_t()
    assert L.hpcgb200_benchmark_report(ctypes.byref(r), None, 0, ctypes.byref(n)) == 0
    buf = ctypes.create_string_buffer(16)
    assert L.hpcgb200_benchmark_report(ctypes.byref(r), buf, 16, ctypes.byref(n)) != 0
    assert n.value > 1000


def test_test_norms_restatement():
    vals = [1e-9 * (1 + 1e-3 * i) for i in range(7)]
    mean, var, ok = OR.test_norms(vals)
    assert math.isclose(mean, float(np.mean(vals)), rel_tol=1e-12) and ok


@pytest.mark.parametrize("argv,want", [
    (["104", "104", "104", "60"], dict(nx=104, ny=104, nz=104, running_time=60, verify=True)),
    (["--nx=256", "--ny=256", "--nz=128", "--rt=0"], dict(nx=256, ny=256, nz=128, running_time=0, verify=True)),
    (["--nx=32", "--tol=1e-6"], dict(nx=32, ny=0, nz=0, verify=False, tol=1e-6)),
    (["8", "9", "5"], dict(nx=0, ny=0, nz=0)),
    (["--nx=64", "--mode=mixed"], dict(nx=64, mode=MODE_MIXED)),
    (["--nx=64", "--mode=fp64_stencil"], dict(nx=64, mode=3)),
])
def test_driver_arguments(argv, want):
    a = B.parse_args(argv)
    for k, v in want.items():
        assert a[k] == v, (k, a)
    assert a["mode"] in (MODE_FP64, MODE_MIXED, 3)


@pytest.mark.parametrize("dims,want", [((0, 0, 0), (16, 16, 16)), ((32, 0, 0), (32, 32, 32)),
                                       ((8, 24, 4), (24, 24, 24)), ((104, 16, 200), (104, 16, 200))])
def test_small_dimension_rule(dims, want):
    assert OR.adjust_dims(*dims) == want


def _dat(tmp_path, text):
    p = tmp_path / "hpcg.dat"
    p.write_text(text)
    return str(p)


def test_hpcg_dat_fallback(tmp_path):
    """src/init.cpp:143-147 + src/ReadHpcgDat.cpp: with no grid argument the
    grid and the seconds come from hpcg.dat; a nonzero --rt= wins over the
    file's time (--rt=0 counts as not given, as in the reference); a grid
    argument skips the file."""
    dat = _dat(tmp_path, "HPCG benchmark input file\nsecond title line\n104 104 96\n60\n")
    a = B.parse_args([], dat_path=dat)
    assert (a["nx"], a["ny"], a["nz"], a["running_time"]) == (104, 104, 96, 60)
    a = B.parse_args(["--rt=5", "--mode=mixed"], dat_path=dat)
    assert (a["nx"], a["running_time"], a["mode"]) == (104, 5, MODE_MIXED)
    assert B.parse_args(["--rt=0"], dat_path=dat)["running_time"] == 60
    a = B.parse_args(["--nx=32"], dat_path=dat)
    assert (a["nx"], a["ny"], a["running_time"]) == (32, 0, 0)
    # missing file: nothing read
    a = B.parse_args([], dat_path=str(tmp_path / "absent.dat"))
    assert (a["nx"], a["ny"], a["nz"], a["running_time"]) == (0, 0, 0, 0)


def test_hpcg_dat_defaults():
    """Values below 16 (or absent) become 16, a missing or negative time 30
    minutes, missing process dimensions 0."""
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "hpcg.dat")
        with open(p, "w") as f:
            f.write("t\nt\n8 200\n-5\n2 x\n")
        dims, seconds, procs = B.read_hpcg_dat(p)
        assert dims == [16, 200, 16] and seconds == 1800 and procs == [2, 0, 0]
        with open(p, "w") as f:
            f.write("only one line\n")
        assert B.read_hpcg_dat(p) == ([16, 16, 16], 1800, [0, 0, 0])


def test_device_and_process_grid_flags(tmp_path):
    absent = str(tmp_path / "none.dat")
    assert B.parse_args(["--nx=64", "--dev=3"], dat_path=absent)["device"] == 3
    assert B.parse_args(["--nx=64"], dat_path=absent)["device"] == -1
    # one rank: a process grid of one is accepted, a larger one refused
    assert B.parse_args(["--nx=64", "--npx=1", "--npy=1", "--npz=1"], dat_path=absent)["nx"] == 64
    with pytest.raises(ValueError):
        B.parse_args(["--nx=64", "--npx=2"], dat_path=absent)
    dat = _dat(tmp_path, "t\nt\n64 64 64\n0\n2 2 1\n")
    with pytest.raises(ValueError):
        B.parse_args([], dat_path=dat)
