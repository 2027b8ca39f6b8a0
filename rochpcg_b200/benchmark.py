"""The HPCG benchmark protocol on one B200 (src/main.cpp:174-563 and
src/ReportResults.cpp): set-up, CheckProblem, reference SpMV+MG timing, the
50-iteration reference residual, OptimizeProblem, TestCG, TestSymmetry, the
optimized CG set-up run, timed CG sets, TestNorms and the rating with
convergence and optimisation overhead.  The report is a JSON document with the
sections and field names of the reference's YAML report.

    python -m rochpcg_b200.benchmark [nx ny nz rt] [--nx=N --ny=N --nz=N --rt=S --tol=T --dev=D]
                                     [--pz= --zl= --zu= --npx= --npy= --npz=]
                                     [--mode=fp64|mixed|fp64_stencil] [--out=FILE]

Arguments follow the reference driver (src/init.cpp:112-183): positional
nx ny nz rt (values below 10 ignored), or --nx= ... --rt=; --tol=T skips the
reference phases and uses T as the reference tolerance; --dev=D runs on CUDA
device D.  With no grid argument at all the grid (and, without --rt=, the
run time) come from hpcg.dat in the working directory (src/ReadHpcgDat.cpp:
two title lines, then nx ny nz, then the seconds, then npx npy npz).  A
dimension below 16 becomes the largest of the others, at least 16; rt = 0
(the default without hpcg.dat) is the QuickPath: one timed CG set.  The
process-grid flags (--pz= --zl= --zu= --npx= --npy= --npz=) are read as the
reference reads them; this driver runs one rank, so a grid of more than one
rank is refused (the decomposed solve is rochpcg_b200.dist).
"""
from __future__ import annotations

import ctypes
import json
import os
import sys
import time

from . import MODE_FP64, MODE_FP64_STENCIL, MODE_MIXED, check, load

MAX_LEVELS = 8


class Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("running_time", ctypes.c_int),
                ("verify", ctypes.c_int), ("tol", ctypes.c_double), ("mode", ctypes.c_int)]


_LL8 = ctypes.c_longlong * MAX_LEVELS


class Result(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("mode", ctypes.c_int),
        ("verify", ctypes.c_int), ("quick_path", ctypes.c_int), ("levels", ctypes.c_int),
        ("rows", _LL8), ("nonzeros", _LL8),
        ("presmoother_steps", ctypes.c_int), ("postsmoother_steps", ctypes.c_int),
        ("times", ctypes.c_double * 10), ("optimize_problem_bytes", ctypes.c_double),
        ("check_problem_errors", ctypes.c_longlong),
        ("ref_max_iters", ctypes.c_int), ("ref_niters", ctypes.c_int), ("ref_tolerance", ctypes.c_double),
        ("opt_max_iters", ctypes.c_int), ("opt_setup_niters", ctypes.c_int), ("tolerance_failures", ctypes.c_int),
        ("err_count", ctypes.c_int), ("global_failure", ctypes.c_int), ("opt_worst_time", ctypes.c_double),
        ("cg_sets", ctypes.c_int),
        ("testcg_count_pass", ctypes.c_int), ("testcg_count_fail", ctypes.c_int),
        ("testcg_expected_niters_no_prec", ctypes.c_int), ("testcg_expected_niters_prec", ctypes.c_int),
        ("testcg_niters_max_no_prec", ctypes.c_int), ("testcg_niters_max_prec", ctypes.c_int),
        ("depsym_spmv", ctypes.c_double), ("depsym_mg", ctypes.c_double), ("symmetry_count_fail", ctypes.c_int),
        ("norms_mean", ctypes.c_double), ("norms_variance", ctypes.c_double), ("norms_pass", ctypes.c_int),
        ("fnops", ctypes.c_double), ("frefnops", ctypes.c_double),
        ("gflops_raw", ctypes.c_double), ("gflops_convergence", ctypes.c_double), ("gflops_final", ctypes.c_double),
        ("gflops_hpcg24", ctypes.c_double), ("gbs_raw", ctypes.c_double), ("gbs_final", ctypes.c_double),
        ("memory_total_gb", ctypes.c_double), ("valid", ctypes.c_int),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if isinstance(v, ctypes.Array):
                v = list(v)[: self.levels] if name in ("rows", "nonzeros") else list(v)
            out[name] = v
        return out


def report(result: Result, L=None) -> dict:
    """The JSON report of a filled Result (host only; no device needed)."""
    L = L or load()
    n = ctypes.c_size_t()
    check(L, L.hpcgb200_benchmark_report(ctypes.byref(result), None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    check(L, L.hpcgb200_benchmark_report(ctypes.byref(result), buf, n.value + 1, ctypes.byref(n)))
    return json.loads(buf.value.decode())


def run(nx: int, ny: int | None = None, nz: int | None = None, running_time: int = 0, verify: bool = True,
        tol: float = 0.0, mode: int = MODE_FP64) -> tuple[dict, dict]:
    """Runs the protocol on the current device; returns (result fields, report)."""
    L = load()
    p = Params(nx, ny if ny is not None else nx, nz if nz is not None else nx, int(running_time), int(verify),
               float(tol), int(mode))
    r = Result()
    check(L, L.hpcgb200_benchmark_run(ctypes.byref(p), ctypes.byref(r)))
    return r.as_dict(), report(r, L)


_PREFIXES = ("--nx=", "--ny=", "--nz=", "--rt=", "--pz=", "--zl=", "--zu=", "--npx=", "--npy=", "--npz=", "--dev=")


def _leading_int(text: str):
    """The integer sscanf("%d") reads at the start of `text`, or None."""
    text = text.lstrip()
    n = 0
    if n < len(text) and text[n] in "+-":
        n += 1
    while n < len(text) and text[n].isdigit():
        n += 1
    try:
        return int(text[:n])
    except ValueError:
        return None


def read_hpcg_dat(path: str = "hpcg.dat"):
    """src/ReadHpcgDat.cpp:42-75: ([nx, ny, nz], seconds, [npx, npy, npz]) from
    the file, or None when it cannot be opened.  Two title lines are skipped; a
    dimension that is missing or below 16 becomes 16, a missing or negative time
    30 minutes, a missing or non-positive process dimension 0 (unspecified)."""
    try:
        with open(path) as f:
            lines = f.read().split("\n")
    except OSError:
        return None
    body = lines[2:] + ["", "", ""]
    dims_tok = body[0].split()
    dims = []
    for i in range(3):
        v = _leading_int(dims_tok[i]) if i < len(dims_tok) else None
        dims.append(v if v is not None and v >= 16 else 16)
    t = _leading_int(body[1].split()[0]) if body[1].split() else None
    seconds = t if t is not None and t >= 0 else 30 * 60
    proc_tok = body[2].split()
    procs = []
    for i in range(3):
        v = _leading_int(proc_tok[i]) if i < len(proc_tok) else None
        procs.append(v if v is not None and v >= 1 else 0)
    return dims, seconds, procs


def parse_args(argv: list[str], dat_path: str = "hpcg.dat") -> dict:
    """src/init.cpp:112-183 for one rank (hpcg.dat when no grid argument is
    given), plus --mode= and --out=."""
    ip = [0] * len(_PREFIXES)
    for i in range(len(_PREFIXES)):
        v = _leading_int(argv[i]) if i < len(argv) else None
        ip[i] = v if v is not None and v >= 10 else 0
    verify, tol, mode, out = True, 0.0, MODE_FP64, None
    for a in argv:
        for j, k in enumerate(_PREFIXES):
            if a.startswith(k):
                v = _leading_int(a[len(k):])
                ip[j] = v if v is not None else 0
        if a.startswith("--tol="):
            tol, verify = float(a[6:]), False
        elif a.startswith("--mode="):
            mode = {"fp64": MODE_FP64, "mixed": MODE_MIXED, "fp64_stencil": MODE_FP64_STENCIL}[a[7:]]
        elif a.startswith("--out="):
            out = a[6:]
    if not ip[0] and not ip[1] and not ip[2]:
        dat = read_hpcg_dat(dat_path)
        if dat is not None:
            ip[0:3] = dat[0]
            if not ip[3]:
                ip[3] = dat[1]
            ip[7:10] = dat[2]
    # (the library applies the small-dimension rule, src/init.cpp:150-160)
    npx, npy, npz = ip[7:10]
    if max(npx, 1) * max(npy, 1) * max(npz, 1) > 1:
        raise ValueError(f"process grid {npx}x{npy}x{npz}: this driver runs one rank (the decomposed solve is "
                         "rochpcg_b200.dist)")
    return dict(nx=ip[0], ny=ip[1], nz=ip[2], running_time=ip[3], verify=verify, tol=tol, mode=mode, out=out,
                device=ip[10] if any(a.startswith("--dev=") for a in argv) else -1)


def main(argv=None):
    # load every kernel when the CUDA context is created (before the timed set-up
    # phase) rather than at each kernel's first launch inside it
    os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")
    a = parse_args(sys.argv[1:] if argv is None else argv)
    out = a.pop("out")
    L = load()
    check(L, L.hpcgb200_init(a.pop("device")))
    res, rep = run(**a)
    text = json.dumps(rep, indent=1)
    if out is None:
        out = time.strftime("HPCG-Benchmark_3.1_%Y-%m-%d_%H-%M-%S.json")
    with open(out, "w") as f:
        f.write(text + "\n")
    fs = rep["Final Summary"]
    rating = fs.get("HPCG result is VALID with a GFLOP/s rating of")
    print(f"grid {res['nx']}x{res['ny']}x{res['nz']}, {res['cg_sets']} CG set(s) of {res['opt_max_iters']} "
          f"iterations in {res['times'][0]:.3f} s; "
          + (f"VALID, rating {rating:.1f} GFLOP/s" if rating is not None else "INVALID") + f"; report: {out}")
    return 0 if res["valid"] else 1


if __name__ == "__main__":
    sys.exit(main())
