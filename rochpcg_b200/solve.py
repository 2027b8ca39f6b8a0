"""One HPCG solve from the command line (the build's solver CLI, beside the
benchmark protocol of ``rochpcg_b200.benchmark``).

    python -m rochpcg_b200.solve [nx ny nz] [--nx=N --ny=N --nz=N] [--precision=fp64|mixed|fp64_stencil]
                                 [--smoother=symgs|learned] [--rhs=ones|normal:SEED] [--tol=T]
                                 [--max-iter=K] [--out=FILE]

The grid arguments follow the reference driver (src/init.cpp:112-183: positional
nx ny nz, or --nx= ...; a missing dimension takes nx).  --rhs=ones solves the
generated system (b_i = 27 - nonzeros of row i, exact solution all ones);
normal:SEED draws b ~ N(0,1) from SEED.  --smoother=learned replaces SymGS on MG
levels 2-3 with the committed conv-net smoother (FP32 V-cycle, flexible CG,
SymGS fallback).  Prints one JSON object: time, iterations, the recurrence's
relative residual and the FP64 true residual ||b - A x|| / ||b||, and the HPCG
flop rate of the solve.
"""
from __future__ import annotations

import json
import sys

MODES = {"fp64": "MODE_FP64", "mixed": "MODE_MIXED", "fp64_stencil": "MODE_FP64_STENCIL"}


def parse_args(argv: list[str]) -> dict:
    """Host-only argument parsing (no device needed)."""
    dims = [0, 0, 0]
    pos = [a for a in argv if not a.startswith("--")]
    for i in range(min(3, len(pos))):
        dims[i] = int(pos[i])
    a = dict(precision="fp64", smoother="symgs", rhs=("ones", None), tol=1e-9, max_iter=1000, out=None)
    for arg in argv:
        if not arg.startswith("--"):
            continue
        key, _, val = arg[2:].partition("=")
        if key in ("nx", "ny", "nz"):
            dims["xyz".index(key[1])] = int(val)
        elif key == "precision":
            if val not in MODES:
                raise ValueError(f"--precision must be one of {sorted(MODES)}")
            a["precision"] = val
        elif key == "smoother":
            if val not in ("symgs", "learned"):
                raise ValueError("--smoother must be symgs or learned")
            a["smoother"] = val
        elif key == "rhs":
            if val == "ones":
                a["rhs"] = ("ones", None)
            elif val.startswith("normal:"):
                a["rhs"] = ("normal", int(val[7:]))
            else:
                raise ValueError("--rhs must be ones or normal:SEED")
        elif key == "tol":
            a["tol"] = float(val)
        elif key == "max-iter":
            a["max_iter"] = int(val)
        elif key == "out":
            a["out"] = val
        else:
            raise ValueError(f"unknown option --{key}")
    nx = dims[0] or 128
    a["dims"] = (nx, dims[1] or nx, dims[2] or nx)
    if a["smoother"] == "learned" and a["precision"] == "fp64_stencil":
        raise ValueError("the learned smoother runs in the FP32 V-cycle (--precision=mixed or fp64)")
    return a


def run(a: dict) -> dict:
    import rochpcg_b200 as R
    from rochpcg_b200.rhs import normal_rhs

    P = R.Problem(*a["dims"])
    try:
        mode = getattr(R, MODES[a["precision"]])
        if a["rhs"][0] == "normal":
            P.set_rhs(normal_rhs(P.rows[0], a["rhs"][1]))
        smoother = None
        if a["smoother"] == "learned":
            from rochpcg_b200 import learned

            smoother = learned.Smoother.load()
            P.set_smoother(smoother, first_level=2)
            mode = R.MODE_LEARNED
        res = P.cg(a["max_iter"], a["tol"], mode=mode)
        flops_it, _ = P.model()
        out = {"grid": list(a["dims"]), "precision": a["precision"], "smoother": a["smoother"],
               "rhs": a["rhs"][0] if a["rhs"][1] is None else f"normal:{a['rhs'][1]}", "tol": a["tol"],
               "iterations": res["niters"], "seconds": res["seconds"],
               "rel_residual_recurrence": res["normr"] / res["normr0"], "rel_residual_fp64_true": P.true_residual(),
               "gflops_hpcg_model": flops_it * res["niters"] / res["seconds"] / 1e9 if res["seconds"] > 0 else None}
        if smoother is not None:
            out["fallback_iteration"] = P.last_fallback()
            P.set_smoother(None)
        return out
    finally:
        P.close()


def main(argv=None) -> int:
    a = parse_args(sys.argv[1:] if argv is None else argv)
    out = run(a)
    text = json.dumps(out)
    print(text)
    if a["out"]:
        with open(a["out"], "w") as f:
            f.write(text + "\n")
    return 0 if out["rel_residual_fp64_true"] <= 2 * a["tol"] else 1


if __name__ == "__main__":
    sys.exit(main())
