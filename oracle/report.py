"""Test oracle (never part of the product): the HPCG report arithmetic restated
in plain Python, to check the library's report numbers on the CPU.

Follows rocHPCG 0.8.9 src/ReportResults.cpp:65-94 (ComputeTotalGFlops),
:134-158 (FLOP model), :160-195 (memory traffic model), :396-418 (GB/s and
GFLOP/s summaries), :430 (validity), src/TestNorms.cpp:31-46 (TestNorms) and
src/init.cpp:150-159 (small-dimension rule).
"""
from __future__ import annotations


def adjust_dims(nx: int, ny: int, nz: int) -> tuple[int, int, int]:
    """src/init.cpp:150-159."""
    d = [nx, ny, nz]
    for i in range(3):
        if d[i] < 16:
            for j in (1, 2):
                if d[(i + j) % 3] > d[i]:
                    d[i] = d[(i + j) % 3]
        if d[i] < 16:
            d[i] = 16
    return tuple(d)


def test_norms(values: list[float]) -> tuple[float, float, bool]:
    """src/TestNorms.cpp:31-46: mean (as a shifted sum), variance, pass."""
    n = len(values)
    mean_delta = sum(v - values[0] for v in values)
    mean = values[0] + mean_delta / n
    var = sum((v - mean) * (v - mean) for v in values) / n
    return mean, var, var < 1.0e-6


def model(rows, nnz, sets, ref_max_iters, opt_max_iters, times, pre=1, post=1) -> dict:
    """Report figures from per-level rows/nonzeros (level 0 first)."""
    L = len(rows)
    fniters = sets * float(opt_max_iters)
    fnrow, fnnz = float(rows[0]), float(nnz[0])
    ddot = (3.0 * fniters + sets) * 2.0 * fnrow                      # :140
    waxpby = (3.0 * fniters + sets) * 2.0 * fnrow                    # :141
    spmv = (fniters + sets) * 2.0 * fnnz                             # :142
    precond = 0.0
    for i in range(L - 1):                                           # :147-153
        precond += pre * fniters * 4.0 * nnz[i]
        precond += fniters * 2.0 * nnz[i]
        precond += post * fniters * 4.0 * nnz[i]
    precond += fniters * 4.0 * nnz[L - 1]                            # :156
    fnops = ddot + waxpby + spmv + precond
    frefnops = fnops * ref_max_iters / opt_max_iters                 # :158
    d8, i4 = 8.0, 4.0
    reads = (3.0 * fniters + sets) * 2.0 * fnrow * d8 * 2            # ddot + waxpby reads (:163,:165)
    writes = (3.0 * fniters + sets) * d8 + (3.0 * fniters + sets) * fnrow * d8
    reads += (fniters + sets) * (fnnz * (d8 + i4) + fnrow * d8)      # :167
    writes += (fniters + sets) * fnrow * d8                          # :169
    for i in range(L - 1):                                           # :174-186
        nz_, nr = float(nnz[i]), float(rows[i])
        reads += pre * fniters * (2.0 * nz_ * (d8 + i4) + nr * d8)
        writes += pre * fniters * nr * d8
        reads += fniters * (nz_ * (d8 + i4) + nr * d8)
        writes += fniters * nz_ * d8
        reads += post * fniters * (2.0 * nz_ * (d8 + i4) + nr * d8)
        writes += post * fniters * nz_ * d8
    reads += fniters * (2.0 * nnz[L - 1] * (d8 + i4) + rows[L - 1] * d8)  # :190
    writes += fniters * rows[L - 1] * d8                             # :191
    conv = ref_max_iters / opt_max_iters
    overhead = times[0] + sets * (times[7] / 10.0 + times[9] / 10.0)
    return {
        "Raw DDOT": ddot, "Raw WAXPBY": waxpby, "Raw SpMV": spmv, "Raw MG": precond, "Total": fnops,
        "Total with convergence overhead": frefnops,
        "raw_gflops": fnops / times[0] / 1e9,                        # :409
        "convergence_gflops": frefnops / times[0] / 1e9,             # :410
        "final_gflops": frefnops / overhead / 1e9,                   # :412
        "gflops24": frefnops / (times[0] + sets * times[7] / 10.0) / 1e9,  # :413
        "raw_gbs": (reads + writes) / times[0] / 1e9,                # :400
        "final_gbs": (reads + writes) * conv / overhead / 1e9,       # :401
        "opt_vs_ref": times[7] / times[8],                           # :418
    }
