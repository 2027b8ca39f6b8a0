#!/usr/bin/env python
"""Benchmark: HPCG multigrid-preconditioned CG on B200.

Default workload (one GPU): a 256^3 HPCG problem (16.8M rows, 449M nonzeros,
4-level MG, generated b with exact solution 1, x0 = 0) solved to relative
residual 1e-9 by the plain FP64 drop-in path.  One step = one full solve.
`value` is HPCG GFLOP/s (src/ReportResults.cpp flop model x iterations /
device time).  The same line carries:

  e2e          the same solve through the C ABI from pinned HOST buffers
               (b in, x out, copies inside the timed region)
  roofline     the dominant kernel (level-0 full SymGS colour sweep) against
               the measured HBM copy bandwidth
  cpu_baseline the reference's own CPU path (CG_ref, OpenMP) on a bounded
               sample, timed on this machine's host cores
  fp64_stencil the same 256^3 solve with the V-cycle and SpMV on the implicit
               stencil (HPCGB200_MODE_FP64_STENCIL): the FP64 residual history
               bit for bit without matrix reads
  mixed        FP64-outer / FP32 V-cycle solve at 320^3 with b ~ N(0,1)
               (seed 0) vs the FP64 path (ELL and implicit) on the same
               system, all verified with an FP64 true residual
  learned      the learned coarse-level smoother vs SymGS at 256^3
               (b ~ N(0,1), seed 9999), with the tcgen05 conv kernel's
               tensor roofline
  largest      560 x 560 x 280 (87.8M rows), FP64 vs mixed vs learned, for
               b ~ N(0,1) seed 7 and the generated b, with the fine-level
               sweep bandwidths
  every solve's final x is also checked on the host with the reference's
  own ComputeSPMV_ref (oracle/_ref, natural order) in a worker process that
  runs beside the GPU work: `rel_residual_ref_spmv` next to each
  `rel_residual_fp64_true`

`--impl reference` times the reference's CPU CG_ref on this machine instead.
Under torchrun (N>1) every rank solves its own local problem (HPCG weak
scaling with ExchangeHalo a single-rank no-op: replicas, no collective on the
data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to rel. residual 1e-9 & HPCG GFLOP/s: mixed/learned vs FP64, 1 B200"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--tol", type=float, default=1e-9)
    ap.add_argument("--mixed-nx", type=int, default=320)
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--max-iter", type=int, default=1000,
                    help="iteration cap per solve (profiling runs use a few iterations)")
    ap.add_argument("--lite", action="store_true",
                    help="solves only: no e2e, operator timing, CPU baseline (profiling runs)")
    ap.add_argument("--mixed-only", action="store_true", help="only the mixed-vs-FP64 comparison")
    ap.add_argument("--profile-case", choices=["conv", "sweep128", "spmv128", "mixed128", "mixed192", "cg128",
                                               "cgmixed192", "vcycle256", "mixed320", "net64", "stencil192"],
                    help="run one small case for a profiler and exit (no JSON line)")
    ap.add_argument("--no-largest", action="store_true",
                    help="skip the largest workload (560x560x280, FP64 vs mixed vs learned, seed-7 and all-ones rhs)")
    ap.add_argument("--no-refcheck", action="store_true",
                    help="skip the host check of each solve's x with the reference's ComputeSPMV_ref")
    ap.add_argument("--learned-nx", type=int, default=256)
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: independent replicas of the 1-GPU run instead of the decomposed solve")
    ap.add_argument("--emulate-ranks", type=int, default=0,
                    help="1 GPU: drive R ranks of the decomposed solve from this process (exchange by device "
                         "copies) to exercise the decomposed path; not a multi-GPU measurement")
    return ap.parse_args()


def level_dims(n):
    return [(n >> l, n >> l, n >> l) for l in range(4)]


def stencil_nnz(d):
    return (3 * d[0] - 2) * (3 * d[1] - 2) * (3 * d[2] - 2)


def model(n):
    from rochpcg_b200 import hpcg_model

    dims = level_dims(n)
    return hpcg_model(dims, [stencil_nnz(d) for d in dims])


def generated_b_natural(nx, ny, nz):
    """b_i = 26 - (nnz_i - 1) of the generated problem, natural order
    (src/GenerateProblem.cpp:298-301)."""
    def cnt(n):
        c = np.full(n, 3, np.int8)
        c[0] -= 1
        c[-1] -= 1
        return c
    cz, cy, cx = cnt(nz), cnt(ny), cnt(nx)
    nnz = (cz[:, None, None].astype(np.int32) * cy[None, :, None] * cx[None, None, :]).reshape(-1)
    return 27.0 - nnz.astype(np.float64)


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- helpers

def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(key: str):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary
    (profiles/ncu_traffic.txt: lines `key bytes_per_launch`), else None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for ln in open(p):
            parts = ln.split()
            if len(parts) >= 2 and parts[0] == key:
                return float(parts[1])
    except OSError:
        pass
    return None


def fp64_algorithmic_bytes_per_iter(rows_per_level):
    """Bytes one FP64 MG-PCG iteration of this implementation must move (the
    per-kernel algorithmic bytes, not the reference's traffic model), per
    level of m rows in 8 colours of m/8 rows, ELL width 27 (12 B per slot):

      zero-guess SymGS (8 forward + 7 backward colour launches): every slot
        but the diagonal read once (26 * 12); forward r, 1/a_ii, diag index,
        x written (28); backward (7 of 8 colours) diag index, x, a_ii,
        1/a_ii, x written (36 * 7/8); neighbour x of earlier / later colours,
        read once per launch (28 + 28)                        = 427.5 B/row
      fused SpMV + restriction (m/8 rows): 27 * 12 + rf + rc + two transfer
        indices (348 / 8), x of the whole fine grid once (8)     = 51.5 B/row
      prolongation (m/8 rows): indices, xc, xf read + written (32 / 8) = 4
      full SymGS (15 colour launches): per launch m/8 rows of
        27 * 12 + r + 1/a_ii + x written (348 / 8) + the other colours' x (7)
                                                                 = 757.5 B/row
      coarsest level: the zero-guess SymGS only                  = 427.5 B/row
      level 0 also: SpMV + p.Ap (27 * 12 + p + Ap = 340), r.z (16), p update
        (24), r and x update (48)                                 = 428 B/row
    """
    total = 0.0
    last = len(rows_per_level) - 1
    for l, m in enumerate(rows_per_level):
        per_row = 427.5 if l == last else 427.5 + 51.5 + 4.0 + 757.5
        if l == 0:
            per_row += 340.0 + 16.0 + 24.0 + 48.0
        total += per_row * m
    return total


def cpu_facts():
    """Model name and core counts of the host the CPU figures ran on."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        import psutil

        physical = psutil.cpu_count(logical=False)
    except Exception:
        physical = None
    return {"cpu_model": model, "physical_cores": physical, "logical_cpus": os.cpu_count()}


def cpu_baseline_sample(n: int, iters: int, min_seconds: float = 0.0):
    """The reference's CPU CG_ref (OpenMP, all host threads) on an n^3 sample:
    `iters` iterations from x0 = 0 on the generated b, repeated until at least
    min_seconds of solve time have been measured.  Returns (GFLOP/s, seconds
    per solve, iterations, solves)."""
    from oracle.oracle import RefProblem

    R = RefProblem(n, n, n)
    flops, _ = model(n)
    secs, its, solves = 0.0, 0, 0
    while solves == 0 or secs < min_seconds:
        r = R.cg(iters, 0.0)
        secs += r["seconds"]
        its = r["niters"]
        solves += 1
    per = secs / solves
    return flops * its / per / 1e9, per, its, solves


def host_threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def cpu_baseline(args):
    """The reference's CPU-runnable case (32^3, 50 CG_ref iterations, generated
    b, x0 = 0) is the primary CPU figure, repeated for about 10 s; a 128^3 x
    10-iteration sample shows the reference at a size whose working set leaves
    the caches."""
    facts = cpu_facts()
    out = {"unit": "GFLOP/s", "cores": host_threads(), "kind": "reference", **facts}
    try:
        g, per, its, solves = cpu_baseline_sample(32, 50, min_seconds=10.0)
        out.update(value=g, sample=f"CG_ref (reference src/*_ref.cpp, OpenMP, {host_threads()} threads) on 32^3 "
                                   f"(the reference's CPU-runnable case): {its} iterations from x0=0, generated b, "
                                   f"{solves} solves of {per * 1e3:.1f} ms")
        g2, per2, its2, _ = cpu_baseline_sample(128, 10)
        out["sample_128"] = {"value": g2, "unit": "GFLOP/s", "iterations": its2, "seconds": per2}
    except Exception as e:
        out.update(value=None, sample=f"unavailable: {e}")
    return out


# ------------------------------------------------------------ reference arm

def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    nx = int(os.environ.get("HPCG_BENCH_REF_SAMPLE", args.nx))
    try:
        from oracle.oracle import RefProblem, ref_lib

        ref_lib()
    except Exception as e:  # the reference library could not be built/loaded
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU path not loadable: {e}"}))
        return 0
    t0 = time.perf_counter()
    R = RefProblem(nx, nx, nx)
    setup_s = time.perf_counter() - t0
    flops_it, _ = model(nx)
    # one step = one CG_ref iteration (preamble + 1 iteration) of the workload
    for _ in range(args.warmup):
        R.cg(1, 0.0)
    times = []
    for _ in range(args.steps):
        r = R.cg(1, 0.0)
        times.append(r["seconds"])
    t = sum(times) / len(times)
    gflops = flops_it / t / 1e9
    cores = host_threads()
    sample = f"CG_ref (src/CG_ref.cpp) on the {nx}^3 problem: 1 iteration + preamble per step, OMP threads={cores}"
    line = {
        "metric": METRIC, "value": gflops, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (HPCG generator)", "impl": "reference",
        "config": {"workload": f"HPCG {nx}^3 FP64 MG-PCG (4 levels), generated b, x0=0", "grid": [nx, nx, nx],
                   "mg_levels": 4, "parallelism": "one CPU process (rank 0), OpenMP threads"},
        "cpu_baseline": {"value": gflops, "unit": "GFLOP/s", "cores": cores, "kind": "reference", "sample": sample,
                         **cpu_facts()},
        "e2e": {"value": gflops, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "setup_s": setup_s,
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------ rank plumbing
# One process per GPU; every rank solves its own local problem (replicas, no
# collective on the data path); the only collectives are the barriers around
# the timed region and the max of the timings.

def ranks() -> tuple[int, int, int]:
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_dist(world: int, local: int, backend: str, timeout_s: int = 600):
    """torch.distributed for world > 1 (nccl on the GPUs, gloo in the CPU
    tests), else None.  MASTER_ADDR / MASTER_PORT come from the launcher."""
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return dist


def max_over(dist, v: float, device: str) -> float:
    """max of v over all ranks (v itself without a process group)."""
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gflops(world: int, flops_per_iter: float, iters: int, seconds_per_step: float) -> float:
    """Whole-job GFLOP/s: every rank solves its own problem of the same size in
    the (max-over-ranks) step time."""
    return world * flops_per_iter * iters / seconds_per_step / 1e9


# ------------------------------------------------------------------ our arm

def attach_ref_residuals(obj, values: dict, errors: dict):
    """Replace every `ref_check_tag` in the result tree by the residual the
    reference-operator checker returned for it (`rel_residual_ref_spmv`)."""
    if isinstance(obj, dict):
        tag = obj.pop("ref_check_tag", None)
        if tag is not None:
            obj["rel_residual_ref_spmv"] = values.get(tag)
            if tag in errors:
                obj["ref_check_error"] = errors[tag]
        for v in obj.values():
            attach_ref_residuals(v, values, errors)


def run_ours(args):
    import torch
    import rochpcg_b200 as R

    world, rank, local = ranks()
    dist = init_dist(world, local, "nccl")
    if dist is None:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        return max_over(dist, v, "cuda")

    if args.mixed_only:
        return run_mixed_only(args, R, barrier)

    nx = args.nx
    grid = (nx, nx, nx)
    # host-side check of every solve with the reference's own SpMV (rank 0):
    # the worker builds the reference problem while the GPU works
    checker = None
    if rank == 0 and not args.lite and not args.no_refcheck:
        from oracle.residual_check import RefResidualChecker

        checker = RefResidualChecker(threads=max(1, host_threads() // 2))
        checker.prepare(grid)

    def refcheck(tag, grid_, rhs, x_natural):
        if checker is not None:
            checker.submit(tag, grid_, rhs, x_natural)
            return tag
        return None

    P = R.Problem(nx)
    flops_it, bytes_it = P.model()
    alg_bytes_it = fp64_algorithmic_bytes_per_iter(P.rows)
    m = P.rows[0]
    stream = torch.cuda.ExternalStream(P.stream_handle)

    # ---- device-timed solves (inputs resident in HBM)
    for _ in range(args.warmup):
        P.cg(args.max_iter, args.tol)
    barrier()
    sampler = ClockSampler(dev)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    runs = []
    for _ in range(args.steps):
        runs.append(P.cg(args.max_iter, args.tol))
    e1.record(stream)
    e1.synchronize()
    barrier()
    clocks = sampler.stop()
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    iters = runs[-1]["niters"]
    ms_step = ms_total / args.steps
    value = job_gflops(world, flops_it, iters, ms_step * 1e-3)
    rel = runs[-1]["normr"] / runs[-1]["normr0"]
    true_rel = P.true_residual()
    fp64_tag = refcheck("fp64_256", grid, ("generated",), P.get_x()) if checker else None
    kpi = P.kernels_per_iteration(R.MODE_FP64)
    # per solve: the preamble's SpMV and residual, the iterations, the last x update
    launches = args.steps * (iters * kpi + 3)

    if args.lite:
        if rank == 0:
            print(json.dumps({"lite": True, "metric": METRIC, "value": value, "unit": "GFLOP/s", "iterations": iters,
                              "ms_per_step": ms_step, "gpu_launches": launches}))
        P.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # ---- end to end through the C ABI from pinned host memory
    b_host = torch.from_numpy(generated_b_natural(nx, nx, nx)).pin_memory()
    x_host = torch.empty(m, dtype=torch.float64).pin_memory()
    P.solve_host(b_host, x_host, 1000, args.tol)  # warm
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        re = P.solve_host(b_host, x_host, 1000, args.tol)
    barrier()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    e2e_val = job_gflops(world, flops_it, re["niters"], e2e_s)
    x_err = float(torch.max(torch.abs(x_host - 1.0)))
    e2e_tag = refcheck("e2e_fp64_256", grid, ("generated",), x_host.numpy().copy())

    # ---- dominant kernel: level-0 full SymGS colour sweep
    nb = P.nblocks[0]
    sweep_ms = P.time_op("symgs_sweep", 20)
    rows_c = m // nb
    alg_bytes = rows_c * (27 * 12 + 3 * 8) + (m - rows_c) * 8
    achieved = alg_bytes / (sweep_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = profile_traffic(f"symgs_sweep_{nx}")
    roofline = {"kernel": "k_symgs_sweep (level-0 colour sweep, FP64 ELL)", "bound": "hbm", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes, "ms_per_launch": sweep_ms}
    spmv_ms = P.time_op("spmv", 20)
    spmv_bytes = m * (27 * 12 + 8 + 8)
    extra_kernels = {"spmv_GBps": spmv_bytes / (spmv_ms * 1e-3) / 1e9, "spmv_ms": spmv_ms,
                     "spmv_traffic": profile_traffic(f"spmv_{nx}"), "spmv_algorithmic_bytes_per_launch": spmv_bytes,
                     "mg_ms": P.time_op("mg", 5)}

    # ---- the same solve on the implicit stencil: FP64 history bit for bit, no matrix reads
    stencil = None
    if P.stencil_ok(0):
        P.cg(args.max_iter, args.tol, mode=R.MODE_FP64_STENCIL)
        barrier()
        s_runs = [P.cg(args.max_iter, args.tol, mode=R.MODE_FP64_STENCIL) for _ in range(args.steps)]
        s_min = min(r["seconds"] for r in s_runs)
        stencil = {"time_to_solution_s": s_min, "iterations": s_runs[-1]["niters"],
                   "gflops_hpcg_model": flops_it * s_runs[-1]["niters"] / s_min / 1e9,
                   "history_bitwise_equal_to_fp64": bool(np.array_equal(s_runs[-1]["hist"], runs[-1]["hist"])),
                   "speedup_vs_fp64_ell": ms_step * 1e-3 / s_min,
                   "rel_residual_fp64_true": P.true_residual(),
                   "ref_check_tag": refcheck("fp64_stencil_256", grid, ("generated",), P.get_x()),
                   "mg_ms": P.time_op("mg_stencil", 5)}
    P.close()
    del P

    # ---- mixed precision vs FP64 at 320^3, b ~ N(0,1) seed 0
    mixed = None
    if not args.no_mixed:
        mixed = mixed_comparison(args, R, barrier, refcheck=refcheck, checker=checker)

    # ---- learned coarse-level smoother vs SymGS at 256^3, b ~ N(0,1) seed 9999
    learned = None
    if not args.no_learned:
        learned = learned_comparison(args, R, barrier, refcheck=refcheck)

    # ---- the largest configuration, 560 x 560 x 280
    largest = None
    if not args.no_largest:
        if checker is not None:
            # free the smaller reference problems before the 87.8M-row one
            checker.drop(grid)
            checker.drop((args.mixed_nx,) * 3)
            checker.drop((args.learned_nx,) * 3)
        largest = largest_comparison(args, R, barrier, refcheck=refcheck, checker=checker)

    ref_values, ref_errors = {}, {}
    if checker is not None:
        ref_values = checker.results()
        ref_errors = dict(checker.errors)
        checker.close()

    # ---- the decomposed path on this GPU: 8 ranks of 64^3 (global 128^3)
    # driven from this process (device-copy exchange), checked against the
    # exact solution; a correctness record, not a multi-GPU measurement
    decomposed = None
    if rank == 0 and world == 1:
        decomposed = decomposed_check()

    # ---- CPU baseline: the reference's CG_ref on host cores (rank 0, N=1),
    # after the checker has exited so that nothing else uses the host cores
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args)

    if rank == 0:
        peak_gbs = measured_peak()[0]
        alg_gbps = world * alg_bytes_it * iters / (ms_step * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (HPCG problem generator, b for x*=1)",
            "config": {"workload": f"HPCG {nx}^3 FP64 MG-PCG solve to rel. residual {args.tol:g}",
                       "grid": [nx, nx, nx], "mg_levels": 4, "rhs": "generated (exact solution ones), x0=0",
                       "l2": "inputs larger than L2 (level-0 ELL is %.1f GB)" % (27 * 12 * m / 1e9),
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "time_to_solution_s": ms_step * 1e-3, "iterations": iters, "rel_residual": rel,
            "rel_residual_fp64_true": true_rel, "ref_check_tag": fp64_tag,
            # this implementation's bytes per iteration (per-kernel algorithmic
            # bytes) and the bandwidth they imply
            "algorithmic_bytes_per_iter": alg_bytes_it,
            "algorithmic_GBps": alg_gbps, "algorithmic_frac_of_hbm": alg_gbps / world / peak_gbs,
            # the reference's traffic model (src/ReportResults.cpp:163-195):
            # charges two matrix passes to the zero-guess smoother and nnz*8
            # bytes of writes to the residual and post-smoother, so it is an
            # accounting figure, not a bandwidth
            "hpcg_traffic_model_bytes_per_iter": bytes_it,
            "hpcg_traffic_model_GBps_not_a_bandwidth": world * bytes_it * iters / (ms_step * 1e-3) / 1e9,
            "e2e": {"value": e2e_val, "unit": "GFLOP/s", "h2d_bytes_per_step": 8 * m, "d2h_bytes_per_step": 8 * m,
                    "seconds_per_step": e2e_s, "max_abs_x_minus_1": x_err, "ref_check_tag": e2e_tag},
            "roofline": roofline, "kernels": extra_kernels, "fp64_stencil": stencil, "cpu_baseline": cpu,
            "mixed": mixed,
            "learned": learned, "largest": largest,
            "gpu_launches": launches, "clocks": clocks, "decomposed_check": decomposed,
        }
        attach_ref_residuals(line, ref_values, ref_errors)
        line["ref_spmv_check"] = ("every solve's final x checked on the host with the reference's ComputeSPMV_ref "
                                  "(oracle/_ref, natural order): rel_residual_ref_spmv = ||b - A x|| / ||b||"
                                  if checker is not None else "skipped")
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def mixed_comparison(args, R, barrier, steps=2, warmup=1, refcheck=None, checker=None):
    """Mixed precision (320^3 by default): FP64-outer / FP32 V-cycle vs plain
    FP64 on the same n^3 system with b ~ N(0,1) (seed 0), both to args.tol,
    both verified with an FP64 true residual."""
    from rochpcg_b200.rhs import normal_rhs

    n3 = args.mixed_nx
    if checker is not None:
        checker.prepare((n3, n3, n3))
    Q = R.Problem(n3)
    Q.set_rhs(normal_rhs(Q.rows[0], 0))
    f3, _ = Q.model()
    from rochpcg_b200 import learned as LS

    res = {}
    hists = {}
    S = LS.Smoother.load()
    for name, mode in (("fp64", R.MODE_FP64), ("fp64_stencil", R.MODE_FP64_STENCIL), ("mixed", R.MODE_MIXED),
                       ("learned", R.MODE_LEARNED)):
        if mode == R.MODE_LEARNED:
            Q.set_smoother(S, 2)
        for _ in range(warmup):
            Q.cg(args.max_iter, args.tol, mode=mode)
        barrier()
        ts = []
        for _ in range(steps):
            r3 = Q.cg(args.max_iter, args.tol, mode=mode)
            ts.append(r3["seconds"])
        hists[name] = r3["hist"]
        res[name] = {"time_to_1e-9_s": min(ts), "iterations": r3["niters"],
                     "rel_residual_recurrence": r3["normr"] / r3["normr0"],
                     "rel_residual_fp64_true": Q.true_residual(),
                     "gflops_hpcg_model": f3 * r3["niters"] / min(ts) / 1e9,
                     "kernels_per_iteration": Q.kernels_per_iteration(mode)}
        if refcheck is not None:
            res[name]["ref_check_tag"] = refcheck(f"mixed{n3}_{name}", (n3, n3, n3), ("normal", 0), Q.get_x())
        if mode == R.MODE_LEARNED:
            res[name]["fallback_iteration"] = Q.last_fallback()
            Q.set_smoother(None)
    res["speedup_mixed_vs_fp64"] = res["fp64"]["time_to_1e-9_s"] / res["mixed"]["time_to_1e-9_s"]
    # the mixed + learned solver against plain FP64 at this size (target >= 2x)
    res["speedup_learned_vs_fp64"] = res["fp64"]["time_to_1e-9_s"] / res["learned"]["time_to_1e-9_s"]
    # FP64 on the implicit stencil: the FP64 residual history bit for bit, no matrix reads
    res["speedup_fp64_stencil_vs_fp64"] = res["fp64"]["time_to_1e-9_s"] / res["fp64_stencil"]["time_to_1e-9_s"]
    res["fp64_stencil_history_bitwise_equal"] = bool(len(hists["fp64"]) == len(hists["fp64_stencil"]) and
                                                     (hists["fp64"] == hists["fp64_stencil"]).all())
    # level-0 kernels of the mixed path, timed alone (CUDA events)
    m3 = Q.rows[0]
    rows_c = m3 // 8
    sw = Q.time_op("symgs32_sweep", 10)
    sw_bytes = rows_c * (4 + 4 + 4) + (m3 - rows_c) * 4
    sp = Q.time_op("spmv_stencil", 10)
    sp_bytes = m3 * (8 + 8 + 8)
    spm = Q.time_op("spmv_mixed", 10)
    res["kernels"] = {"k32_sweep_ms": sw, "k32_sweep_GBps": sw_bytes / (sw * 1e-3) / 1e9,
                      "k32_sweep_algorithmic_bytes": sw_bytes,
                      # the mixed CG's outer operator (separable sum)
                      "k64_spmv_sep_ms": spm, "k64_spmv_sep_GBps": sp_bytes / (spm * 1e-3) / 1e9,
                      # the ELL-ordered stencil product of the FP64 stencil mode
                      "k64_spmv_stencil_ms": sp, "k64_spmv_stencil_GBps": sp_bytes / (sp * 1e-3) / 1e9,
                      "mg_mixed_ms": Q.time_op("mg_mixed", 5), "mg_fp64_ms": Q.time_op("mg", 3),
                      "mg_fp64_stencil_ms": Q.time_op("mg_stencil", 5)}
    res["grid"] = [n3, n3, n3]
    res["rhs"] = "N(0,1) i.i.d., seed 0 (SplitMix64 + Box-Muller, natural row order)"
    Q.close()
    return res


def conv_kernel_timing(nb, n, reps=50):
    """Layer-2 convolution (16 -> 16 channels, tcgen05) on nb samples of n^3
    points, timed with CUDA events on torch's stream."""
    import ctypes

    import torch

    L = R_load()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    g = torch.Generator(device="cuda").manual_seed(1)
    w = torch.randn(27 * 256, device="cuda", generator=g) * 0.1
    wB = torch.empty(L.hpcgb200_conv_weight_tile_bytes(), dtype=torch.uint8, device="cuda")
    L.hpcgb200_conv_prepare_weights(vp(w), vp(wB), 0, st)
    pts = nb * n ** 3
    x = (torch.randn(pts * 16, device="cuda", generator=g)).to(torch.bfloat16)
    out = torch.empty_like(x)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(3):
        L.hpcgb200_conv16(nb, n, n, n, vp(x), vp(wB), 0, vp(out), None, vp(status), st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        L.hpcgb200_conv16(nb, n, n, n, vp(x), vp(wB), 0, vp(out), None, vp(status), st)
    e1.record()
    torch.cuda.synchronize()
    us = e0.elapsed_time(e1) * 1e3 / reps
    flops = pts * 27 * 16 * 16 * 2
    return {"points": pts, "us_per_launch": us, "tflops": flops / us * 1e-6, "status": int(status.item())}


def R_load():
    import rochpcg_b200 as R

    return R.load()


def learned_comparison(args, R, barrier, steps=2, refcheck=None):
    """Learned smoother (256^3 by default): levels 2-3 SymGS replaced by the trained conv net (committed
    weights), flexible CG with fallback, vs the plain FP32 V-cycle and FP64, on
    an n^3 system with b ~ N(0,1) (seed 9999), all to args.tol."""
    from rochpcg_b200 import learned as LS
    from rochpcg_b200.rhs import normal_rhs

    n = args.learned_nx
    Q = R.Problem(n)
    Q.set_rhs(normal_rhs(Q.rows[0], 9999))
    f, _ = Q.model()
    S = LS.Smoother.load()
    res = {}
    for name, mode in (("fp64", R.MODE_FP64), ("mixed", R.MODE_MIXED), ("learned", R.MODE_LEARNED)):
        if mode == R.MODE_LEARNED:
            Q.set_smoother(S, 2)
        Q.cg(args.max_iter, args.tol, mode=mode)  # warm-up
        barrier()
        ts = []
        for _ in range(steps):
            r = Q.cg(args.max_iter, args.tol, mode=mode)
            ts.append(r["seconds"])
        res[name] = {"time_to_1e-9_s": min(ts), "iterations": r["niters"],
                     "rel_residual_fp64_true": Q.true_residual(),
                     "gflops_hpcg_model": f * r["niters"] / min(ts) / 1e9,
                     "kernels_per_iteration": Q.kernels_per_iteration(mode)}
        if refcheck is not None:
            res[name]["ref_check_tag"] = refcheck(f"learned{n}_{name}", (n, n, n), ("normal", 9999), Q.get_x())
        if mode == R.MODE_LEARNED:
            res[name]["fallback_iteration"] = Q.last_fallback()
            res[name]["vcycle_ms_graph"] = Q.time_op("graph:mg_learned", 20)  # as the solver runs it
        elif mode == R.MODE_MIXED:
            res[name]["vcycle_ms_graph"] = Q.time_op("graph:mg_mixed", 20)
    res["speedup_learned_vs_fp64"] = res["fp64"]["time_to_1e-9_s"] / res["learned"]["time_to_1e-9_s"]
    res["speedup_learned_vs_mixed"] = res["mixed"]["time_to_1e-9_s"] / res["learned"]["time_to_1e-9_s"]
    # the literal rule: fall back at the first iteration that does not reduce the FP64 residual norm
    Q.set_fallback_rule("first-increase")
    Q.cg(args.max_iter, args.tol, mode=R.MODE_LEARNED)
    r = Q.cg(args.max_iter, args.tol, mode=R.MODE_LEARNED)
    res["learned_first_increase_fallback"] = {"time_to_1e-9_s": r["seconds"], "iterations": r["niters"],
                                              "fallback_iteration": Q.last_fallback(),
                                              "rel_residual_fp64_true": Q.true_residual()}
    if refcheck is not None:
        res["learned_first_increase_fallback"]["ref_check_tag"] = refcheck(
            f"learned{n}_first_increase", (n, n, n), ("normal", 9999), Q.get_x())
    Q.set_fallback_rule("default")
    Q.set_smoother(None)
    Q.close()
    meta = S.meta
    conv = conv_kernel_timing(2, n >> 2)  # level 2, both branches of the odd evaluation
    peak = measured_bf16_peak()
    label = "k_conv16 (layer 2, 16->16, tcgen05 M128 K16, dz and dx taps stacked in N<=144, one TMA box per brick)"
    res["conv_kernel"] = dict(conv, kernel=label, bound="tensor", peak_tflops=peak,
                              frac=conv["tflops"] / peak if peak else None)
    res["weights"] = {"file": "rochpcg_b200/weights/smoother_l23.npz", "sha256": meta.get("sha256"),
                      "symmetry": meta.get("symmetry"), "heldout": meta.get("heldout"),
                      "training": {k: meta.get("training", {}).get(k) for k in ("epochs", "loss", "lr0", "lr1")}}
    res["grid"] = [n, n, n]
    res["rhs"] = "N(0,1) i.i.d., seed 9999"
    return res


def largest_comparison(args, R, barrier, refcheck=None, checker=None):
    """Largest workload: 560 x 560 x 280 (87.8M rows), FP64 outer CG with the FP32
    V-cycle and the learned level-2/3 smoother, against plain mixed and FP64,
    for b ~ N(0,1) seed 7 and for the generated b (exact solution ones), all to
    args.tol verified in FP64; fine-level bandwidth from the HPCG byte model
    with the mixed path's element sizes."""
    from rochpcg_b200 import learned as LS
    from rochpcg_b200.rhs import normal_rhs

    grid = (560, 560, 280)
    if checker is not None:
        checker.prepare(grid)
    Q = R.Problem(*grid)
    f, bytes64 = Q.model()
    alg64 = fp64_algorithmic_bytes_per_iter(Q.rows)
    m = Q.rows[0]
    S = LS.Smoother.load()
    out = {"grid": [560, 560, 280], "rows": m}
    for rhs in ("seed7", "ones"):
        Q.set_rhs(normal_rhs(m, 7) if rhs == "seed7" else None)
        res = {}
        for name, mode in (("fp64", R.MODE_FP64), ("mixed", R.MODE_MIXED), ("learned", R.MODE_LEARNED)):
            if mode == R.MODE_LEARNED:
                Q.set_smoother(S, 2)
            Q.cg(args.max_iter, args.tol, mode=mode)  # warm-up
            barrier()
            r = Q.cg(args.max_iter, args.tol, mode=mode)
            res[name] = {"time_to_1e-9_s": r["seconds"], "iterations": r["niters"],
                         "rel_residual_fp64_true": Q.true_residual(),
                         "gflops_hpcg_model": f * r["niters"] / r["seconds"] / 1e9}
            if refcheck is not None:
                res[name]["ref_check_tag"] = refcheck(f"largest_{rhs}_{name}", grid,
                                                      ("normal", 7) if rhs == "seed7" else ("generated",), Q.get_x())
            if mode == R.MODE_FP64:
                res[name]["algorithmic_GBps"] = alg64 * r["niters"] / r["seconds"] / 1e9
                res[name]["hpcg_traffic_model_GBps_not_a_bandwidth"] = bytes64 * r["niters"] / r["seconds"] / 1e9
            if mode == R.MODE_LEARNED:
                res[name]["fallback_iteration"] = Q.last_fallback()
                Q.set_smoother(None)
        res["speedup_learned_vs_fp64"] = res["fp64"]["time_to_1e-9_s"] / res["learned"]["time_to_1e-9_s"]
        res["speedup_mixed_vs_fp64"] = res["fp64"]["time_to_1e-9_s"] / res["mixed"]["time_to_1e-9_s"]
        out[rhs] = res
    # fine-level FP32 sweep of the mixed path, timed alone
    rows_c = m // 8
    sw = Q.time_op("symgs32_sweep", 10)
    out["fine_level_k32_sweep"] = {"ms": sw, "GBps": (rows_c * 12 + (m - rows_c) * 4) / (sw * 1e-3) / 1e9}
    sw64 = Q.time_op("symgs_sweep", 10)
    out["fine_level_k_symgs_sweep_fp64"] = {"ms": sw64, "GBps": (rows_c * (27 * 12 + 3 * 8) + (m - rows_c) * 8)
                                            / (sw64 * 1e-3) / 1e9}
    Q.close()
    return out


def measured_bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        for k in ("bf16_tflops", "bf16_dense_tflops"):
            if k in d:
                return float(d[k])
    except Exception:
        pass
    return 1590.0


def run_mixed_only(args, R, barrier):
    res = mixed_comparison(args, R, barrier, steps=args.steps, warmup=args.warmup)
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps({"mixed_only": True, "metric": METRIC, "mixed": res}))
    return 0


def run_profile_case(case: str) -> int:
    """Small fixed workloads for ncu captures (see profiles/)."""
    import torch

    import rochpcg_b200 as R

    torch.cuda.set_device(0)
    if case == "conv":
        # layer-2 convolution at MG level 2 of 256^3 (64^3 points, both odd branches)
        print(json.dumps(conv_kernel_timing(2, 64, reps=2)))
    elif case == "sweep128":
        P = R.Problem(128)
        print(json.dumps({"symgs_sweep_ms": P.time_op("symgs_sweep", 2)}))
    elif case == "spmv128":
        # the FP64 ELL SpMV at 128^3 (2.1M rows, 680 MB of ELL)
        P = R.Problem(128)
        print(json.dumps({"spmv_ms": P.time_op("spmv", 2)}))
    elif case in ("cg128", "cgmixed192"):
        # two CG iterations (FP64 ELL at 128^3, or mixed at 192^3); run with HPCGB200_GRAPH=0 so that a
        # profiler sees the kernels as launches
        P = R.Problem(128 if case == "cg128" else 192)
        r = P.cg(2, 0.0, mode=R.MODE_FP64 if case == "cg128" else R.MODE_MIXED)
        print(json.dumps({"niters": r["niters"], "normr": r["normr"]}))
    elif case in ("mixed128", "mixed192"):
        # the mixed path's level-0 kernels: separable outer SpMV, FP32 colour sweeps
        P = R.Problem(128 if case == "mixed128" else 192)
        print(json.dumps({"spmv_mixed_ms": P.time_op("spmv_mixed", 2), "symgs32_sweep_ms": P.time_op("symgs32_sweep", 1)}))
    elif case == "net64":
        # the learned smoother's evaluation on one 64^3 sample, both odd branches
        # (layer 1 and layer 3 in their one-channel tensor-core forms)
        from rochpcg_b200 import learned as LS

        S = LS.Smoother.load()
        g = torch.Generator(device="cuda").manual_seed(3)
        r = torch.randn(64 ** 3, device="cuda", generator=g)
        for _ in range(3):
            y = S.forward(r, (64, 64, 64), 1)
        torch.cuda.synchronize()
        print(json.dumps({"net64_norm": float(y.norm())}))
    elif case == "stencil192":
        # the FP64 stencil V-cycle at 192^3 (eager launches; its level-0 passes are the TMA-staged double kernels)
        P = R.Problem(192)
        print(json.dumps({"mg_stencil_ms": P.time_op("mg_stencil", 1)}))
    elif case == "mixed320":
        # one mixed V-cycle + one stencil SpMV at 320^3 (eager launches)
        P = R.Problem(320)
        print(json.dumps({"mg_mixed_ms": P.time_op("mg_mixed", 1), "spmv_stencil_ms": P.time_op("spmv_stencil", 1)}))
    else:
        from rochpcg_b200 import learned as LS

        P = R.Problem(256)
        P.set_smoother(LS.Smoother.load(), 2)
        print(json.dumps({"mg_learned_ms": P.time_op("mg_learned", 2), "mg_mixed_ms": P.time_op("mg_mixed", 2)}))
    return 0


# ------------------------------------------------------------ decomposed solve

def decomposed_check(nranks: int = 8, n: int = 64) -> dict:
    """The decomposed solve with every rank in this process on one GPU: the
    global 2n x 2n x 2n problem's generated b, x = 1 expected."""
    from rochpcg_b200 import dist as D

    R = [D.DistProblem(n, n, n, nranks, r) for r in range(nranks)]
    try:
        D.group_cg(R, 500, 1e-9)  # captures the steady-iteration graph
        r = D.group_cg(R, 500, 1e-9)
        err = max(float(np.max(np.abs(P.get_x() - 1.0))) for P in R)
        g = R[0].grid
        return {"ranks": nranks, "local_grid": [n, n, n], "process_grid": list(g),
                "global_grid": [g[0] * n, g[1] * n, g[2] * n], "iterations": r["niters"],
                "rel_residual": r["normr"] / r["normr0"], "max_abs_x_minus_1": err, "seconds": r["seconds"],
                "exchange": "device copies between the ranks' buffers (one GPU)"}
    finally:
        for P in R:
            P.close()

def dist_launches_per_iter(P) -> int:
    """Our kernels per CG iteration of one rank of the decomposed solve (NCCL's
    own kernels not counted): per MG level the zero-guess colours, pack +
    interior + halo of the restriction, the prolongation, pack + colour 0 +
    halo + the other sweeps; CG: 2 dots, p update, pack + SpMV + halo, x/r update."""
    n = 0
    L = P.levels
    for l, lv in enumerate(L):
        nb = lv["nblocks"]
        n += 2 * nb - 1
        if l + 1 < len(L):
            n += 3 + 1 + (3 + (nb - 1) + (nb - 1))
    return n + 2 + 1 + 3 + 1


def dist_model(nx: int, grid, nlevels: int = 4):
    """HPCG flop model of the GLOBAL problem (src/ReportResults.cpp:134-195 with
    the global row and nonzero counts)."""
    from rochpcg_b200 import hpcg_model

    dims = [(grid[0] * (nx >> l), grid[1] * (nx >> l), grid[2] * (nx >> l)) for l in range(nlevels)]
    return hpcg_model(dims, [stencil_nnz(d) for d in dims]), dims


def run_dist(args, world: int, rank: int, local: int, emulate: int = 0):
    """The decomposed FP64 MG-PCG: every rank one nx^3 brick of the global grid
    (HPCG's weak scaling), halos over NCCL (or, emulated, device copies)."""
    import torch
    from rochpcg_b200 import dist as D

    os.environ.setdefault("HPCGB200_DIST_TIMEOUT_S", "180")
    nranks = emulate or world
    pg = init_dist(world, local, "nccl") if not emulate else None
    if pg is None:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    nx = args.nx
    grid = D.shape(nranks)

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    if emulate:
        ranks = [D.DistProblem(nx, nx, nx, nranks, r) for r in range(nranks)]
        solve = lambda: D.group_cg(ranks, args.max_iter, args.tol)  # noqa: E731
        mine = ranks[0]
    else:
        mine = D.DistProblem(nx, nx, nx, world, rank)
        barrier()
        D.attach_nccl(mine, pg)
        ranks = [mine]
        solve = lambda: mine.cg(args.max_iter, args.tol)  # noqa: E731
    (flops_it, _), gdims = dist_model(nx, grid)
    for _ in range(args.warmup):
        solve()
    barrier()
    sampler = ClockSampler(dev)
    sampler.start()
    runs = [solve() for _ in range(args.steps)]
    barrier()
    clocks = sampler.stop()
    sec = max_over(pg, sum(r["seconds"] for r in runs) / args.steps, "cuda")
    iters = runs[-1]["niters"]
    value = flops_it * iters / sec / 1e9
    rel = runs[-1]["normr"] / runs[-1]["normr0"]
    xerr = max(float(np.max(np.abs(P.get_x() - 1.0))) for P in ranks)
    xerr = max_over(pg, xerr, "cuda")
    # end to end through the rank API: b from host memory, x back to host memory
    m = mine.levels[0]["m"]
    nat_b = [P.field("b")[P.field("perm")] for P in ranks]
    x_host = np.empty(m)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for P, b in zip(ranks, nat_b):
            P.set_rhs(b)
        re = solve()
        for P in ranks:
            x_host = P.get_x()
    barrier()
    e2e_s = max_over(pg, (time.perf_counter() - t0) / args.steps, "cuda")
    launches = args.steps * nranks * (iters * dist_launches_per_iter(mine) + 6)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (HPCG problem generator, b for x*=1)",
            "config": {"workload": f"HPCG domain decomposition, {nranks} ranks of {nx}^3 (global "
                                   f"{gdims[0][0]}x{gdims[0][1]}x{gdims[0][2]}), FP64 MG-PCG to {args.tol:g}",
                       "grid": list(gdims[0]), "local_grid": [nx, nx, nx], "process_grid": list(grid),
                       "mg_levels": 4, "rhs": "generated (exact solution ones), x0=0",
                       "l2": "inputs larger than L2 (level-0 ELL of one rank is %.1f GB)" % (27 * 12 * m / 1e9),
                       "parallelism": (f"emulated {nranks} ranks on 1 GPU (device-copy exchange)" if emulate else
                                       f"domain decomposition {grid[0]}x{grid[1]}x{grid[2]}, halo exchange and "
                                       f"dot allreduce over NCCL")},
            "decomposed": True, "emulated": bool(emulate),
            "time_to_solution_s": sec, "iterations": iters, "rel_residual": rel, "max_abs_x_minus_1": xerr,
            "e2e": {"value": flops_it * re["niters"] / e2e_s / 1e9, "unit": "GFLOP/s",
                    "h2d_bytes_per_step": 8 * m, "d2h_bytes_per_step": 8 * m, "seconds_per_step": e2e_s},
            "roofline": None, "roofline_note": "per-kernel roofline is reported by the 1-GPU run",
            "cpu_baseline": None, "gpu_launches": launches, "clocks": clocks,
        }
        print(json.dumps(line))
    for P in ranks:
        P.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.profile_case:
        return run_profile_case(args.profile_case)
    if args.impl == "reference":
        return run_reference(args)
    world, rank, local = ranks()
    if args.emulate_ranks > 1 and world == 1:
        return run_dist(args, 1, 0, 0, emulate=args.emulate_ranks)
    if world > 1 and not args.replicas:
        return run_dist(args, world, rank, local)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
