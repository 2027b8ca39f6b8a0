"""The N > 1 path of bench.py on the CPU: two gloo ranks take the timing
collectives the GPU ranks take (barrier, max over ranks) and aggregate the
whole-job value the way the bench does for replicas; the reference arm runs on
rank 0 only."""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, _ = bench.ranks()
    d = bench.init_dist(w, r, "gloo", timeout_s=60)
    try:
        d.barrier()
        step_s = 0.5 + r          # a slower rank sets the job's step time
        t = bench.max_over(d, step_s, "cpu")
        v = bench.job_gflops(w, 6.2241e9, 129, t)
        d.barrier()
        q.put((r, t, v))
    finally:
        d.destroy_process_group()


def test_two_gloo_ranks_time_as_max_and_aggregate_replicas():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    out = sorted(q.get(timeout=5) for _ in range(world))
    want_t = 0.5 + (world - 1)
    want_v = world * 6.2241e9 * 129 / want_t / 1e9
    for r, t, v in out:
        assert t == want_t
        assert v == pytest.approx(want_v, rel=1e-15)


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.init_dist(1, 0, "gloo") is None
    assert bench.max_over(None, 3.25, "cpu") == 3.25


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", HPCG_BENCH_REF_SAMPLE="16",
               OMP_NUM_THREADS="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--gpus", "2"], capture_output=True, text=True, env=env, timeout=300,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    env["RANK"] = "0"
    env["LOCAL_RANK"] = "0"
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--gpus", "2"], capture_output=True, text=True, env=env, timeout=300,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference"


def test_decomposed_bench_model_and_launch_count():
    """bench.py's decomposed line: the HPCG flop model of the GLOBAL grid, and
    the kernels one rank launches per CG iteration."""
    sys.path.insert(0, ROOT)
    import bench
    from rochpcg_b200 import hpcg_model

    (f, _), dims = bench.dist_model(256, (2, 2, 1))
    assert dims[0] == (512, 512, 256) and dims[3] == (64, 64, 32)
    want, _ = hpcg_model(dims, [bench.stencil_nnz(d) for d in dims])
    assert f == want

    class FakeRank:
        levels = [{"nblocks": 8}] * 4
    # 3 levels with restriction/prolongation: (15) + 3 + 1 + (3 + 7 + 7); coarsest (15); CG 7
    assert bench.dist_launches_per_iter(FakeRank()) == 3 * (15 + 4 + 17) + 15 + 7
