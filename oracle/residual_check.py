"""Final-residual check with the reference's own CPU operator.  TEST AND
MEASUREMENT INFRASTRUCTURE ONLY (used by bench.py and tests as the checker,
never by the product).

A worker process (started with ``spawn``, so it never inherits a CUDA
context) holds the reference's generated problem for a grid --
``GenerateProblem_ref`` + ``SetupHalo_ref`` (src/GenerateProblem_ref.cpp,
src/SetupHalo_ref.cpp), level 0, natural row order -- and, for a solution x
handed over in natural order, returns ||b - A x||_2 / ||b||_2 with A x from
``ComputeSPMV_ref`` (src/ComputeSPMV_ref.cpp:48-75) and b either the
reference's own generated b (src/GenerateProblem_ref.cpp:178-180, exact
solution all ones) or the seeded N(0,1) right-hand side of
``rochpcg_b200.rhs.normal_rhs`` (pure numpy, regenerated here).

The worker runs beside the GPU work: building the reference problem takes
seconds to a minute of host time per grid, which overlaps the device solves.
Solutions go through files in a temporary directory (a pipe would block the
caller while the worker is busy building).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import shutil
import tempfile

import numpy as np


def _worker(conn, threads: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(threads)  # before the reference library loads libgomp
    from oracle.oracle import RefProblem
    from rochpcg_b200.rhs import normal_rhs

    probs: dict = {}

    def get(grid):
        if grid not in probs:
            probs[grid] = RefProblem(*grid, nlevels=1)
        return probs[grid]

    while True:
        msg = conn.recv()
        kind = msg[0]
        if kind == "stop":
            break
        try:
            if kind == "prepare":
                get(msg[1])
            elif kind == "drop":
                probs.pop(msg[1], None)
            elif kind == "check":
                _, tag, grid, rhs, path = msg
                P = get(grid)
                x = np.load(path)
                os.remove(path)
                y = P.spmv(0, x)
                if rhs[0] == "generated":
                    b = P.rhs()[0]
                else:
                    b = normal_rhs(P.nrows[0], int(rhs[1]))
                r = b - y
                conn.send((tag, float(np.linalg.norm(r) / np.linalg.norm(b)), None))
        except Exception as e:  # reported per check, the worker keeps serving
            if kind == "check":
                conn.send((msg[1], None, f"{type(e).__name__}: {e}"))


class RefResidualChecker:
    """Asynchronous checker: ``prepare(grid)`` starts building a grid's
    reference problem, ``submit(tag, grid, rhs, x_natural)`` queues a check,
    ``results()`` waits for every queued check and returns {tag: value}
    (None with an ``errors`` entry when a check failed)."""

    def __init__(self, threads: int = 8):
        ctx = mp.get_context("spawn")
        self.conn, child = ctx.Pipe()
        self.proc = ctx.Process(target=_worker, args=(child, threads), daemon=True)
        self.proc.start()
        self.tmp = tempfile.mkdtemp(prefix="hpcg_refcheck_")
        self.pending = []
        self.values: dict = {}
        self.errors: dict = {}

    def _send(self, msg) -> bool:
        try:
            self.conn.send(msg)
            return True
        except (BrokenPipeError, OSError):  # the worker exited (e.g. out of host memory)
            return False

    def prepare(self, grid) -> None:
        self._send(("prepare", tuple(grid)))

    def drop(self, grid) -> None:
        self._send(("drop", tuple(grid)))

    def submit(self, tag: str, grid, rhs, x_natural: np.ndarray) -> None:
        """rhs: ("generated",) or ("normal", seed)."""
        if not self.proc.is_alive():
            self.values[tag] = None
            self.errors[tag] = f"checker exited (exit code {self.proc.exitcode})"
            return
        path = os.path.join(self.tmp, f"x{len(self.pending) + len(self.values)}.npy")
        np.save(path, np.ascontiguousarray(x_natural, np.float64))
        if self._send(("check", tag, tuple(grid), tuple(rhs), path)):
            self.pending.append(tag)
        else:
            self.values[tag] = None
            self.errors[tag] = f"checker exited (exit code {self.proc.exitcode})"

    def results(self, timeout_s: float = 900.0) -> dict:
        for _ in range(len(self.pending)):
            try:
                ready = self.conn.poll(timeout_s)
                got = self.conn.recv() if ready else None
            except (EOFError, OSError):
                got = None
            if got is None:
                why = "timed out" if self.proc.is_alive() else f"checker exited (exit code {self.proc.exitcode})"
                for t in self.pending:
                    self.values.setdefault(t, None)
                    self.errors.setdefault(t, why)
                self.pending = []
                break
            tag, val, err = got
            self.values[tag] = val
            if err:
                self.errors[tag] = err
            self.pending.remove(tag)
        return dict(self.values)

    def close(self) -> None:
        try:
            self.conn.send(("stop",))
        except (BrokenPipeError, OSError):
            pass
        self.proc.join(timeout=30)
        if self.proc.is_alive():
            self.proc.kill()
        shutil.rmtree(self.tmp, ignore_errors=True)
