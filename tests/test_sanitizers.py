"""Host index code under AddressSanitizer and UndefinedBehaviorSanitizer.

compute-sanitizer is not available for the device code on the machines these
tests target, so bounds and races there are pinned by the bit-exact index and
operator comparisons against the CPU restatements (tests/test_gpu_*.py) and by
compile-time checks of the TMA tile plans.  The host code that builds those
index arrays, and the restatements themselves, are checked here: the halo
plan of rochpcg_b200/host/halo_plan.cpp for 1 to 27 ranks and every level
(tests/sanitize/halo_plan_check.cpp, which also checks that every send list
is its partner's receive list), and the multi-rank restatements of the
optimized and reference paths (tests/sanitize/oracle_check.c).  Each driver
is compiled with -fsanitize=address,undefined and must run clean.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer", "-g", "-O1"]


def _need(compiler):
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")


def _run(exe):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "ERROR: AddressSanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-4000:]
    return r.stdout


def test_halo_plan_under_sanitizers(tmp_path):
    _need("g++")
    exe = str(tmp_path / "halo_plan_check")
    subprocess.run(["g++", "-std=c++17", *SAN, "-I", os.path.join(ROOT, "rochpcg_b200", "host"),
                    os.path.join(ROOT, "tests", "sanitize", "halo_plan_check.cpp"),
                    os.path.join(ROOT, "rochpcg_b200", "host", "halo_plan.cpp"), "-o", exe],
                   check=True, timeout=300)
    assert "all checks hold" in _run(exe)


def test_oracle_restatements_under_sanitizers(tmp_path):
    _need("gcc")
    exe = str(tmp_path / "oracle_check")
    o = os.path.join(ROOT, "oracle")
    subprocess.run(["gcc", "-std=c11", *SAN, "-ffp-contract=off", "-fopenmp", "-I", o,
                    os.path.join(ROOT, "tests", "sanitize", "oracle_check.c"), os.path.join(o, "colored.c"),
                    os.path.join(o, "distributed.c"), os.path.join(o, "distributed_ref.c"), "-lm", "-o", exe],
                   check=True, timeout=300)
    assert "all runs clean" in _run(exe)
