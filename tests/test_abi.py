"""The C ABI boundary on CPU: the library loads, exports exactly what
include/hpcg_b200.h declares, validates arguments, and -- without a device --
reports an error instead of falling back to any CPU path."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import rochpcg_b200 as R
from rochpcg_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hpcg_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(hpcgb200_[a-z0-9_]+)\s*\(", text)))


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", R.LIB_PATH], capture_output=True, text=True, check=True)
    return sorted({ln.split()[-1] for ln in out.stdout.splitlines() if ln.split()[-1].startswith("hpcgb200_")})


def test_library_present_and_loads():
    assert os.path.exists(R.LIB_PATH), "libhpcgb200.so must be built in-tree"
    L = R.load()
    assert L.hpcgb200_version().startswith(b"hpcg-b200")


def test_every_declared_symbol_is_exported():
    d, e = declared_symbols(), exported_symbols()
    assert len(d) >= 40
    missing = [s for s in d if s not in e]
    assert not missing, missing
    extra = [s for s in e if s not in d]
    assert not extra, extra


def test_python_signatures_cover_header():
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_glibc_rand_sequence_matches_libc():
    L = R.load()
    out = np.zeros(64, np.int32)
    assert L.hpcgb200_rand_sequence(0x586744, 64, out.ctypes.data_as(ctypes.c_void_p)) == 0
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(0x586744)
    ref = [libc.rand() for _ in range(64)]
    assert out.tolist() == ref
    # the colour pairs of the first four JPL rounds (src/MultiColoring.cpp:283-284)
    assert [v % 8 for v in ref[:8]] == [0, 7, 1, 2, 4, 3, 5, 6]


def test_argument_validation_without_device():
    L = R.load()
    assert L.hpcgb200_spmv(0, None, None, None, None, None) == 1
    assert b"bad arguments" in L.hpcgb200_last_error()
    assert L.hpcgb200_dot(10, None, None, None, None, 0, None) == 1
    assert L.hpcgb200_f2c_operator(3, 4, 4, None, None, None) == 1  # odd fine dimension
    ws = L.hpcgb200_reduction_workspace_bytes()
    assert ws >= 1184 * 16
    # reference routines, protocol and learned-solve entry points reject bad input before any device work
    assert L.hpcgb200_ref_spmv(0, 4, 4, None, None, None, None, None, None) == 1
    assert L.hpcgb200_ref_symgs(4, 4, 4, None, None, None, None, None, None, None) == 1
    assert L.hpcgb200_problem_cg_ref(None, 50, 0.0, 1, None, None, None, None) == 1
    assert L.hpcgb200_problem_mg_ref(None, None, None) == 1
    assert L.hpcgb200_benchmark_run(None, None) == 1
    assert L.hpcgb200_benchmark_report(None, None, 0, None) == 1
    assert L.hpcgb200_problem_set_fallback(None, 2.0, 16, 16, 0.8) == 1


def test_no_cpu_fallback_without_device():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a device is visible here")
    except ImportError:
        pass
    with pytest.raises(R.HpcgError) as ei:
        R.Problem(16)
    assert ei.value.code == 7  # HPCGB200_ERR_NO_DEVICE


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(ImportError):
        _lib.load(str(tmp_path / "libhpcgb200.so"))
