"""In-tree build of libhpcgb200.so (CUDA kernels + C ABI + C++ host layer) for sm_100a.

Run ``python -m rochpcg_b200.build`` (or call :func:`build`).  Objects go to
``rochpcg_b200/_build/`` and the shared library to ``rochpcg_b200/libhpcgb200.so``;
a rebuild only recompiles sources newer than their object (or any header).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhpcgb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nccl_include() -> list[str]:
    """nccl.h for the decomposed solver's types (the library itself is
    opened at run time): the NCCL wheel's headers, else the system ones."""
    try:
        import nvidia.nccl as nc

        for d in nc.__path__:
            inc = os.path.join(d, "include")
            if os.path.isfile(os.path.join(inc, "nccl.h")):
                return ["-I" + inc]
    except ImportError:
        pass
    return []


NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
              "-I" + os.path.join(ROOT, "include")] + _nccl_include() + ARCH


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    cu = sorted(glob.glob(os.path.join(PKG, "csrc", "*.cu")))
    cpp = sorted(glob.glob(os.path.join(PKG, "host", "*.cpp")))
    return cu + cpp


def _headers():
    hs = glob.glob(os.path.join(PKG, "csrc", "*.cuh")) + glob.glob(os.path.join(PKG, "host", "*.hpp"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return hs


def _obj(src: str) -> str:
    rel = os.path.relpath(src, PKG).replace(os.sep, "_")
    return os.path.join(BUILD, rel + ".o")


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    newest_header = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    todo = []
    for s in srcs:
        o = _obj(s)
        if not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), newest_header):
            todo.append(s)
    cc = nvcc()

    def compile_one(src: str):
        cmd = [cc] + NVCC_FLAGS + ["-x", "cu", "-c", src, "-o", _obj(src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        return src

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for _ in ex.map(compile_one, todo):
                pass
    objs = [_obj(s) for s in srcs]
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [cc] + ARCH + ["-shared", "-o", tmp] + objs + ["-ldl", "-Xlinker", "--no-undefined"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
