"""Build the B200 SMM library (C host layer + sm_100a kernels) in-tree.

Produces ``libxstream_b200/_lib/libxstream_b200.so``: a self-contained shared library (CUDA runtime
linked statically, only ``libcuda.so.1`` needed at run time) that exports the DBCSR ACC ABI
(``c_dbcsr_acc_*``), the LIBSMM ABI (``libsmm_acc_*``) and the ``libxstream_b200_*`` extensions.
Objects are rebuilt only when a source or header is newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OUT_DIR = PKG / "_lib"
OBJ_DIR = PKG / "_build"
LIB = OUT_DIR / "libxstream_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
C_SOURCES = ["acc_runtime.c", "smm_params.c", "smm_acc.c", "profile.c", "gemm_api.c", "predictor.c", "offload_cp2k.c"]
CU_SOURCES = ["smm_kernels.cu", "stack_sort.cu", "smm_noalloc.cu", "ozaki_gemm.cu", "ozaki2_gemm.cu", "dgemm.cu", "ozaki_smm.cu", "tune.cu", "mlp.cu"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libxstream_b200")
    return cand


def _cuda_include() -> str:
    return str(Path(_nvcc()).resolve().parent.parent / "include")


def _newest_input() -> float:
    files = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return max(f.stat().st_mtime for f in files if f.is_file())


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + proc.stdout + proc.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} (exit {proc.returncode})")


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every source for sm_100a and link the shared library; returns its path."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= _newest_input():
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    OBJ_DIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in C_SOURCES:
        obj = OBJ_DIR / (src + ".o")
        _run(["gcc", "-O2", "-std=c11", "-D_GNU_SOURCE", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter",
              "-I", _cuda_include(), "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(obj)
    jobs = []
    for src in CU_SOURCES:
        obj = OBJ_DIR / (src + ".o")
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    for cmd, proc in jobs:
        out, _ = proc.communicate()
        if verbose and out:
            sys.stderr.write(out)
        if proc.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + out)
            raise RuntimeError(f"nvcc failed on {cmd[-3]}")
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs), "-lpthread", "-ldl"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
