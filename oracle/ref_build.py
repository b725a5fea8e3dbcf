"""Builds the reference's own SMM kernels (samples/smm/kernels/multiply.cl and transpose.cl, read in
place under the reference tree) as host C shared libraries into oracle/_ref/, with the shim in
oracle/ref_shim/. Test infrastructure only: used to pin the oracle and to generate the golden
fixtures; the product never loads these. Needs the reference tree (this build container), not a GPU.

Configurations mirror the reference host's build parameters (samples/smm/smm_kernel.c:339-347):
T=double, SM/SN/SK = block shape, BM/BN/BK tile, BS mini-batch, WG = ceil(SM/BM)*ceil(SN/BN)
work-items; REG_A/REG_B (private copies) may be set; local-memory variants are not built (see the
shim's execution model).
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# The reference tree: XS_REFERENCE_ROOT, else a checkout named "reference" beside this repository. Where
# neither exists (the GPU box), available() is False and everything that needs the tree skips.
REFERENCE = Path(os.environ["XS_REFERENCE_ROOT"]) if os.environ.get("XS_REFERENCE_ROOT") else HERE.parent.parent / "reference"
MULTIPLY = REFERENCE / "samples" / "smm" / "kernels" / "multiply.cl"
TRANSPOSE = REFERENCE / "samples" / "smm" / "kernels" / "transpose.cl"


def available() -> bool:
    return MULTIPLY.exists() and TRANSPOSE.exists()


def _compile(src: Path, defines: dict[str, object], tag: str) -> Path:
    OUT.mkdir(exist_ok=True)
    key = hashlib.sha1(repr(sorted(defines.items())).encode() + src.read_bytes()).hexdigest()[:12]
    lib = OUT / f"{tag}_{key}.so"
    if lib.exists():
        return lib
    dflags = [f"-D{k}={v}" if v is not None else f"-D{k}" for k, v in defines.items()]
    cmd = ["gcc", "-O1", "-shared", "-fPIC", "-std=gnu99", "-w", "-ffp-contract=off", "-I", str(HERE / "ref_shim"),
           "-include", str(HERE / "ref_shim" / "opencl_host.h"), *dflags, "-x", "c", str(src), "-x", "c",
           str(HERE / "ref_shim" / "ref_driver.c"), "-o", str(lib), "-lm"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("reference kernel build failed:\n" + " ".join(cmd) + "\n" + proc.stderr[-4000:])
    return lib


def multiply(m: int, n: int, k: int, bm: int | None = None, bn: int = 1, bk: int = 1, bs: int = 1, reg_a: bool = False,
             reg_b: bool = False, atomic_inc_nz: bool = False):
    """ctypes function xs_ref_process(stack, S, param_format, a, b, c) of the reference multiply kernel."""
    bm = m if bm is None else bm
    wg = -(-m // bm) * -(-n // bn)
    d = {"T": "double", "GPU": 0, "CONSTANT": "global", "WG": wg, "SG": 0, "INTEL": 0, "FN": "xs_ref_kernel", "REPEAT": 1,
         "LU": -1, "SM": m, "SN": n, "SK": k, "BS": bs, "VL": 1, "BM": bm, "BN": bn, "BK": bk, "XS_REF_MULTIPLY": 1}
    if bs > 1:
        d["BSC"] = None
    if reg_a:
        d["REG_A"] = None
    if reg_b:
        d["REG_B"] = None
    if atomic_inc_nz:
        d["ATOMIC_INC_NZ"] = None
    lib = ctypes.CDLL(str(_compile(MULTIPLY, d, f"multiply_{m}x{n}x{k}")))
    f = lib.xs_ref_process
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = None
    return f


def transpose(m: int, n: int, bs: int = 1):
    """ctypes function xs_ref_transpose(trs, offset, S, matrix) of the reference transpose kernel."""
    d = {"T": "double", "CONSTANT": "global", "WG": 1, "FN": "xs_ref_kernel", "SM": m, "SN": n, "BS": bs, "INPLACE": 0,
         "XS_REF_TRANSPOSE": 1}
    lib = ctypes.CDLL(str(_compile(TRANSPOSE, d, f"transpose_{m}x{n}")))
    f = lib.xs_ref_transpose
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    f.restype = None
    return f
