"""CPU oracle of the DBCSR SMM stack path (test infrastructure only).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this
package, as the checker; the product (``libxstream_b200``) never imports it. The C restatement of
the reference semantics is in ``smm_oracle.c`` (see its header for the reference citations).
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from .build import OUT, build

_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = build()
        _lib = ctypes.CDLL(str(path))
        _lib.oracle_smm_f64.argtypes = [_ip, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int]
        _lib.oracle_smm_f64_omp.argtypes = [_ip, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.oracle_smm_f64_fast.argtypes = [_ip, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int]
        _lib.oracle_transpose_f64.argtypes = [_ip, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int]
        _lib.oracle_norms.argtypes = [_dp, ctypes.c_int, _ip, _ip, ctypes.POINTER(ctypes.c_float)]
        _lib.oracle_block_relerr.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int]
        _lib.oracle_block_relerr.restype = ctypes.c_double
        _lib.oracle_max_threads.restype = ctypes.c_int
        _lib.oracle_fast_balance.argtypes = [ctypes.c_int, ctypes.c_int]
        _lib.oracle_fast_balance.restype = ctypes.c_double
        _lib.oracle_ozaki_slice.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_byte), _ip]
        _lib.oracle_ozaki_gemm.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int]
        _lib.oracle_ozaki_smm.argtypes = [_ip, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.oracle_slice_low_bit.argtypes = [ctypes.c_int]
        _lib.oracle_slice_low_bit.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def smm(stack: np.ndarray, a: np.ndarray, b: np.ndarray, c: np.ndarray, m: int, n: int, k: int,
        b_rowmajor: bool = True, threads: int = 1) -> np.ndarray:
    """C += A*B over the stack (int32 triples, 1-based offsets) in place; returns c."""
    stack = np.ascontiguousarray(stack, dtype=np.int32)
    assert a.dtype == b.dtype == c.dtype == np.float64 and c.flags.c_contiguous
    S = stack.size // 3
    if threads == 1:
        lib().oracle_smm_f64(_p(stack, ctypes.c_int), S, _p(a, ctypes.c_double), _p(b, ctypes.c_double),
                             _p(c, ctypes.c_double), m, n, k, int(b_rowmajor))
    else:
        lib().oracle_smm_f64_omp(_p(stack, ctypes.c_int), S, _p(a, ctypes.c_double), _p(b, ctypes.c_double),
                                 _p(c, ctypes.c_double), m, n, k, int(b_rowmajor), int(threads))
    return c


def smm_fast(stack: np.ndarray, a: np.ndarray, b: np.ndarray, c: np.ndarray, m: int, n: int, k: int,
             threads: int = 0) -> np.ndarray:
    """Timed CPU baseline (register-tiled, FMA, all threads; B column-major): C += A*B in place. The
    stack is grouped by C and cut into equal contiguous ranges, one per thread (balanced whatever the
    C distribution)."""
    stack = np.ascontiguousarray(stack, dtype=np.int32)
    assert a.dtype == b.dtype == c.dtype == np.float64 and c.flags.c_contiguous
    lib().oracle_smm_f64_fast(_p(stack, ctypes.c_int), stack.size // 3, _p(a, ctypes.c_double), _p(b, ctypes.c_double),
                              _p(c, ctypes.c_double), m, n, k, int(threads))
    return c


def transpose(trs: np.ndarray, offset: int, data: np.ndarray, m: int, n: int) -> np.ndarray:
    trs = np.ascontiguousarray(trs, dtype=np.int32)
    S = trs.size - offset
    lib().oracle_transpose_f64(_p(trs, ctypes.c_int), offset, S, _p(data, ctypes.c_double), m, n)
    return data


def norms(mat: np.ndarray, offsets: np.ndarray, nelems: np.ndarray) -> np.ndarray:
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    nelems = np.ascontiguousarray(nelems, dtype=np.int32)
    out = np.zeros(offsets.size, dtype=np.float32)
    lib().oracle_norms(_p(mat, ctypes.c_double), offsets.size, _p(offsets, ctypes.c_int), _p(nelems, ctypes.c_int),
                       _p(out, ctypes.c_float))
    return out


def block_relerr(x: np.ndarray, ref: np.ndarray, blocksize: int) -> float:
    """max over blocks of max|x - ref| / max|ref| (per C block)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    ref = np.ascontiguousarray(ref, dtype=np.float64)
    return float(lib().oracle_block_relerr(_p(x, ctypes.c_double), _p(ref, ctypes.c_double), ref.size // blocksize,
                                           blocksize))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def fast_balance(S: int, threads: int) -> float:
    """Busiest thread's share of smm_fast's entries relative to the mean (1.0 = balanced)."""
    return float(lib().oracle_fast_balance(int(S), int(threads)))


def ozaki_slice(x: np.ndarray, rows: int, cols: int, rs: int, cs: int, nslices: int):
    """Digit planes int8[nslices, rows, cols] and per-row biased max exponent int32[rows]."""
    digits = np.zeros((nslices, rows, cols), dtype=np.int8)
    emax = np.zeros(rows, dtype=np.int32)
    lib().oracle_ozaki_slice(_p(x, ctypes.c_double), rows, cols, rs, cs, nslices, _p(digits, ctypes.c_byte),
                             _p(emax, ctypes.c_int))
    return digits, emax


def ozaki_gemm(A: np.ndarray, B: np.ndarray, C: np.ndarray, M: int, N: int, K: int, nslices: int,
               cutoff: int = -1) -> np.ndarray:
    """Scheme-1 Ozaki C += A*B (column-major operands) in place."""
    lib().oracle_ozaki_gemm(_p(A, ctypes.c_double), _p(B, ctypes.c_double), _p(C, ctypes.c_double), M, N, K, nslices,
                            cutoff)
    return C


def ozaki_smm(stack: np.ndarray, a: np.ndarray, b: np.ndarray, c: np.ndarray, m: int, n: int, k: int, nslices: int,
              cutoff: int = -1, b_rowmajor: bool = True) -> np.ndarray:
    """Ozaki scheme-1 stack multiply (per-block row/column scaling) C += A*B in place; returns c."""
    stack = np.ascontiguousarray(stack, dtype=np.int32)
    lib().oracle_ozaki_smm(_p(stack, ctypes.c_int), stack.size // 3, _p(a, ctypes.c_double), _p(b, ctypes.c_double),
                           _p(c, ctypes.c_double), m, n, k, int(b_rowmajor), nslices, cutoff)
    return c


__all__ = ["lib", "smm", "smm_fast", "fast_balance", "transpose", "norms", "block_relerr", "max_threads", "ozaki_slice", "ozaki_gemm", "ozaki_smm", "OUT",
           "Path"]
