"""Thin Python wrappers over the C-ABI, mirroring how DBCSR and the reference's acc_bench drive it.

Every call goes through the exported ``c_dbcsr_acc_*`` / ``libsmm_acc_*`` symbols; nothing here
computes on the CPU. Buffers are raw device pointers from ``c_dbcsr_acc_dev_mem_allocate`` and
pinned host memory from ``c_dbcsr_acc_host_mem_allocate`` viewed as numpy arrays.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import DBCSR_TYPE_REAL_8, check, lib


def init() -> None:
    check(lib().c_dbcsr_acc_init(), "c_dbcsr_acc_init")
    check(lib().libsmm_acc_init(), "libsmm_acc_init")


def finalize() -> None:
    check(lib().libsmm_acc_finalize(), "libsmm_acc_finalize")
    check(lib().c_dbcsr_acc_finalize(), "c_dbcsr_acc_finalize")


def ndevices() -> int:
    n = ctypes.c_int(0)
    check(lib().c_dbcsr_acc_get_ndevices(ctypes.byref(n)), "c_dbcsr_acc_get_ndevices")
    return n.value


class Stream:
    def __init__(self, name: str = "stream", priority: int = -1):
        h = ctypes.c_void_p()
        check(lib().c_dbcsr_acc_stream_create(ctypes.byref(h), name.encode(), priority), "stream_create")
        self.handle = h.value

    def sync(self) -> None:
        check(lib().c_dbcsr_acc_stream_sync(self.handle), "stream_sync")

    def destroy(self) -> None:
        if self.handle:
            check(lib().c_dbcsr_acc_stream_destroy(self.handle), "stream_destroy")
            self.handle = None


class Event:
    def __init__(self):
        h = ctypes.c_void_p()
        check(lib().c_dbcsr_acc_event_create(ctypes.byref(h)), "event_create")
        self.handle = h.value

    def record(self, stream: Stream | None) -> None:
        check(lib().c_dbcsr_acc_event_record(self.handle, stream.handle if stream else None), "event_record")

    def query(self) -> bool:
        occ = ctypes.c_int(0)
        check(lib().c_dbcsr_acc_event_query(self.handle, ctypes.byref(occ)), "event_query")
        return bool(occ.value)

    def sync(self) -> None:
        check(lib().c_dbcsr_acc_event_synchronize(self.handle), "event_synchronize")

    def destroy(self) -> None:
        if self.handle:
            check(lib().c_dbcsr_acc_event_destroy(self.handle), "event_destroy")
            self.handle = None


class DevBuf:
    """Device allocation through c_dbcsr_acc_dev_mem_allocate."""

    def __init__(self, nbytes: int):
        h = ctypes.c_void_p()
        check(lib().c_dbcsr_acc_dev_mem_allocate(ctypes.byref(h), int(nbytes)), "dev_mem_allocate")
        self.ptr = h.value
        self.nbytes = int(nbytes)

    @classmethod
    def from_array(cls, arr: np.ndarray, stream: Stream | None = None) -> "DevBuf":
        arr = np.ascontiguousarray(arr)
        buf = cls(arr.nbytes)
        buf.upload(arr, stream)
        return buf

    def upload(self, arr: np.ndarray, stream: Stream | None = None) -> None:
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes <= self.nbytes
        check(lib().c_dbcsr_acc_memcpy_h2d(arr.ctypes.data, self.ptr, arr.nbytes, stream.handle if stream else None),
              "memcpy_h2d")

    def download(self, out: np.ndarray, stream: Stream | None = None) -> np.ndarray:
        assert out.flags.c_contiguous and out.nbytes <= self.nbytes
        check(lib().c_dbcsr_acc_memcpy_d2h(self.ptr, out.ctypes.data, out.nbytes, stream.handle if stream else None),
              "memcpy_d2h")
        return out

    def zero(self, stream: Stream | None = None, offset: int = 0, nbytes: int | None = None) -> None:
        n = self.nbytes - offset if nbytes is None else nbytes
        check(lib().c_dbcsr_acc_memset_zero(self.ptr, offset, n, stream.handle if stream else None), "memset_zero")

    def free(self) -> None:
        if self.ptr:
            check(lib().c_dbcsr_acc_dev_mem_deallocate(self.ptr), "dev_mem_deallocate")
            self.ptr = None


class HostBuf:
    """Pinned host allocation through c_dbcsr_acc_host_mem_allocate, viewed as a numpy array."""

    def __init__(self, shape, dtype, stream: Stream | None = None):
        dtype = np.dtype(dtype)
        count = int(np.prod(shape))
        h = ctypes.c_void_p()
        check(lib().c_dbcsr_acc_host_mem_allocate(ctypes.byref(h), max(1, count * dtype.itemsize),
                                                  stream.handle if stream else None), "host_mem_allocate")
        self.ptr = h.value
        raw = (ctypes.c_char * max(1, count * dtype.itemsize)).from_address(self.ptr)
        self.array = np.frombuffer(raw, dtype=dtype, count=count).reshape(shape)

    def free(self, stream: Stream | None = None) -> None:
        if self.ptr:
            self.array = None
            check(lib().c_dbcsr_acc_host_mem_deallocate(self.ptr, stream.handle if stream else None), "host_free")
            self.ptr = None


def process(stack: DevBuf, stack_size: int, a: DevBuf, b: DevBuf, c: DevBuf, m: int, n: int, k: int,
            stream: Stream | None, max_kernel_dim: int = 80, def_mnk: int = 1, dtype: int = DBCSR_TYPE_REAL_8,
            host_stack=None) -> int:
    """libsmm_acc_process; returns its code (0 ok, -1 = not handled, host fallback)."""
    hs = None if host_stack is None else host_stack.ctypes.data
    return lib().libsmm_acc_process(hs, stack.ptr, stack_size, dtype, a.ptr, b.ptr, c.ptr, m, n, k, max_kernel_dim,
                                    def_mnk, stream.handle if stream else None, stream.handle if stream else None)


def transpose(trs: DevBuf, offset: int, stack_size: int, data: DevBuf, m: int, n: int, stream: Stream | None,
              max_kernel_dim: int = 80, dtype: int = DBCSR_TYPE_REAL_8) -> int:
    return lib().libsmm_acc_transpose(trs.ptr, offset, stack_size, data.ptr, dtype, m, n, max_kernel_dim,
                                      stream.handle if stream else None)


def norms(mat: DevBuf, nblks: int, offsets: DevBuf, nelems: DevBuf, out: DevBuf, stream: Stream | None) -> int:
    return lib().c_calculate_norms(mat.ptr, nblks, offsets.ptr, nelems.ptr, out.ptr, stream.handle if stream else None)


def set_params(m: int, n: int, k: int, chunk: int, mt: int, nt: int, kp: int = 4, wpb: int = 4) -> None:
    check(lib().libxstream_b200_set_params(m, n, k, chunk, mt, nt, kp, wpb), "set_params")


def get_params(m: int, n: int, k: int, stack_size: int) -> dict:
    out = (ctypes.c_int * 6)()
    check(lib().libxstream_b200_get_params(m, n, k, stack_size, out), "get_params")
    return dict(zip(("chunk", "mt", "nt", "kp", "wpb", "sorted"), list(out)))


def fp64_peak(stream: Stream | None = None) -> float:
    return float(lib().libxstream_b200_fp64_peak(stream.handle if stream else None))


def ozaki_gemm(transa: str, transb: str, M: int, N: int, K: int, alpha: float, a: DevBuf, lda: int, b: DevBuf,
               ldb: int, beta: float, c: DevBuf, ldc: int, nslices: int = 8, trim: int = 0,
               stream: Stream | None = None) -> int:
    """libxstream_b200_ozaki_gemm: C = alpha*op(A)*op(B) + beta*C (column-major, device buffers)."""
    return lib().libxstream_b200_ozaki_gemm(transa.encode(), transb.encode(), M, N, K, alpha, a.ptr, lda, b.ptr, ldb,
                                            beta, c.ptr, ldc, nslices, trim, stream.handle if stream else None)


def ozaki2_gemm(transa: str, transb: str, M: int, N: int, K: int, alpha: float, a: DevBuf, lda: int, b: DevBuf,
                ldb: int, beta: float, c: DevBuf, ldc: int, nmoduli: int = 0, stream: Stream | None = None) -> int:
    """libxstream_b200_ozaki2_gemm: C = alpha*op(A)*op(B) + beta*C by the CRT scheme (column-major, device buffers)."""
    return lib().libxstream_b200_ozaki2_gemm(transa.encode(), transb.encode(), M, N, K, alpha, a.ptr, lda, b.ptr, ldb,
                                             beta, c.ptr, ldc, nmoduli, stream.handle if stream else None)


def dgemm(M: int, N: int, K: int, alpha: float, a: DevBuf, lda: int, b: DevBuf, ldb: int, beta: float, c: DevBuf,
          ldc: int, stream: Stream | None = None) -> int:
    """libxstream_b200_dgemm (plain FP64 DMMA GEMM, 'N', 'N')."""
    return lib().libxstream_b200_dgemm(b"N", b"N", M, N, K, alpha, a.ptr, lda, b.ptr, ldb, beta, c.ptr, ldc,
                                       stream.handle if stream else None)


def process_ozaki(stack: DevBuf, stack_size: int, m: int, n: int, k: int, a: DevBuf, na: int, b: DevBuf, nb: int,
                  c: DevBuf, nslices: int = 7, trim: int = 0, stream: Stream | None = None) -> int:
    """libxstream_b200_process_ozaki (B pool already transposed to k x n row-major)."""
    return lib().libxstream_b200_process_ozaki(stack.ptr, stack_size, m, n, k, a.ptr, na, b.ptr, nb, c.ptr, nslices, trim,
                                               stream.handle if stream else None)
