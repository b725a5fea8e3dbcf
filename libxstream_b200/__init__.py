"""B200-native DBCSR small-matrix-multiply (SMM) stack library.

The product is the C-ABI shared library ``libxstream_b200/_lib/libxstream_b200.so`` (C host code on
the CUDA runtime plus hand-written sm_100a kernels). This package only binds it with ``ctypes`` so
that Python tests and benchmarks call exactly the entry points DBCSR calls (``c_dbcsr_acc_*``,
``libsmm_acc_*``). There is no Python or CPU fallback: if the library is missing, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "_lib" / "libxstream_b200.so"

_lib = None

c_int_p = ctypes.POINTER(ctypes.c_int)
c_void_pp = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); every function the headers in include/ declare
SIGNATURES = {
    # include/dbcsr_acc.h
    "c_dbcsr_acc_init": (ctypes.c_int, []),
    "c_dbcsr_acc_finalize": (ctypes.c_int, []),
    "c_dbcsr_acc_clear_errors": (None, []),
    "c_dbcsr_acc_get_ndevices": (ctypes.c_int, [c_int_p]),
    "c_dbcsr_acc_set_active_device": (ctypes.c_int, [ctypes.c_int]),
    "c_dbcsr_acc_device_synchronize": (ctypes.c_int, []),
    "c_dbcsr_acc_stream_priority_range": (ctypes.c_int, [c_int_p, c_int_p]),
    "c_dbcsr_acc_stream_create": (ctypes.c_int, [c_void_pp, ctypes.c_char_p, ctypes.c_int]),
    "c_dbcsr_acc_stream_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "c_dbcsr_acc_stream_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "c_dbcsr_acc_stream_wait_event": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "c_dbcsr_acc_event_create": (ctypes.c_int, [c_void_pp]),
    "c_dbcsr_acc_event_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "c_dbcsr_acc_event_record": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "c_dbcsr_acc_event_query": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "c_dbcsr_acc_event_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "c_dbcsr_acc_dev_mem_allocate": (ctypes.c_int, [c_void_pp, ctypes.c_size_t]),
    "c_dbcsr_acc_dev_mem_deallocate": (ctypes.c_int, [ctypes.c_void_p]),
    "c_dbcsr_acc_dev_mem_set_ptr": (ctypes.c_int, [c_void_pp, ctypes.c_void_p, ctypes.c_size_t]),
    "c_dbcsr_acc_host_mem_allocate": (ctypes.c_int, [c_void_pp, ctypes.c_size_t, ctypes.c_void_p]),
    "c_dbcsr_acc_host_mem_deallocate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "c_dbcsr_acc_memcpy_h2d": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "c_dbcsr_acc_memcpy_d2h": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "c_dbcsr_acc_memcpy_d2d": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "c_dbcsr_acc_memset_zero": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p]),
    "c_dbcsr_acc_dev_mem_info": (ctypes.c_int, [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "c_dbcsr_timeset": (None, [ctypes.c_void_p, c_int_p, c_int_p]),
    "c_dbcsr_timestop": (None, [c_int_p]),
    # include/libsmm_acc.h
    "libsmm_acc_init": (ctypes.c_int, []),
    "libsmm_acc_finalize": (ctypes.c_int, []),
    "libsmm_acc_is_thread_safe": (ctypes.c_int, []),
    "libsmm_acc_transpose": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "libsmm_acc_process": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "c_calculate_norms": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    # include/libxstream_b200.h
    "libxstream_b200_process_suitable": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                        ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "libxstream_b200_last_error": (ctypes.c_int, []),
    "libxstream_b200_fp64_peak": (ctypes.c_double, [ctypes.c_void_p]),
    "libxstream_b200_set_params": (ctypes.c_int, [ctypes.c_int] * 8),
    "libxstream_b200_get_params": (ctypes.c_int, [ctypes.c_int] * 4 + [c_int_p]),
    "libxstream_b200_clear_params": (None, []),
    "libxstream_b200_load_params": (ctypes.c_int, [ctypes.c_char_p]),
    "libxstream_b200_inject_alloc_failure": (None, [ctypes.c_int]),
    "libxstream_b200_profile_enable": (None, [ctypes.c_int]),
    "libxstream_b200_profile_reset": (None, []),
    "libxstream_b200_profile_query": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_long),
                                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                                     ctypes.POINTER(ctypes.c_double)]),
    "libxstream_b200_profile_kernels": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "libxstream_b200_event_create_timed": (ctypes.c_int, [c_void_pp]),
    "libxstream_b200_event_elapsed_ms": (ctypes.c_double, [ctypes.c_void_p, ctypes.c_void_p]),
    "libxstream_b200_graph_begin": (ctypes.c_int, [ctypes.c_void_p]),
    "libxstream_b200_graph_end": (ctypes.c_int, [ctypes.c_void_p, c_void_pp, c_int_p]),
    "libxstream_b200_graph_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "libxstream_b200_graph_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "libxstream_b200_ozaki_gemm": (ctypes.c_int, [ctypes.c_char, ctypes.c_char, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "libxstream_b200_ozaki2_gemm": (ctypes.c_int, [ctypes.c_char, ctypes.c_char, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                   ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_void_p]),
    "libxstream_b200_dgemm": (ctypes.c_int, [ctypes.c_char, ctypes.c_char, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "libxstream_b200_process_ozaki": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                     ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                     ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "libxstream_b200_tune_candidates": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]),
    "libxstream_b200_tune": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_uint, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "libxstream_b200_mlp_nweights": (ctypes.c_int, []),
    "libxstream_b200_mlp_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]),
    "libxstream_b200_mlp_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p]),
    "libxstream_b200_mlp_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "libxstream_b200_mlp_predict": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p]),
    "libxstream_b200_mlp_install": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "libxstream_b200_mlp_lookup": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_void_p]),
    "libxstream_b200_set_dbm_launch_fn": (None, [ctypes.c_void_p]),
    "libxstream_b200_dbm_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    # CP2K offload API (include/offload_cp2k.h)
    "offloadGetErrorName": (ctypes.c_char_p, [ctypes.c_int]),
    "offloadGetLastError": (ctypes.c_int, []),
    "offloadMemsetAsync": (None, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p]),
    "offloadMemset": (None, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t]),
    "offloadMemcpyAsyncHtoD": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "offloadMemcpyAsyncDtoH": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "offloadMemcpyAsyncDtoD": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "offloadMemcpyHtoD": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "offloadMemcpyDtoH": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "offloadMemcpyToSymbol": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "offloadEventCreate": (None, [ctypes.c_void_p]),
    "offloadEventDestroy": (None, [ctypes.c_void_p]),
    "offloadEventSynchronize": (None, [ctypes.c_void_p]),
    "offloadEventRecord": (None, [ctypes.c_void_p, ctypes.c_void_p]),
    "offloadEventQuery": (ctypes.c_bool, [ctypes.c_void_p]),
    "offloadStreamCreate": (None, [ctypes.c_void_p]),
    "offloadStreamDestroy": (None, [ctypes.c_void_p]),
    "offloadStreamSynchronize": (None, [ctypes.c_void_p]),
    "offloadStreamWaitEvent": (None, [ctypes.c_void_p, ctypes.c_void_p]),
    "offloadMallocHost": (None, [ctypes.c_void_p, ctypes.c_size_t]),
    "offloadMalloc": (None, [ctypes.c_void_p, ctypes.c_size_t]),
    "offloadFree": (None, [ctypes.c_void_p]),
    "offloadFreeHost": (None, [ctypes.c_void_p]),
    "offloadDeviceSynchronize": (None, []),
    "offloadEnsureMallocHeapSize": (None, [ctypes.c_size_t]),
    "libxstream_b200_process_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                       ctypes.c_void_p, ctypes.c_void_p]),
    "libxstream_b200_noalloc_scratch_bytes": (ctypes.c_size_t, []),
    "libxstream_b200_process_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "libxstream_b200_device_error": (ctypes.c_int, [ctypes.c_int]),
    "libxstream_b200_set_wait_limit": (None, [ctypes.c_longlong]),
    "libxstream_b200_get_wait_limit": (ctypes.c_longlong, []),
    "libxstream_b200_process_scratch_bytes": (ctypes.c_size_t, [ctypes.c_int] * 4),
}

DBCSR_TYPE_REAL_4 = 1
DBCSR_TYPE_REAL_8 = 3


class LibraryMissing(RuntimeError):
    pass


class StackDesc(ctypes.Structure):
    """libxstream_b200_stack_t (include/libxstream_b200.h): one stack of a batch."""
    _fields_ = [("dev_param_stack", ctypes.c_void_p), ("stack_size", ctypes.c_int), ("m", ctypes.c_int),
                ("n", ctypes.c_int), ("k", ctypes.c_int), ("a", ctypes.c_void_p), ("b", ctypes.c_void_p),
                ("c", ctypes.c_void_p)]


def lib() -> ctypes.CDLL:
    """Load the CUDA library (building it first if the sources are newer). Raises if unavailable."""
    global _lib
    if _lib is None:
        if os.environ.get("LIBXSTREAM_B200_NOBUILD") != "1":
            try:
                from . import build as _build
                _build.build()
            except Exception as exc:  # the prebuilt library may still be there
                if not LIB_PATH.exists():
                    raise LibraryMissing(f"cannot build {LIB_PATH}: {exc}") from exc
        if not LIB_PATH.exists():
            raise LibraryMissing(f"{LIB_PATH} is missing: run `python -m libxstream_b200.build`")
        handle = ctypes.CDLL(str(LIB_PATH), mode=ctypes.RTLD_GLOBAL)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(rc: int, what: str = "call") -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed with code {rc} (last CUDA error {lib().libxstream_b200_last_error()})")


from . import acc  # noqa: E402  (thin wrappers over the C-ABI)

__all__ = ["lib", "check", "acc", "SIGNATURES", "LIB_PATH", "DBCSR_TYPE_REAL_8", "DBCSR_TYPE_REAL_4",
           "LibraryMissing"]
