"""GPU test of the CP2K offload API (include/offload_cp2k.h; the reference's libxstream_cp2k.h):
streams, events, device/host memory, copies and memsets in the order CP2K's offload layer uses them."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_offload_roundtrip(acc):
    A, _ = acc
    L = A.lib()
    n = 1 << 16
    s1, s2, ev = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    L.offloadStreamCreate(ctypes.byref(s1))
    L.offloadStreamCreate(ctypes.byref(s2))
    L.offloadEventCreate(ctypes.byref(ev))
    d1, d2, hp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    L.offloadMalloc(ctypes.byref(d1), n)
    L.offloadMalloc(ctypes.byref(d2), n)
    L.offloadMallocHost(ctypes.byref(hp), n)
    host = np.ctypeslib.as_array(ctypes.cast(hp, ctypes.POINTER(ctypes.c_ubyte)), shape=(n,))
    src = (np.arange(n) % 251).astype(np.uint8)
    host[:] = src
    L.offloadMemcpyAsyncHtoD(d1, hp, n, s1)
    L.offloadEventRecord(ev, s1)
    L.offloadStreamWaitEvent(s2, ev)
    L.offloadMemcpyAsyncDtoD(d2, d1, n, s2)
    L.offloadMemsetAsync(d1, 7, n // 2, s2)
    L.offloadStreamSynchronize(s2)
    assert L.offloadEventQuery(ev)
    L.offloadEventSynchronize(ev)
    out = np.zeros(n, dtype=np.uint8)
    L.offloadMemcpyDtoH(out.ctypes.data_as(ctypes.c_void_p), d2, n)
    assert np.array_equal(out, src)
    L.offloadMemcpyDtoH(out.ctypes.data_as(ctypes.c_void_p), d1, n)
    assert np.all(out[: n // 2] == 7) and np.array_equal(out[n // 2:], src[n // 2:])
    L.offloadMemset(d1, 0, n)
    L.offloadMemcpyDtoH(out.ctypes.data_as(ctypes.c_void_p), d1, n)
    assert not np.any(out)
    L.offloadMemcpyToSymbol(None, None, 0)
    L.offloadEnsureMallocHeapSize(1 << 20)
    L.offloadDeviceSynchronize()
    assert L.offloadGetLastError() == 0
    assert L.offloadGetErrorName(0) == b"cudaSuccess"
    L.offloadFree(d1)
    L.offloadFree(d2)
    L.offloadFreeHost(hp)
    L.offloadEventDestroy(ev)
    L.offloadStreamDestroy(s1)
    L.offloadStreamDestroy(s2)
