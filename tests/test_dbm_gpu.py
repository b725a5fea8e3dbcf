"""GPU tests of the DBM interplay: libxstream_b200_dbm_launch runs DBM-format task batches (6-int
records (m, n, k, a, b, c) with 0-based offsets, C += alpha*A*B) on the stack kernels, and the hook
installed with libxstream_b200_set_dbm_launch_fn receives libsmm_acc_process's stacks
(samples/smm/smm_acc.c:579-585 semantics)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W

pytestmark = pytest.mark.gpu


def dbm_records(case: W.StackCase) -> np.ndarray:
    rec = np.empty((case.S, 6), dtype=np.int32)
    rec[:, 0], rec[:, 1], rec[:, 2] = case.m, case.n, case.k
    rec[:, 3:] = case.stack - 1  # 0-based offsets
    return rec


@pytest.mark.parametrize("shape,alpha", [((23, 23, 23), -0.5), ((5, 13, 7), 2.0), ((45, 45, 45), 1.0)])
def test_dbm_launch_format_and_alpha(acc, shape, alpha):
    A, stream = acc
    m, n, k = shape
    case = W.stack_case(m, n, k, 5000, 200, 200, 40, seed=31 + m)
    c0 = W.rng(8).uniform(-1, 1, size=case.nc * m * n)
    da, db = A.DevBuf.from_array(case.a, stream), A.DevBuf.from_array(case.b_rowmajor(), stream)
    dc = A.DevBuf.from_array(c0, stream)
    dp = A.DevBuf.from_array(dbm_records(case), stream)
    fmt = m | (n << 8) | (k << 16)
    rc = A.lib().libxstream_b200_dbm_launch(stream.handle, alpha, case.S, fmt, None, dp.ptr, da.ptr, db.ptr, dc.ptr)
    got = dc.download(np.zeros_like(c0), stream)
    stream.sync()
    assert rc == 0
    prod = np.zeros_like(c0)
    oracle.smm(case.stack, case.a, case.b, prod, m, n, k, b_rowmajor=False)
    ref = c0 + alpha * prod
    assert oracle.block_relerr(got, ref, m * n) <= 1e-13
    assert A.lib().libxstream_b200_dbm_launch(stream.handle, alpha, case.S, 0, None, dp.ptr, da.ptr, db.ptr, dc.ptr) == -1
    for b in (da, db, dc, dp):
        b.free()


def test_hook_receives_libsmm_stacks(acc):
    A, stream = acc
    lib = A.lib()
    calls = []
    proto = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)

    @proto
    def hook(stream_h, alpha, ntasks, fmt, params_host, params, a, b, c):
        calls.append((alpha, ntasks, fmt))
        return 0

    case = W.stack_case(8, 9, 10, 100, 10, 10, 5, seed=2)
    da, db = A.DevBuf.from_array(case.a, stream), A.DevBuf.from_array(case.b_rowmajor(), stream)
    ds, dc = A.DevBuf.from_array(case.stack, stream), A.DevBuf(case.nc * 72 * 8)
    dc.zero(stream)
    lib.libxstream_b200_set_dbm_launch_fn(ctypes.cast(hook, ctypes.c_void_p))
    try:
        assert A.process(ds, case.S, da, db, dc, 8, 9, 10, stream) == 0
    finally:
        lib.libxstream_b200_set_dbm_launch_fn(None)
    assert calls == [(1.0, case.S, 8 | (9 << 8) | (10 << 16))]
    assert not np.any(dc.download(np.zeros(case.nc * 72), stream))  # the hook did the work (nothing here)
    stream.sync()
    for b in (da, db, ds, dc):
        b.free()
