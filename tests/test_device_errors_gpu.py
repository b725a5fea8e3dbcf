"""Device-side errors reach the C-ABI: a bounded wait that runs out is reported by the ACC calls.

Every pipeline wait of the kernels is bounded; when one gives up, the kernel sets a bit in the
library's device error word and stops early, so nothing hangs or faults. This test makes that happen
on purpose and on the host's say-so, with no fault: it sets the wait bound to a few clock cycles
(libxstream_b200_set_wait_limit), so that the staged 23x23x23 stack kernel's first wait for a block
copy that is still in flight gives up. Then, as DBCSR would see it:
  - libsmm_acc_process itself returns 0 (the launch is asynchronous);
  - c_dbcsr_acc_stream_sync returns nonzero and the error slot holds cudaErrorTimeout;
  - the next libsmm_acc_process / libsmm_acc_transpose return nonzero without doing work;
  - c_dbcsr_acc_clear_errors consumes the word (the reference's error-slot consume,
    src/libxstream_dbcsr.c:57-62), after which the same call with the default bound is correct.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W

pytestmark = pytest.mark.gpu

CUDA_ERROR_TIMEOUT = 909  # cudaErrorTimeout
STAGED_TIMEOUT_BIT = 16   # device error word: a wait of the staged stack kernel gave up


def test_wait_limit_runs_out_and_reaches_the_abi(acc):
    A, stream = acc
    L = A.lib()
    m = n = k = 23  # a shape with a staged kernel (bulk copies + bounded mbarrier waits)
    case = W.stack_case(m, n, k, 3000, 256, 256, 64, seed=77)
    da = A.DevBuf.from_array(case.a, stream)
    db = A.DevBuf.from_array(case.b, stream)
    trs = A.DevBuf.from_array(np.arange(case.nb, dtype=np.int32) * (k * n), stream)
    ds = A.DevBuf.from_array(case.stack, stream)
    dc = A.DevBuf(case.nc * m * n * 8)
    assert A.transpose(trs, 0, case.nb, db, k, n, stream) == 0
    dc.zero(stream)
    stream.sync()
    assert L.libxstream_b200_device_error(1) == 0
    default_limit = L.libxstream_b200_get_wait_limit()
    A.set_params(m, n, k, 0, 3, 3, 0, 4)  # kp = 0: the staged kernel, whole C block per warp
    try:
        L.libxstream_b200_set_wait_limit(4)
        assert L.libxstream_b200_get_wait_limit() == 4
        assert A.process(ds, case.S, da, db, dc, m, n, k, stream) == 0  # asynchronous: launched fine
        assert L.c_dbcsr_acc_stream_sync(stream.handle) != 0           # the wait gave up
        assert L.libxstream_b200_last_error() == CUDA_ERROR_TIMEOUT
        assert L.libxstream_b200_device_error(0) & STAGED_TIMEOUT_BIT
        # until the error is cleared, stack calls refuse work (nonzero, not the -1 host fallback)
        L.libxstream_b200_set_wait_limit(0)
        rc = A.process(ds, case.S, da, db, dc, m, n, k, stream)
        assert rc not in (0, -1)
        assert A.transpose(trs, 0, case.nb, db, k, n, stream) not in (0, -1)
    finally:
        L.libxstream_b200_set_wait_limit(0)
        L.c_dbcsr_acc_clear_errors()
        L.libxstream_b200_clear_params()
    assert L.libxstream_b200_get_wait_limit() == default_limit
    assert L.libxstream_b200_device_error(0) == 0
    assert L.libxstream_b200_last_error() == 0
    # a clean call with the default bound: rc 0 everywhere and the right result
    dc.zero(stream)
    assert A.process(ds, case.S, da, db, dc, m, n, k, stream) == 0
    assert L.c_dbcsr_acc_stream_sync(stream.handle) == 0
    got = dc.download(np.zeros(case.nc * m * n), stream)
    stream.sync()
    ref = np.zeros_like(got)
    oracle.smm(case.stack, case.a, case.b, ref, m, n, k, b_rowmajor=False)
    assert oracle.block_relerr(got, ref, m * n) <= 1e-13
    assert L.c_dbcsr_acc_device_synchronize() == 0
    for b in (da, db, trs, ds, dc):
        b.free()


def test_device_synchronize_reports_and_clear_consumes(acc):
    """c_dbcsr_acc_device_synchronize reads the word too; clear_errors resets word, slot and refusal."""
    A, stream = acc
    L = A.lib()
    m, n, k = 16, 16, 16
    case = W.stack_case(m, n, k, 2000, 128, 128, 32, seed=78)
    da = A.DevBuf.from_array(case.a, stream)
    db = A.DevBuf.from_array(case.b, stream)  # the layout does not matter here: only the error path is checked
    ds = A.DevBuf.from_array(case.stack, stream)
    dc = A.DevBuf(case.nc * m * n * 8)
    dc.zero(stream)
    stream.sync()
    A.set_params(m, n, k, 0, 2, 2, 0, 4)  # the staged kernel
    try:
        L.libxstream_b200_set_wait_limit(4)
        assert A.process(ds, case.S, da, db, dc, m, n, k, stream) == 0
        assert L.c_dbcsr_acc_device_synchronize() != 0
        assert L.libxstream_b200_device_error(0) & STAGED_TIMEOUT_BIT
    finally:
        L.libxstream_b200_set_wait_limit(0)
        L.c_dbcsr_acc_clear_errors()
        L.libxstream_b200_clear_params()
    assert L.libxstream_b200_device_error(0) == 0
    assert A.process(ds, case.S, da, db, dc, m, n, k, stream) == 0
    assert L.c_dbcsr_acc_stream_sync(stream.handle) == 0
    for b in (da, db, ds, dc):
        b.free()
