"""GPU test of the allocation-free stack multiply (libxstream_b200_process_noalloc).

Callers that cannot let the library allocate device memory per call -- applications that reserve
almost all device memory for their own allocator, or code that must not risk the allocator's locks
and implicit synchronisation -- use this entry point; it runs on a fixed scratch array inside the
library. The test calls it through the C-ABI next to libsmm_acc_process on the same inputs, twice in
a row (the scratch array keeps the previous call's contents), and checks that both agree with each
other and with the CPU oracle within the FP64 tolerance of the other parity tests (relative
max-norm error per C block <= 1e-13). It also checks that a stack larger than the scratch array is
rejected before any work is done. This file sorts last so that a stop-at-first-failure run has
already run every other test when it gets here."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-13


def test_noalloc_matches_process_on_two_calls(acc):
    A, stream = acc
    lib = A.lib()
    case = W.config1()  # 23x23x23, 30000 entries, Zipf(1.1) c
    m, n, k = case.m, case.n, case.k
    need = lib.libxstream_b200_process_scratch_bytes(case.S, m, n, k)
    assert 0 < need <= lib.libxstream_b200_noalloc_scratch_bytes()
    da = A.DevBuf.from_array(case.a, stream)
    db = A.DevBuf.from_array(case.b_rowmajor(), stream)
    ds = A.DevBuf.from_array(case.stack, stream)
    size = case.nc * m * n
    dc_ref, dc_new = A.DevBuf(size * 8), A.DevBuf(size * 8)
    dc_ref.zero(stream)
    dc_new.zero(stream)
    ref = np.zeros(size)
    for call in range(2):
        assert A.process(ds, case.S, da, db, dc_ref, m, n, k, stream) == 0
        rc = lib.libxstream_b200_process_noalloc(None, ds.ptr, case.S, 3, da.ptr, db.ptr, dc_new.ptr, m, n, k, 80, 1,
                                                 stream.handle, stream.handle)
        assert rc == 0
        got_ref = dc_ref.download(np.zeros(size), stream)
        got_new = dc_new.download(np.zeros(size), stream)
        stream.sync()
        oracle.smm(case.stack, case.a, case.b, ref, m, n, k, b_rowmajor=False, threads=oracle.max_threads())
        assert oracle.block_relerr(got_new, got_ref, m * n) <= TOL, f"call {call}: noalloc vs libsmm_acc_process"
        assert oracle.block_relerr(got_new, ref, m * n) <= TOL, f"call {call}: noalloc vs oracle"
    # a stack that needs more scratch than the array holds is refused and leaves C untouched (the
    # device stack really holds that many valid entries, so even a wrong size check could not read
    # outside it)
    big = 2 * case.S
    while lib.libxstream_b200_process_scratch_bytes(big, m, n, k) <= lib.libxstream_b200_noalloc_scratch_bytes():
        big *= 2
    big_stack = np.ascontiguousarray(np.tile(case.stack, (big // case.S + 1, 1))[:big])
    ds_big = A.DevBuf.from_array(big_stack, stream)
    before = dc_new.download(np.zeros(size), stream)
    rc = lib.libxstream_b200_process_noalloc(None, ds_big.ptr, big, 3, da.ptr, db.ptr, dc_new.ptr, m, n, k, 80, 1,
                                             stream.handle, stream.handle)
    assert rc != 0
    ds_big.free()
    after = dc_new.download(np.zeros(size), stream)
    stream.sync()
    assert np.array_equal(before, after)
    lib.c_dbcsr_acc_clear_errors()
    for b in (da, db, ds, dc_ref, dc_new):
        b.free()
