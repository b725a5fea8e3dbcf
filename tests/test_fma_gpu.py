"""GPU parity of the register-blocked FMA stack kernel (parameter kp = -1) against the CPU oracle,
through libsmm_acc_process. It holds C as per-lane register blocks and issues plain FP64 FMAs (no
padded DMMA tiles), with the same chunks, segments and in-kernel combine as the DMMA kernels, so the
bar is the same: relative max-norm error per C block <= 1e-13, and bitwise reproducible results.
Reference: the work-item loop the FMA kernel replaces, samples/smm/kernels/multiply.cl:314-323."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W
from test_smm_gpu import oracle_c, run_device

pytestmark = pytest.mark.gpu

TOL = 1e-13
FMA = -1  # kp value that selects the FMA kernel

# shapes compiled with their own lane grid, and shapes served by the runtime-shape classes
COMPILED = [(4, 4, 4), (5, 5, 5), (6, 6, 18), (13, 4, 16), (32, 9, 9), (16, 64, 9), (7, 10, 5)]
RUNTIME = [(1, 1, 1), (2, 3, 5), (8, 8, 8), (9, 9, 9), (13, 13, 13), (16, 16, 16), (22, 22, 22), (23, 23, 23),
           (26, 26, 26), (32, 32, 32), (7, 45, 13), (3, 17, 80), (16, 50, 1)]


def forced(A, m, n, k, chunk=0):
    A.set_params(m, n, k, chunk, 1, 1, FMA, 4)


@pytest.mark.parametrize("shape", COMPILED + RUNTIME, ids=[f"{m}x{n}x{k}" for m, n, k in COMPILED + RUNTIME])
def test_fma_parity(acc, shape):
    A, stream = acc
    m, n, k = shape
    case = W.stack_case(m, n, k, 1500, 97, 89, 31, seed=m * 10000 + n * 100 + k)
    c0 = W.rng(2).uniform(-1, 1, size=case.nc * m * n)  # C accumulates onto existing content
    forced(A, m, n, k)
    try:
        got = run_device(A, stream, case, c0=c0)
    finally:
        A.lib().libxstream_b200_clear_params()
    assert oracle.block_relerr(got, oracle_c(case, c0=c0), m * n) <= TOL


@pytest.mark.parametrize("shape", [(4, 4, 4), (32, 9, 9), (6, 6, 18), (16, 64, 9)], ids=lambda s: "x".join(map(str, s)))
def test_fma_large_stack(acc, shape):
    """10^5 entries over 2048 C blocks with a skewed c distribution: hot segments span many CTAs, so
    the two-level in-kernel combine runs."""
    A, stream = acc
    m, n, k = shape
    S = 100000
    na, nb, nc = W.pool_sizes(S)
    case = W.stack_case(m, n, k, S, na, nb, nc, seed=21)
    forced(A, m, n, k)
    try:
        got = run_device(A, stream, case)
        again = run_device(A, stream, case)
    finally:
        A.lib().libxstream_b200_clear_params()
    assert oracle.block_relerr(got, oracle_c(case), m * n) <= TOL
    assert np.array_equal(got, again)  # bitwise reproducible


@pytest.mark.parametrize("chunk", [1, 3, 64])
def test_fma_chunk_lengths(acc, chunk):
    """Chunks of 1 and 3 entries put segment boundaries at every chunk and CTA boundary."""
    A, stream = acc
    case = W.stack_case(13, 4, 16, 3000, 200, 200, 40, seed=chunk)
    forced(A, 13, 4, 16, chunk)
    try:
        got = run_device(A, stream, case)
    finally:
        A.lib().libxstream_b200_clear_params()
    assert oracle.block_relerr(got, oracle_c(case), 13 * 4) <= TOL


def test_fma_single_hot_block(acc):
    A, stream = acc
    case = W.stack_case(5, 5, 5, 20000, 300, 300, 1, seed=4)
    forced(A, 5, 5, 5)
    try:
        got = run_device(A, stream, case)
    finally:
        A.lib().libxstream_b200_clear_params()
    assert oracle.block_relerr(got, oracle_c(case), 25) <= TOL


def test_fma_unsupported_shape_reports_error(acc):
    """A block whose C does not fit any FMA lane grid (m > 32) is refused with an error, not run."""
    A, stream = acc
    case = W.stack_case(45, 45, 45, 100, 10, 10, 5, seed=1)
    forced(A, 45, 45, 45)
    try:
        da = A.DevBuf.from_array(case.a, stream)
        db = A.DevBuf.from_array(case.b_rowmajor(), stream)
        dc = A.DevBuf(case.nc * 45 * 45 * 8)
        dc.zero(stream)
        ds = A.DevBuf.from_array(case.stack, stream)
        rc = A.process(ds, case.S, da, db, dc, 45, 45, 45, stream)
        stream.sync()
    finally:
        A.lib().libxstream_b200_clear_params()
        A.lib().c_dbcsr_acc_clear_errors()
    assert rc != 0
    for b in (da, db, dc, ds):
        b.free()
