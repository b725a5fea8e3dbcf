"""GPU tests of the Ozaki scheme-1 stack form (libxstream_b200_process_ozaki): per-block row/column
scaled int8 slices, slice products on the tensor cores, FP64 recombination. Compared with the CPU
restatement of the same scheme (oracle.ozaki_smm: same digits and pairs, FP64 sums in another
order) and with the plain FP64 oracle (error per slice count), on uniform and exponent-spread
(mantissa U[1,2) x 2^e, e in [-20, 20]) inputs."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W

pytestmark = pytest.mark.gpu

SCHEME_TOL = 1e-14  # device vs the oracle of the same scheme (summation order only)


def run_oz(A, stream, case: W.StackCase, nslices: int, trim: int = 0, c0=None):
    size = case.nc * case.m * case.n
    c0 = np.zeros(size) if c0 is None else c0
    da = A.DevBuf.from_array(case.a, stream)
    db = A.DevBuf.from_array(case.b_rowmajor(), stream)
    ds = A.DevBuf.from_array(case.stack, stream)
    dc = A.DevBuf.from_array(c0, stream)
    rc = A.process_ozaki(ds, case.S, case.m, case.n, case.k, da, case.na, db, case.nb, dc, nslices, trim, stream)
    out = dc.download(np.zeros(size), stream)
    stream.sync()
    for buf in (da, db, ds, dc):
        buf.free()
    return rc, out


def scheme_ref(case, nslices, cutoff, c0=None):
    ref = np.zeros(case.nc * case.m * case.n) if c0 is None else c0.copy()
    oracle.ozaki_smm(case.stack, case.a, case.b_rowmajor(), ref, case.m, case.n, case.k, nslices, cutoff)
    return ref


def plain_ref(case, c0=None):
    ref = np.zeros(case.nc * case.m * case.n) if c0 is None else c0.copy()
    oracle.smm(case.stack, case.a, case.b, ref, case.m, case.n, case.k, b_rowmajor=False, threads=oracle.max_threads())
    return ref


@pytest.mark.parametrize("shape", [(32, 32, 32), (45, 45, 45), (64, 64, 64), (23, 23, 23), (5, 13, 40), (64, 17, 33),
                                   (1, 1, 1), (64, 64, 7)])
def test_matches_scheme_oracle(acc, shape):
    A, stream = acc
    m, n, k = shape
    S = 400 if m * n * k > 30000 else 1500
    case = W.stack_case(m, n, k, S, 60, 60, 12, seed=900 + m + n + k, values="spread")
    c0 = W.rng(3).uniform(-1, 1, size=case.nc * m * n)
    rc, got = run_oz(A, stream, case, 7, trim=6, c0=c0)
    assert rc == 0
    ref = scheme_ref(case, 7, 6, c0)
    assert oracle.block_relerr(got, ref, m * n) <= SCHEME_TOL


@pytest.mark.parametrize("nslices,trim,bound", [(3, 2, 1e-4), (5, 4, 1e-8), (6, 5, 1e-10), (7, 6, 1e-13), (8, 0, 1e-14)])
def test_error_per_slice_count(acc, nslices, trim, bound):
    A, stream = acc
    case = W.stack_case(32, 32, 32, 3000, 200, 200, 40, seed=77, values="spread")
    rc, got = run_oz(A, stream, case, nslices, trim)
    assert rc == 0
    assert oracle.block_relerr(got, plain_ref(case), 32 * 32) <= bound


def test_hot_block_and_chunk_crossing(acc):
    """Zipf-hot C blocks: segments of ~25k entries cross chunk boundaries and are combined from
    pieces; the 8-slice scheme stays within 1e-13 of FP64 over such long sums."""
    A, stream = acc
    case = W.stack_case(16, 16, 16, 40000, 500, 500, 8, seed=4, zipf_s=2.0)
    rc, got = run_oz(A, stream, case, 8, 0)
    assert rc == 0
    assert oracle.block_relerr(got, plain_ref(case), 256) <= 1e-13


def test_deterministic(acc):
    A, stream = acc
    case = W.stack_case(45, 45, 45, 5000, 300, 300, 50, seed=12, values="spread")
    _, x = run_oz(A, stream, case, 7, 6)
    _, y = run_oz(A, stream, case, 7, 6)
    assert np.array_equal(x, y)


def test_unsuitable_shapes_and_empty(acc):
    A, stream = acc
    case = W.stack_case(65, 8, 8, 10, 4, 4, 2, seed=1)
    rc, got = run_oz(A, stream, case, 7)
    assert rc == -1 and not np.any(got)
    case = W.stack_case(8, 8, 8, 10, 4, 4, 2, seed=1)
    da = A.DevBuf.from_array(case.a, stream)
    assert A.process_ozaki(da, 0, 8, 8, 8, da, 4, da, 4, da, 7, 0, stream) == 0
    da.free()
