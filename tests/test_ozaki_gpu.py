"""GPU tests of the Ozaki scheme-1 FP64 GEMM on the int8 tensor cores (libxstream_b200_ozaki_gemm):
the device result against the CPU restatement of the same scheme (same digits, same slice pairs;
only the FP64 summation order differs: the oracle adds every slice pair in FP64, the device adds
exact int32 sums per anti-diagonal), and the error of the scheme against a plain FP64 GEMM
(numpy/BLAS) stated per slice count."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W

pytestmark = pytest.mark.gpu

SUM_ORDER_TOL = 1e-14  # device vs oracle: same products, different FP64 summation order


def relerr(x, ref):
    return float(np.max(np.abs(x - ref)) / max(np.max(np.abs(ref)), 1e-300))


def run(A, stream, transa, transb, M, N, K, a, b, c0, alpha=1.0, beta=1.0, nslices=8, trim=0):
    lda = a.shape[0]
    ldb = b.shape[0]
    da = A.DevBuf.from_array(np.asfortranarray(a).ravel(order="F"), stream)
    db = A.DevBuf.from_array(np.asfortranarray(b).ravel(order="F"), stream)
    dc = A.DevBuf.from_array(np.asfortranarray(c0).ravel(order="F"), stream)
    rc = A.ozaki_gemm(transa, transb, M, N, K, alpha, da, lda, db, ldb, beta, dc, M, nslices, trim, stream)
    assert rc == 0
    out = dc.download(np.zeros(M * N), stream)
    stream.sync()
    for buf in (da, db, dc):
        buf.free()
    return out.reshape((M, N), order="F")


def oracle_ref(a_op, b_op, c0, nslices, cutoff, alpha=1.0, beta=1.0):
    M, K = a_op.shape
    N = b_op.shape[1]
    acc = np.zeros(M * N)
    oracle.ozaki_gemm(np.asfortranarray(a_op).ravel(order="F"), np.asfortranarray(b_op).ravel(order="F"), acc, M, N, K,
                      nslices, cutoff)
    return beta * c0 + alpha * acc.reshape((M, N), order="F")


@pytest.mark.parametrize("shape", [(128, 256, 128), (200, 300, 130), (64, 40, 1000), (300, 260, 17)])
@pytest.mark.parametrize("nslices", [3, 5, 8])
def test_matches_oracle(acc, shape, nslices):
    A, stream = acc
    M, N, K = shape
    g = W.rng(1000 + M + nslices)
    a = g.uniform(-1, 1, size=(M, K))
    b = g.uniform(-1, 1, size=(K, N))
    c0 = g.uniform(-1, 1, size=(M, N))
    got = run(A, stream, "N", "N", M, N, K, a, b, c0, nslices=nslices)
    ref = oracle_ref(a, b, c0, nslices, 2 * (nslices - 1))
    assert relerr(got, ref) <= SUM_ORDER_TOL


@pytest.mark.parametrize("trans", ["NT", "TN", "TT"])
def test_transposes_and_alpha_beta(acc, trans):
    A, stream = acc
    M, N, K = 150, 270, 200
    g = W.rng(77)
    a_op = g.uniform(-1, 1, size=(M, K))
    b_op = g.uniform(-1, 1, size=(K, N))
    a = a_op.T.copy() if trans[0] == "T" else a_op
    b = b_op.T.copy() if trans[1] == "T" else b_op
    c0 = g.uniform(-1, 1, size=(M, N))
    got = run(A, stream, trans[0], trans[1], M, N, K, a, b, c0, alpha=-0.75, beta=0.5, nslices=6, trim=3)
    ref = oracle_ref(a_op, b_op, c0, 6, 2 * 5 - 3, alpha=-0.75, beta=0.5)
    assert relerr(got, ref) <= SUM_ORDER_TOL


def test_beta_zero_ignores_nan_c(acc):
    A, stream = acc
    M, N, K = 130, 257, 64
    g = W.rng(5)
    a = g.uniform(-1, 1, size=(M, K))
    b = g.uniform(-1, 1, size=(K, N))
    c0 = np.full((M, N), np.nan)
    got = run(A, stream, "N", "N", M, N, K, a, b, c0, beta=0.0)
    assert np.all(np.isfinite(got))
    assert relerr(got, a @ b) <= 1e-15


@pytest.mark.parametrize("nslices", [3, 4, 5, 6, 7, 8])
def test_error_per_slice_count(acc, nslices):
    """Error against FP64 (numpy/BLAS) shrinks by about 2^-7 per slice; 7 and 8 slices are at FP64
    level (<= 1e-13 relative max-norm), including rows scaled by 2^u, u in [-30, 30]."""
    A, stream = acc
    M = N = K = 512
    g = W.rng(2024)
    a = g.uniform(-1, 1, size=(M, K)) * np.ldexp(1.0, g.integers(-30, 31, size=(M, 1)))
    b = g.uniform(-1, 1, size=(K, N))
    ref = a @ b
    got = run(A, stream, "N", "N", M, N, K, a, b, np.zeros((M, N)), beta=0.0, nslices=nslices)
    # per-row relative error (rows carry their own scale)
    err = float(np.max(np.max(np.abs(got - ref), axis=1) / np.max(np.abs(ref), axis=1)))
    bound = {3: 1e-4, 4: 1e-6, 5: 1e-8, 6: 1e-10, 7: 1e-13, 8: 1e-13}[nslices]
    assert err <= bound, err


def test_long_k_runs_in_chunks(acc):
    """K above 16384 runs in several launches (the int32 sum of one diagonal stays exact)."""
    A, stream = acc
    M, N, K = 128, 256, 16384 + 300
    g = W.rng(9)
    a = g.uniform(-1, 1, size=(M, K))
    b = g.uniform(-1, 1, size=(K, N))
    c0 = g.uniform(-1, 1, size=(M, N))
    got = run(A, stream, "N", "N", M, N, K, a, b, c0, nslices=8)
    assert relerr(got, c0 + a @ b) <= 1e-14


@pytest.mark.parametrize("shape", [(128, 128, 16), (200, 300, 130), (129, 257, 1001), (64, 40, 7)])
def test_plain_dgemm_matches_fp64(acc, shape):
    """The plain FP64 DMMA GEMM (the comparison baseline) against numpy/BLAS FP64."""
    A, stream = acc
    M, N, K = shape
    g = W.rng(4242 + K)
    a = g.uniform(-1, 1, size=(M, K))
    b = g.uniform(-1, 1, size=(K, N))
    c0 = g.uniform(-1, 1, size=(M, N))
    da = A.DevBuf.from_array(a.ravel(order="F"), stream)
    db = A.DevBuf.from_array(b.ravel(order="F"), stream)
    dc = A.DevBuf.from_array(c0.ravel(order="F"), stream)
    assert A.dgemm(M, N, K, 0.5, da, M, db, K, -2.0, dc, M, stream) == 0
    got = dc.download(np.zeros(M * N), stream).reshape((M, N), order="F")
    stream.sync()
    assert relerr(got, 0.5 * (a @ b) - 2.0 * c0) <= 1e-14
    for buf in (da, db, dc):
        buf.free()


@pytest.mark.parametrize("shape,trans", [((4160, 4100, 200), "NN"), ((4097, 4200, 96), "TN")])
def test_read_modify_write_form_above_4096_squared(acc, shape, trans):
    """Products with M*N above 4096^2 run the 128 x 256 read-modify-write kernel form (the smaller ones
    keep the FP64 partial sum in tensor memory): its result against numpy/BLAS FP64 with alpha, beta
    and a ragged last tile in both directions."""
    A, stream = acc
    M, N, K = shape
    g = W.rng(77 + M)
    a_op = g.uniform(-1, 1, size=(M, K))
    b = g.uniform(-1, 1, size=(K, N))
    c0 = g.uniform(-1, 1, size=(M, N))
    a = a_op if "N" == trans[0] else np.asfortranarray(a_op.T)
    got = run(A, stream, trans[0], trans[1], M, N, K, a, b, c0, alpha=0.75, beta=-0.5, nslices=7, trim=6)
    assert relerr(got, 0.75 * (a_op @ b) - 0.5 * c0) <= 1e-13


@pytest.mark.parametrize("N", [4096, 4104])
def test_benchmark_size_against_numpy(acc, N):
    """Square sizes of the GEMM benchmark, s = 7 triangle, against numpy/BLAS FP64 (an oracle independent
    of the library's DMMA GEMM): 4096 runs the tensor-memory partial form, 4104 (just above 4096^2)
    the read-modify-write form."""
    A, stream = acc
    g = W.rng(N)
    a = g.uniform(-1, 1, size=(N, N))
    b = g.uniform(-1, 1, size=(N, N))
    got = run(A, stream, "N", "N", N, N, N, a, b, np.zeros((N, N)), beta=0.0, nslices=7, trim=6)
    assert relerr(got, a @ b) <= 1e-13
