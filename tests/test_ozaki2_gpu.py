"""GPU tests of the Ozaki scheme-2 (Chinese remainder) FP64 GEMM on the int8 tensor cores
(libxstream_b200_ozaki2_gemm): the device result against the CPU restatement of the same scheme
(same integers, same moduli, exact CRT in Python integers; only the device's reconstruction, a
128-bit binary fraction times P, rounds), and the error of the scheme against a plain FP64 GEMM
(numpy/BLAS) per modulus count."""
from __future__ import annotations

import numpy as np
import pytest

from libxstream_b200 import workloads as W
from oracle import ozaki2 as O

pytestmark = pytest.mark.gpu

RECON_TOL = 4e-16  # device vs exact scheme, relative to the largest |C|: reconstruction rounding
FP64_TOL = 1e-14   # scheme with all 53 bits vs FP64 GEMM (numpy), relative max-norm


def relerr(x, ref):
    return float(np.max(np.abs(x - ref)) / max(np.max(np.abs(ref)), 1e-300))


def run(A, stream, transa, transb, M, N, K, a, b, c0, alpha=1.0, beta=0.0, nmod=0):
    """a, b: the stored matrices (op applied by the library); column-major upload."""
    da = A.DevBuf.from_array(np.asfortranarray(a).ravel(order="F"), stream)
    db = A.DevBuf.from_array(np.asfortranarray(b).ravel(order="F"), stream)
    dc = A.DevBuf.from_array(np.asfortranarray(c0).ravel(order="F"), stream)
    rc = A.ozaki2_gemm(transa, transb, M, N, K, alpha, da, a.shape[0], db, b.shape[0], beta, dc, M, nmod, stream)
    assert rc == 0
    out = dc.download(np.zeros(M * N), stream)
    stream.sync()
    for buf in (da, db, dc):
        buf.free()
    return out.reshape((M, N), order="F")


@pytest.mark.parametrize("shape", [(128, 256, 128), (100, 70, 300), (33, 260, 17)])
@pytest.mark.parametrize("nmod", [0, 12, 8])
def test_matches_exact_scheme(acc, shape, nmod):
    A, stream = acc
    M, N, K = shape
    g = W.rng(2000 + M + nmod)
    a = g.uniform(-1, 1, size=(M, K))
    b = g.uniform(-1, 1, size=(K, N))
    got = run(A, stream, "N", "N", M, N, K, a, b, np.zeros((M, N)), nmod=nmod)
    ref = O.ozaki2_gemm(a, b, nmod if nmod else O.default_moduli(K))
    assert relerr(got, ref) <= RECON_TOL
    err = relerr(got, a @ b)
    if 0 == nmod:
        assert err <= FP64_TOL
    else:  # fewer moduli: inputs keep mb bits, the error follows 2^-mb
        mb = O.mantissa_bits(nmod, K)
        assert err <= 2.0 ** (1 - mb) * 4 and err > 2.0 ** (-mb - 12)


@pytest.mark.parametrize("ta,tb", [("T", "N"), ("N", "T"), ("T", "T")])
def test_transposes_alpha_beta(acc, ta, tb):
    A, stream = acc
    M, N, K = 96, 130, 77
    g = W.rng(7)
    a_op = g.uniform(-1, 1, size=(M, K))
    b_op = g.uniform(-1, 1, size=(K, N))
    c0 = g.uniform(-1, 1, size=(M, N))
    a = a_op.T.copy() if ta == "T" else a_op
    b = b_op.T.copy() if tb == "T" else b_op
    got = run(A, stream, ta, tb, M, N, K, a, b, c0, alpha=2.5, beta=-0.5)
    assert relerr(got, 2.5 * (a_op @ b_op) - 0.5 * c0) <= FP64_TOL


def test_row_scaled_inputs(acc):
    """Rows of A scaled by 2^u, u in [-30, 30]: per-row scaling keeps every row at full precision."""
    A, stream = acc
    M, N, K = 200, 150, 256
    g = W.rng(8)
    a = g.uniform(-1, 1, size=(M, K)) * np.exp2(g.integers(-30, 31, size=(M, 1)))
    b = g.uniform(-1, 1, size=(K, N))
    got = run(A, stream, "N", "N", M, N, K, a, b, np.zeros((M, N)))
    ref = a @ b
    per_row = np.max(np.abs(got - ref), axis=1) / np.max(np.abs(ref), axis=1)
    assert float(per_row.max()) <= FP64_TOL


def test_long_k_runs_in_chunks(acc):
    """K = 40000 exceeds one launch's exact int32 range (32768): residues accumulate over chunks."""
    A, stream = acc
    M, N, K = 64, 96, 40000
    g = W.rng(9)
    a = g.uniform(-1, 1, size=(M, K))
    b = g.uniform(-1, 1, size=(K, N))
    got = run(A, stream, "N", "N", M, N, K, a, b, np.zeros((M, N)))
    assert relerr(got, a @ b) <= FP64_TOL


def test_long_k_ragged_rows_match_row_subset(acc):
    """K = 40000 (two launches accumulating residues) over three row tiles, the last one ragged:
    the first 128 rows of the 300-row product equal the 128-row product of the same rows bit for
    bit (each row keeps its own scaling, tiles do not interact)."""
    A, stream = acc
    M, N, K = 300, 100, 40000
    g = W.rng(14)
    a = g.uniform(-1, 1, size=(M, K))
    b = g.uniform(-1, 1, size=(K, N))
    tall = run(A, stream, "N", "N", M, N, K, a, b, np.zeros((M, N)))
    short = run(A, stream, "N", "N", 128, N, K, np.ascontiguousarray(a[:128]), b, np.zeros((128, N)))
    assert relerr(tall, a @ b) <= FP64_TOL
    assert np.array_equal(tall[:128], short)


def test_zero_rows_and_special_sizes(acc):
    A, stream = acc
    M, N, K = 130, 257, 33
    g = W.rng(10)
    a = g.uniform(-1, 1, size=(M, K))
    a[5] = 0.0
    b = g.uniform(-1, 1, size=(K, N))
    b[:, 7] = 0.0
    got = run(A, stream, "N", "N", M, N, K, a, b, np.zeros((M, N)))
    assert relerr(got, a @ b) <= FP64_TOL
    assert not np.any(got[5]) and not np.any(got[:, 7])


def test_large_square(acc):
    A, stream = acc
    N = 1024
    g = W.rng(11)
    a = g.uniform(-1, 1, size=(N, N))
    b = g.uniform(-1, 1, size=(N, N))
    got = run(A, stream, "N", "N", N, N, N, a, b, np.zeros((N, N)))
    assert relerr(got, a @ b) <= FP64_TOL


def test_near_cancellation(acc):
    """Outputs many orders of magnitude below |A| |B| (pairs of products that nearly cancel): the
    reconstruction keeps its double-double precision whatever the sign of the small result."""
    A, stream = acc
    M, N, K = 64, 256, 64
    g = W.rng(12)
    a = g.uniform(-1, 1, size=(M, K))
    a[:, 1::2] = a[:, 0::2]
    b = g.uniform(-1, 1, size=(K, N))
    b[1::2] = -b[0::2] * (1.0 + g.uniform(-1e-6, 1e-6, size=(K // 2, N)))
    got = run(A, stream, "N", "N", M, N, K, a, b, np.zeros((M, N)))
    ref = O.ozaki2_gemm(a, b, O.default_moduli(K))
    assert np.max(np.abs(ref)) < 1e-4
    assert relerr(got, ref) <= RECON_TOL


def test_benchmark_size_against_numpy(acc):
    """N = 4096, the smallest square of the GEMM benchmark above 2048, uniform and row-scaled (2^u,
    u in [-30, 30]) inputs, against numpy/BLAS FP64 (an oracle independent of the library's DMMA GEMM)."""
    A, stream = acc
    N = 4096
    g = W.rng(4096)
    a = g.uniform(-1, 1, size=(N, N))
    b = g.uniform(-1, 1, size=(N, N))
    got = run(A, stream, "N", "N", N, N, N, a, b, np.zeros((N, N)))
    assert relerr(got, a @ b) <= FP64_TOL
    a_rs = a * np.exp2(g.integers(-30, 31, size=N))[:, None]
    got = run(A, stream, "N", "N", N, N, N, a_rs, b, np.zeros((N, N)))
    ref = a_rs @ b
    assert float(np.max(np.max(np.abs(got - ref), axis=1) / np.max(np.abs(ref), axis=1))) <= FP64_TOL
