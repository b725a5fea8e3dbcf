"""CPU tests of the oracle (the checker) against independent numpy restatements and invariants."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W


def numpy_smm(case: W.StackCase) -> np.ndarray:
    """Independent restatement with numpy matmul per entry (B column-major k x n)."""
    m, n, k = case.m, case.n, case.k
    c = np.zeros(case.nc * m * n)
    for a0, b0, c0 in case.stack:
        A = case.a[a0 - 1:a0 - 1 + m * k].reshape(k, m).T
        B = case.b[b0 - 1:b0 - 1 + k * n].reshape(n, k).T
        c[c0 - 1:c0 - 1 + m * n] += (A @ B).T.reshape(-1)
    return c


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 3, 5), (4, 4, 4), (5, 7, 3), (23, 23, 23), (13, 9, 26)])
def test_oracle_matches_numpy(shape):
    m, n, k = shape
    case = W.stack_case(m, n, k, 300, 20, 20, 7, seed=11)
    ref = numpy_smm(case)
    c = np.zeros(case.nc * m * n)
    oracle.smm(case.stack, case.a, case.b, c, m, n, k, b_rowmajor=False)
    assert oracle.block_relerr(c, ref, m * n) < 1e-14
    # the device layout (B transposed by libsmm_acc_transpose) gives bitwise the same result
    c2 = np.zeros_like(c)
    oracle.smm(case.stack, case.a, case.b_rowmajor(), c2, m, n, k, b_rowmajor=True)
    assert np.array_equal(c, c2)


def test_oracle_threads_bitwise_equal():
    case = W.stack_case(23, 23, 23, 5000, 200, 200, 64, seed=3)
    c1 = np.zeros(case.nc * 23 * 23)
    c2 = np.zeros_like(c1)
    oracle.smm(case.stack, case.a, case.b, c1, 23, 23, 23, b_rowmajor=False)
    oracle.smm(case.stack, case.a, case.b, c2, 23, 23, 23, b_rowmajor=False, threads=4)
    assert np.array_equal(c1, c2)


@pytest.mark.parametrize("shape", [(23, 23, 23), (5, 5, 5), (45, 45, 45), (9, 13, 7), (64, 3, 80)])
def test_timed_baseline_matches_checker(shape):
    """The timed CPU baseline (register-tiled, FMA) agrees with the exact checker to 1e-13."""
    m, n, k = shape
    case = W.stack_case(m, n, k, 2000, 80, 80, 30, seed=12)
    ref = np.zeros(case.nc * m * n)
    fast = np.zeros_like(ref)
    oracle.smm(case.stack, case.a, case.b, ref, m, n, k, b_rowmajor=False)
    oracle.smm_fast(case.stack, case.a, case.b, fast, m, n, k, threads=4)
    assert oracle.block_relerr(fast, ref, m * n) < 1e-13


@pytest.mark.parametrize("threads", [1, 3, 16, 64])
def test_timed_baseline_balanced_on_zipf_stack(threads):
    """The timed CPU baseline gives every thread the same number of entries even when one C block
    takes ~18% of the stack (config 1's Zipf(1.1) c); boundary-crossing segments stay correct."""
    case = W.config1()
    m, n, k = case.m, case.n, case.k
    assert oracle.fast_balance(case.S, threads) <= 1.1
    sub = case.stack[: 3 * 6000]  # a prefix keeps the exact checker quick
    ref = np.zeros(case.nc * m * n)
    fast = np.zeros_like(ref)
    oracle.smm(sub, case.a, case.b, ref, m, n, k, b_rowmajor=False)
    oracle.smm_fast(sub, case.a, case.b, fast, m, n, k, threads=threads)
    assert oracle.block_relerr(fast, ref, m * n) < 1e-13


def test_oracle_transpose_numpy():
    g = W.rng(5)
    m, n = 7, 5
    data = g.uniform(-1, 1, size=10 * m * n)
    trs = np.arange(10, dtype=np.int32) * (m * n)
    ref = data.reshape(10, n, m).transpose(0, 2, 1).copy().reshape(-1)  # m x n col-major -> n x m col-major
    out = oracle.transpose(trs, 0, data.copy(), m, n)
    assert np.array_equal(out, ref)


def test_oracle_norms():
    g = W.rng(6)
    mat = g.uniform(-1, 1, size=1000)
    offs = np.array([0, 100, 250, 999], dtype=np.int32)
    ne = np.array([100, 150, 1, 1], dtype=np.int32)
    out = oracle.norms(mat, offs, ne)
    ref = np.array([np.linalg.norm(mat[o:o + e]) for o, e in zip(offs, ne)], dtype=np.float32)
    np.testing.assert_allclose(out, ref, rtol=1e-6)


def test_block_relerr_metric():
    ref = np.array([1.0, -2.0, 0.5, 0.0, 0.0, 0.0])
    x = ref.copy()
    x[1] += 2e-13
    assert abs(oracle.block_relerr(x, ref, 3) - 1e-13) < 1e-16


def test_ozaki_digits_reconstruct_significand():
    """With 8 slices every aligned significand bit is covered: sum_s d_s * 2^low_s == aligned."""
    g = W.rng(7)
    x = W.spread_pool(g, 1, 6, 40)  # 6 rows of 40
    digits, emax = oracle.ozaki_slice(x, 6, 40, 40, 1, 8)
    lows = [oracle.lib().oracle_slice_low_bit(s) for s in range(8)]
    assert lows == [46, 39, 32, 25, 18, 11, 4, 0]
    for r in range(6):
        for kk in range(40):
            v = x[r * 40 + kk]
            recon = sum(int(digits[s, r, kk]) * (1 << lows[s]) for s in range(8))
            bits = np.float64(v).view(np.uint64)
            be = int((bits >> np.uint64(52)) & np.uint64(2047))
            mant = int(bits & np.uint64((1 << 52) - 1)) | (1 << 52)
            shift = int(emax[r]) - be
            aligned = mant >> shift if shift <= 52 else 0
            assert recon == (-aligned if v < 0 else aligned)
    assert np.abs(digits).max() <= 127


@pytest.mark.parametrize("nslices,bound", [(3, 1e-4), (5, 1e-8), (8, 1e-14)])
def test_ozaki_gemm_error_decreases(nslices, bound):
    g = W.rng(8)
    M, N, K = 16, 12, 20
    A = g.uniform(-1, 1, size=M * K)
    B = g.uniform(-1, 1, size=K * N)
    ref = (A.reshape(K, M).T @ B.reshape(N, K).T).T.reshape(-1)
    C = np.zeros(M * N)
    oracle.ozaki_gemm(A, B, C, M, N, K, nslices)
    err = np.abs(C - ref).max() / np.abs(ref).max()
    assert err < bound
