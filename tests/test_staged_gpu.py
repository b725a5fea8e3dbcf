"""GPU parity of the staged stack kernel (kp = 0: A/B blocks brought into a per-warp shared-memory
ring by bulk copies, the whole C block as one warp tile) against the CPU oracle and the register
kernel. Tolerance: relative max-norm error per C block <= 1e-13 (FP64)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W
from test_smm_gpu import TOL, oracle_c, run_device

pytestmark = pytest.mark.gpu

STAGED = [4, 8, 9, 13, 16, 22, 23, 26, 32]  # square shapes (32: the register kernel runs)
STAGED3 = [(23, 22, 13), (22, 22, 23), (32, 9, 9), (13, 4, 16), (16, 26, 5), (26, 23, 26),
           (22, 32, 32)]  # non-square shapes with a staged kernel


def _run_with(A, stream, case, chunk, kp, wpb=4, c0=None):
    m, n = case.m, case.n
    A.set_params(case.m, case.n, case.k, chunk, (m + 7) // 8, (n + 7) // 8, kp, wpb)
    try:
        return run_device(A, stream, case, c0=c0)
    finally:
        A.lib().libxstream_b200_clear_params()


@pytest.mark.parametrize("s", STAGED)
@pytest.mark.parametrize("chunk", [0, 1, 7, 40, 100])
def test_staged_parity(acc, s, chunk):
    """Chunks of 1 (every segment crosses), 7, 40 and 100 (entry windows of 32 roll over) and the
    one-wave default; C accumulates onto existing content."""
    A, stream = acc
    case = W.stack_case(s, s, s, 3000, 201, 199, 37, seed=1000 * s + chunk)
    c0 = W.rng(s).uniform(-1, 1, size=case.nc * s * s)
    got = _run_with(A, stream, case, chunk, 0, c0=c0)
    assert oracle.block_relerr(got, oracle_c(case, c0=c0), s * s) <= TOL


@pytest.mark.parametrize("wpb", [1, 2, 3])
def test_staged_warps_per_cta(acc, wpb):
    A, stream = acc
    case = W.stack_case(23, 23, 23, 5000, 301, 300, 60, seed=wpb)
    got = _run_with(A, stream, case, 0, 0, wpb=wpb)
    assert oracle.block_relerr(got, oracle_c(case), 529) <= TOL


def test_staged_single_hot_block(acc):
    """One segment spans every chunk and every CTA."""
    A, stream = acc
    case = W.stack_case(23, 23, 23, 20000, 301, 299, 1, seed=4)
    assert oracle.block_relerr(_run_with(A, stream, case, 0, 0), oracle_c(case), 529) <= TOL


def test_staged_config1_matches_register_kernel(acc):
    """The 23x23x23 workload (30000 triples, Zipf(1.1) c): staged and register kernels agree with the
    oracle, and the staged kernel is bitwise reproducible."""
    A, stream = acc
    case = W.config1()
    ref = oracle_c(case)
    staged = _run_with(A, stream, case, 0, 0)
    again = _run_with(A, stream, case, 0, 0)
    reg = _run_with(A, stream, case, 0, 2)
    assert oracle.block_relerr(staged, ref, 529) <= TOL
    assert oracle.block_relerr(reg, ref, 529) <= TOL
    assert np.array_equal(staged, again)


def test_staged_single_entry(acc):
    A, stream = acc
    case = W.stack_case(16, 16, 16, 1, 3, 3, 1, seed=6)
    assert oracle.block_relerr(_run_with(A, stream, case, 0, 0), oracle_c(case), 256) <= TOL


@pytest.mark.parametrize("shape", STAGED3, ids=[f"{m}x{n}x{k}" for m, n, k in STAGED3])
@pytest.mark.parametrize("chunk", [0, 1, 40])
def test_staged_nonsquare_parity(acc, shape, chunk):
    A, stream = acc
    m, n, k = shape
    case = W.stack_case(m, n, k, 3000, 211, 197, 41, seed=m * 1000 + n * 10 + k + chunk)
    c0 = W.rng(k).uniform(-1, 1, size=case.nc * m * n)
    got = _run_with(A, stream, case, chunk, 0, c0=c0)
    assert oracle.block_relerr(got, oracle_c(case, c0=c0), m * n) <= TOL


def test_staged_wide_tile_parity(acc):
    """16x64x9: the staged kernel with a warp tile of 2 x 8 fragments (wider than the register kernels
    take), chosen by the untuned parameter lookup; C accumulates onto existing content."""
    A, stream = acc
    A.lib().libxstream_b200_clear_params()
    p = A.get_params(16, 64, 9, 30000)
    assert (p["mt"], p["nt"], p["kp"]) == (2, 8, 0)
    case = W.stack_case(16, 64, 9, 30000, 800, 800, 300, seed=1664)
    c0 = W.rng(9).uniform(-1, 1, size=case.nc * 16 * 64)
    got = run_device(A, stream, case, c0=c0)
    assert oracle.block_relerr(got, oracle_c(case, c0=c0), 16 * 64) <= TOL
