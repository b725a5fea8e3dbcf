"""CPU tests that pin the oracle to the reference's own kernels: samples/smm/kernels/multiply.cl and
transpose.cl compiled as host C (oracle/ref_build.py) produced the committed golden fixtures
(tests/golden/make_golden.py), and -- where the reference tree is present -- are run live on further
shapes, kernel configurations and the 6-int parameter format."""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import ref_build as R

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden as G  # noqa: E402

META = json.loads((GOLDEN / "stack_path_reference.json").read_text())
DATA = np.load(GOLDEN / "stack_path_reference.npz")


@pytest.mark.parametrize("i", range(len(G.SMM_CASES)))
def test_oracle_matches_reference_kernel_fixture(i):
    case = G.smm_case(G.SMM_CASES[i])
    assert G.digest(case.stack, case.a, case.b) == META["smm"][i]["inputs_sha256"]  # same inputs as at generation
    got = np.zeros(case.nc * case.m * case.n)
    oracle.smm(case.stack, case.a, case.b, got, case.m, case.n, case.k, b_rowmajor=False)
    assert oracle.block_relerr(got, DATA[f"smm{i}_c"], case.m * case.n) <= 1e-14


@pytest.mark.parametrize("i", range(len(G.TRANSPOSE_CASES)))
def test_oracle_transpose_matches_reference_kernel_fixture(i):
    m, n, nblk, _ = G.TRANSPOSE_CASES[i]
    data, trs = G.transpose_input(G.TRANSPOSE_CASES[i])
    assert G.digest(data, trs) == META["transpose"][i]["inputs_sha256"]
    oracle.transpose(trs, 0, data, m, n)
    assert np.array_equal(data.view(np.uint64), DATA[f"tr{i}_out"].view(np.uint64))  # bit-exact, NaN payloads too


needs_reference = pytest.mark.skipif(not R.available(), reason="reference tree not present")


@needs_reference
@pytest.mark.parametrize("shape,cfg", [((23, 23, 23), {"bs": 16, "reg_b": True}), ((7, 80, 3), {"bs": 4}),
                                       ((80, 5, 80), {"bm": 8, "bn": 1, "bs": 8}), ((32, 32, 32), {"bm": 8, "bn": 4, "bs": 8}),
                                       ((9, 9, 9), {"bs": 1, "atomic_inc_nz": True})])
def test_live_reference_kernel_agrees_with_oracle(shape, cfg):
    from libxstream_b200 import workloads as W
    m, n, k = shape
    case = W.stack_case(m, n, k, 1200, 70, 70, 20, seed=sum(shape), values="spread")
    ref = np.zeros(case.nc * m * n)
    st = np.ascontiguousarray(case.stack, dtype=np.int32)
    bt = case.b_rowmajor()  # keep the array alive across the call
    R.multiply(m, n, k, **cfg)(st.ctypes.data, case.S, 0, case.a.ctypes.data, bt.ctypes.data, ref.ctypes.data)
    got = np.zeros_like(ref)
    oracle.smm(case.stack, case.a, case.b, got, m, n, k, b_rowmajor=False)
    assert oracle.block_relerr(got, ref, m * n) <= 1e-14


@needs_reference
def test_live_reference_kernel_dbm_format():
    """param_format != 0: 6-int records (m, n, k, a, b, c) with 0-based offsets (multiply.cl:96-99)."""
    from libxstream_b200 import workloads as W
    case = W.stack_case(13, 13, 13, 800, 40, 40, 10, seed=5)
    rec = np.empty((case.S, 6), dtype=np.int32)
    rec[:, :3] = 13
    rec[:, 3:] = case.stack - 1
    ref = np.zeros(case.nc * 169)
    bt = case.b_rowmajor()  # keep the array alive across the call
    R.multiply(13, 13, 13, bs=4)(rec.ctypes.data, case.S, 1, case.a.ctypes.data, bt.ctypes.data, ref.ctypes.data)
    got = np.zeros_like(ref)
    oracle.smm(case.stack, case.a, case.b, got, 13, 13, 13, b_rowmajor=False)
    assert oracle.block_relerr(got, ref, 169) <= 1e-14
