"""GPU parity against the golden fixtures produced by the reference's own kernels
(tests/golden/make_golden.py): the stack path (single calls and one batch call of all cases) within
1e-13 relative max-norm per C block, the transpose bit-exact (NaN payloads included)."""
from __future__ import annotations

import ctypes
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from libxstream_b200 import StackDesc

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu
DATA = np.load(GOLDEN / "stack_path_reference.npz")
TOL = 1e-13


@pytest.mark.parametrize("i", range(len(G.SMM_CASES)))
def test_stack_path_matches_reference_fixture(acc, i):
    A, stream = acc
    case = G.smm_case(G.SMM_CASES[i])
    da, db = A.DevBuf.from_array(case.a, stream), A.DevBuf.from_array(case.b_rowmajor(), stream)
    ds, dc = A.DevBuf.from_array(case.stack, stream), A.DevBuf(case.nc * case.m * case.n * 8)
    dc.zero(stream)
    assert A.process(ds, case.S, da, db, dc, case.m, case.n, case.k, stream) == 0
    got = dc.download(np.zeros(case.nc * case.m * case.n), stream)
    stream.sync()
    assert oracle.block_relerr(got, DATA[f"smm{i}_c"], case.m * case.n) <= TOL
    for b in (da, db, ds, dc):
        b.free()


def test_batch_matches_reference_fixtures(acc):
    A, stream = acc
    keep, descs, cs = [], [], []
    for spec in G.SMM_CASES:
        case = G.smm_case(spec)
        da, db = A.DevBuf.from_array(case.a, stream), A.DevBuf.from_array(case.b_rowmajor(), stream)
        ds, dc = A.DevBuf.from_array(case.stack, stream), A.DevBuf(case.nc * case.m * case.n * 8)
        dc.zero(stream)
        keep.append((da, db, ds, dc))
        cs.append(case)
        descs.append(StackDesc(ds.ptr, case.S, case.m, case.n, case.k, da.ptr, db.ptr, dc.ptr))
    arr = (StackDesc * len(descs))(*descs)
    assert A.lib().libxstream_b200_process_batch(ctypes.cast(arr, ctypes.c_void_p), len(descs), 80, stream.handle) == 0
    for i, (case, bufs) in enumerate(zip(cs, keep)):
        got = bufs[3].download(np.zeros(case.nc * case.m * case.n), stream)
        stream.sync()
        assert oracle.block_relerr(got, DATA[f"smm{i}_c"], case.m * case.n) <= TOL
        for b in bufs:
            b.free()


@pytest.mark.parametrize("i", range(len(G.TRANSPOSE_CASES)))
def test_transpose_matches_reference_fixture(acc, i):
    A, stream = acc
    m, n, nblk, _ = G.TRANSPOSE_CASES[i]
    data, trs = G.transpose_input(G.TRANSPOSE_CASES[i])
    dd, dt = A.DevBuf.from_array(data, stream), A.DevBuf.from_array(trs, stream)
    assert A.transpose(dt, 0, nblk, dd, m, n, stream) == 0
    got = dd.download(np.zeros_like(data), stream)
    stream.sync()
    assert np.array_equal(got.view(np.uint64), DATA[f"tr{i}_out"].view(np.uint64))
    dd.free()
    dt.free()
