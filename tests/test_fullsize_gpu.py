"""Full-size GPU parity of the workloads the benchmark measures, each against the CPU oracle.

- Config 2 (mixed-shape batch): 12 FP64 stacks with (m, n, k) from {4,5,9,13,16,22,23,26,32,45,64}^3,
  entries U[-1,1], c Zipf(1.1); both the stated log-uniform 100..200000 sizes and the same 12 stacks
  scaled to 2.0M triples, through libxstream_b200_process_batch captured once into a CUDA graph and
  replayed; relative max-norm error per C block <= 1e-13.
- Config 2 (transposes): 100000 square blocks of 5..64 (one libsmm_acc_transpose call per size),
  bit for bit against numpy, NaN payloads included.
- Config 3 (Ozaki int8 stack form): 200000 triples of 32^3, 45^3 and 64^3 blocks, entries mantissa
  U[1,2) x 2^e, e uniform in [-20, 20], random sign; s = 7 (triangle of pairs) and s = 8 (all pairs);
  relative max-norm error per C block <= 1e-13 against the FP64 oracle.
The device-vs-host check at full size mirrors the reference's own (samples/smm/acc_bench.c:397-419).
The oracle here is its balanced multi-threaded restatement (oracle_smm_f64_fast), which agrees with
the exact sequential checker to 1e-13 (tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from libxstream_b200 import StackDesc
from libxstream_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _cpu(case: W.StackCase, c0: np.ndarray | None = None) -> np.ndarray:
    ref = np.zeros(case.nc * case.m * case.n) if c0 is None else c0.copy()
    oracle.smm_fast(case.stack, case.a, case.b, ref, case.m, case.n, case.k, threads=oracle.max_threads())
    return ref


@pytest.mark.parametrize("workload", ["stated", "scaled2m"])
def test_config2_mixed_batch_graph(acc, workload):
    """12 mixed-shape stacks in one batch call, captured as a CUDA graph and replayed twice (C
    accumulates: the result must equal two oracle passes)."""
    A, stream = acc
    L = A.lib()
    cases = W.mixed_shapes() if workload == "stated" else W.mixed_shapes_scaled()
    if workload == "scaled2m":
        assert 1_900_000 <= sum(c.S for c in cases) <= 2_100_000
    bufs, descs = [], []
    for c in cases:
        da, db = A.DevBuf.from_array(c.a, stream), A.DevBuf.from_array(c.b_rowmajor(), stream)
        ds, dc = A.DevBuf.from_array(c.stack, stream), A.DevBuf(c.nc * c.m * c.n * 8)
        dc.zero(stream)
        bufs.append((da, db, ds, dc))
        descs.append(StackDesc(ds.ptr, c.S, c.m, c.n, c.k, da.ptr, db.ptr, dc.ptr))
    arr = (StackDesc * len(descs))(*descs)
    stream.sync()
    gexec, nk = ctypes.c_void_p(), ctypes.c_int(0)
    assert L.libxstream_b200_graph_begin(stream.handle) == 0
    rc = L.libxstream_b200_process_batch(ctypes.cast(arr, ctypes.c_void_p), len(descs), 80, stream.handle)
    assert L.libxstream_b200_graph_end(stream.handle, ctypes.byref(gexec), ctypes.byref(nk)) == 0
    assert rc == 0 and nk.value >= 1
    for _ in range(2):
        assert L.libxstream_b200_graph_launch(gexec, stream.handle) == 0
    stream.sync()
    assert L.libxstream_b200_graph_destroy(gexec) == 0
    worst = 0.0
    for c, (da, db, ds, dc) in zip(cases, bufs):
        got = dc.download(np.zeros(c.nc * c.m * c.n), stream)
        stream.sync()
        ref = _cpu(c)
        ref = _cpu(c, ref)
        err = oracle.block_relerr(got, ref, c.m * c.n)
        worst = max(worst, err)
        assert err <= TOL, (c.m, c.n, c.k, c.S, err)
        for b in (da, db, ds, dc):
            b.free()
    assert worst <= TOL


def test_config2_transposes_100k_blocks(acc):
    """100000 square blocks of 5..64 (uniform sizes), one libsmm_acc_transpose per size: bit-exact."""
    A, stream = acc
    tw = W.transpose_workload()
    assert sum(tw.values()) == 100000
    g = W.rng(4242)
    for size, count in tw.items():
        data = g.uniform(-1, 1, size=count * size * size)
        bits = data.view(np.uint64)
        bits[:: 97] = np.uint64(0x7FF8000000000000) | (np.arange(bits[:: 97].size, dtype=np.uint64) + np.uint64(1))
        dd = A.DevBuf.from_array(data, stream)
        trs = A.DevBuf.from_array(np.arange(count, dtype=np.int32) * (size * size), stream)
        assert A.transpose(trs, 0, count, dd, size, size, stream) == 0
        got = dd.download(np.zeros(data.size), stream)
        stream.sync()
        want = data.reshape(count, size, size).transpose(0, 2, 1).reshape(-1)
        assert np.array_equal(got.view(np.uint64), np.ascontiguousarray(want).view(np.uint64)), size
        dd.free()
        trs.free()


@pytest.mark.parametrize("size", [32, 45, 64])
def test_config3_ozaki_stacks_200k(acc, size):
    """Ozaki int8 stack form at full size: 200000 triples, A/B pools of 8192 blocks, C pool of 2048
    blocks, exponent-spread entries; s = 7 triangle and s = 8 all pairs within 1e-13 of FP64."""
    A, stream = acc
    m = n = k = size
    S = 200000
    case = W.stack_case(m, n, k, S, 8192, 8192, 2048, seed=25071975 + size, values="spread")
    ref = _cpu(case)
    da, db = A.DevBuf.from_array(case.a, stream), A.DevBuf.from_array(case.b_rowmajor(), stream)
    ds = A.DevBuf.from_array(case.stack, stream)
    dc = A.DevBuf(case.nc * m * n * 8)
    errs = {}
    for ns, trim in ((7, 6), (8, 0)):
        dc.zero(stream)
        assert A.process_ozaki(ds, S, m, n, k, da, case.na, db, case.nb, dc, ns, trim, stream) == 0
        got = dc.download(np.zeros(case.nc * m * n), stream)
        stream.sync()
        errs[(ns, trim)] = oracle.block_relerr(got, ref, m * n)
    for b in (da, db, ds, dc):
        b.free()
    assert all(e <= TOL for e in errs.values()), errs
