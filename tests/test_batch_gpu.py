"""GPU parity tests of the batched stack path (libxstream_b200_process_batch): all stacks of one
multiplication in one call -- one grouping pass, then one persistent kernel that runs every stack's
work items and combines their CTA-crossing segments itself -- against the CPU oracle (relative
max-norm error per C block <= 1e-13), with CUDA-graph capture/replay."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from libxstream_b200 import StackDesc
from libxstream_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-13


class DevCase:
    """Device copies of one StackCase (B uploaded already transposed) and its C pool."""

    def __init__(self, A, stream, case: W.StackCase, c0: np.ndarray | None = None):
        self.case = case
        self.size = case.nc * case.m * case.n
        self.a = A.DevBuf.from_array(case.a, stream)
        self.b = A.DevBuf.from_array(case.b_rowmajor(), stream)
        self.s = A.DevBuf.from_array(case.stack, stream)
        self.c0 = np.zeros(self.size) if c0 is None else c0
        self.c = A.DevBuf.from_array(self.c0, stream)

    def desc(self) -> StackDesc:
        c = self.case
        return StackDesc(self.s.ptr, c.S, c.m, c.n, c.k, self.a.ptr, self.b.ptr, self.c.ptr)

    def result(self, stream) -> np.ndarray:
        out = self.c.download(np.zeros(self.size), stream)
        stream.sync()
        return out

    def reference(self, times: int = 1) -> np.ndarray:
        ref = self.c0.copy()
        for _ in range(times):
            oracle.smm(self.case.stack, self.case.a, self.case.b, ref, self.case.m, self.case.n, self.case.k,
                       b_rowmajor=False, threads=oracle.max_threads())
        return ref

    def free(self):
        for buf in (self.a, self.b, self.s, self.c):
            buf.free()


def run_batch(A, stream, devs, max_kernel_dim=80) -> int:
    arr = (StackDesc * len(devs))(*[d.desc() for d in devs])
    return A.lib().libxstream_b200_process_batch(ctypes.cast(arr, ctypes.c_void_p), len(devs), max_kernel_dim,
                                                 stream.handle)


def mixed_cases(seed: int, nstacks: int, smax: int):
    return W.mixed_shapes(seed=seed, nstacks=nstacks, smin=100, smax=smax)


def test_mixed_shapes_batch(acc):
    A, stream = acc
    cases = mixed_cases(101, 12, 20000)
    devs = [DevCase(A, stream, c, c0=W.rng(i).uniform(-1, 1, size=c.nc * c.m * c.n)) for i, c in enumerate(cases)]
    assert run_batch(A, stream, devs) == 0
    for d in devs:
        got = d.result(stream)
        assert oracle.block_relerr(got, d.reference(), d.case.m * d.case.n) <= TOL, (d.case.m, d.case.n, d.case.k)
        d.free()


def test_batch_deterministic_and_graph_replay(acc):
    A, stream = acc
    lib = A.lib()
    cases = mixed_cases(202, 6, 30000)
    devs = [DevCase(A, stream, c) for c in cases]
    assert run_batch(A, stream, devs) == 0
    first = [d.result(stream) for d in devs]
    for d in devs:
        d.c.zero(stream)
    assert run_batch(A, stream, devs) == 0
    second = [d.result(stream) for d in devs]
    for x, y in zip(first, second):
        assert np.array_equal(x, y)
    # capture one batch call into a CUDA graph and replay it twice: C receives the stacks twice
    for d in devs:
        d.c.zero(stream)
    stream.sync()
    gexec, nk = ctypes.c_void_p(), ctypes.c_int(0)
    assert lib.libxstream_b200_graph_begin(stream.handle) == 0
    rc = run_batch(A, stream, devs)
    assert lib.libxstream_b200_graph_end(stream.handle, ctypes.byref(gexec), ctypes.byref(nk)) == 0
    assert rc == 0 and nk.value == 2  # one grouping launch + the persistent kernel: no combine launch
    for _ in range(2):
        assert lib.libxstream_b200_graph_launch(gexec, stream.handle) == 0
    stream.sync()
    assert lib.libxstream_b200_graph_destroy(gexec) == 0
    for d in devs:
        assert oracle.block_relerr(d.result(stream), d.reference(times=2), d.case.m * d.case.n) <= TOL
        d.free()


def test_batch_shared_c_pool(acc):
    """Stacks with the same (m, n) and different k update the same C blocks (as DBCSR's stacks of one
    multiplication do): contributions add up correctly."""
    A, stream = acc
    m = n = 13
    nc = 40
    c0 = np.zeros(nc * m * n)
    cases = [W.stack_case(m, n, k, 3000, 60, 60, nc, seed=300 + k) for k in (5, 13, 22, 64)]
    dc = A.DevBuf.from_array(c0, stream)
    keep = []
    arr = (StackDesc * len(cases))()
    for i, c in enumerate(cases):
        da, db, ds = (A.DevBuf.from_array(c.a, stream), A.DevBuf.from_array(c.b_rowmajor(), stream),
                      A.DevBuf.from_array(c.stack, stream))
        keep += [da, db, ds]
        arr[i] = StackDesc(ds.ptr, c.S, m, n, c.k, da.ptr, db.ptr, dc.ptr)
    assert A.lib().libxstream_b200_process_batch(ctypes.cast(arr, ctypes.c_void_p), len(cases), 80, stream.handle) == 0
    got = dc.download(np.zeros_like(c0), stream)
    stream.sync()
    ref = c0.copy()
    for c in cases:
        oracle.smm(c.stack, c.a, c.b, ref, m, n, c.k, b_rowmajor=False)
    assert oracle.block_relerr(got, ref, m * n) <= TOL
    for b in keep + [dc]:
        b.free()


def test_batch_needs_several_grouping_launches(acc):
    """More entries than one cooperative grouping launch holds (148 tiles of 4096): the grouping runs
    in several launches into one sorted array, the stack kernel still runs once."""
    A, stream = acc
    cases = [W.stack_case(4, 4, 4, 260000, 4096, 4096, 2048, seed=400 + i) for i in range(3)]
    devs = [DevCase(A, stream, c) for c in cases]
    assert run_batch(A, stream, devs) == 0
    for d in devs:
        assert oracle.block_relerr(d.result(stream), d.reference(), 16) <= TOL
        d.free()


def test_single_stack_larger_than_one_grouping_launch(acc):
    A, stream = acc
    case = W.stack_case(5, 5, 5, 700000, 5000, 5000, 3000, seed=500)
    d = DevCase(A, stream, case)
    assert A.process(d.s, case.S, d.a, d.b, d.c, 5, 5, 5, stream) == 0
    assert oracle.block_relerr(d.result(stream), d.reference(), 25) <= TOL
    d.free()


def test_batch_rejects_unsuitable_stacks(acc):
    A, stream = acc
    case = W.stack_case(8, 8, 8, 100, 10, 10, 5, seed=600)
    d = DevCase(A, stream, case)
    bad = StackDesc(d.s.ptr, case.S, 90, 90, 8, d.a.ptr, d.b.ptr, d.c.ptr)  # m*n > 80^2
    arr = (StackDesc * 2)(d.desc(), bad)
    assert A.lib().libxstream_b200_process_batch(ctypes.cast(arr, ctypes.c_void_p), 2, 80, stream.handle) == -1
    assert not np.any(d.result(stream))  # nothing was done
    assert A.lib().libxstream_b200_process_batch(None, 0, 80, stream.handle) == 0
    d.free()


def test_batch_mixed_item_kinds(acc):
    """Large and small stacks of the same shapes in one persistent launch: 23^3 and 16x64x9 items run
    their staged item functions (16x64x9 with a 2 x 8-fragment tile), 45^3 items the register kernel
    with sub-tiles; every stack combines its CTA-crossing segments in the kernel. Parity and bitwise
    reproducibility."""
    A, stream = acc
    cases = [W.stack_case(16, 64, 9, 120000, 2000, 2000, 500, seed=701),
             W.stack_case(16, 64, 9, 900, 100, 100, 30, seed=702),
             W.stack_case(23, 23, 23, 90000, 2000, 2000, 400, seed=703),
             W.stack_case(23, 23, 23, 700, 50, 50, 20, seed=704),
             W.stack_case(45, 45, 45, 2000, 100, 100, 40, seed=705)]
    devs = [DevCase(A, stream, c, c0=W.rng(i).uniform(-1, 1, size=c.nc * c.m * c.n)) for i, c in enumerate(cases)]
    assert run_batch(A, stream, devs) == 0
    first = [d.result(stream) for d in devs]
    for d, got in zip(devs, first):
        assert oracle.block_relerr(got, d.reference(), d.case.m * d.case.n) <= TOL, (d.case.m, d.case.n, d.case.k)
    for d in devs:  # same inputs again from the same C: bitwise equal results
        d.c.upload(d.c0, stream)
    assert run_batch(A, stream, devs) == 0
    for d, got in zip(devs, first):
        assert np.array_equal(d.result(stream), got)
        d.free()
