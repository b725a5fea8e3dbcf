"""GPU parity tests of libsmm_acc_process / libsmm_acc_transpose / c_calculate_norms through the
C-ABI against the CPU oracle. Tolerance for FP64 stacks: relative max-norm error per C block
<= 1e-13; transposes and the stack sort are bit-exact."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from libxstream_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-13


def run_device(A, stream, case: W.StackCase, c0: np.ndarray | None = None, transpose_on_device: bool = True,
               stack: np.ndarray | None = None) -> np.ndarray:
    """Upload pools, transpose B on the device (as acc_bench.c:317-328 does), run the stack, download C."""
    m, n, k = case.m, case.n, case.k
    st = case.stack if stack is None else stack
    S = st.shape[0]
    da = A.DevBuf.from_array(case.a, stream)
    if transpose_on_device and k * n <= 80 * 80:  # the ABI transposes blocks up to max_kernel_dim^2 only
        db = A.DevBuf.from_array(case.b, stream)
        trs = A.DevBuf.from_array(np.arange(case.nb, dtype=np.int32) * (k * n), stream)
        assert A.transpose(trs, 0, case.nb, db, k, n, stream) == 0
    else:
        db = A.DevBuf.from_array(case.b_rowmajor(), stream)
        trs = None
    c = np.zeros(case.nc * m * n) if c0 is None else c0.copy()
    dc = A.DevBuf.from_array(c, stream)
    ds = A.DevBuf.from_array(st if S else np.zeros(3, np.int32), stream)
    rc = A.process(ds, S, da, db, dc, m, n, k, stream, host_stack=st)
    assert rc == 0
    dc.download(c, stream)
    stream.sync()
    for buf in (da, db, dc, ds) + ((trs,) if trs else ()):
        buf.free()
    return c


def oracle_c(case: W.StackCase, c0: np.ndarray | None = None, stack=None) -> np.ndarray:
    c = np.zeros(case.nc * case.m * case.n) if c0 is None else c0.copy()
    oracle.smm(case.stack if stack is None else stack, case.a, case.b, c, case.m, case.n, case.k, b_rowmajor=False,
               threads=oracle.max_threads())
    return c


def test_config1_parity(acc):
    """The 23x23x23 workload at full size (30000 triples, Zipf(1.1) c)."""
    A, stream = acc
    case = W.config1()
    got = run_device(A, stream, case)
    ref = oracle_c(case)
    assert oracle.block_relerr(got, ref, 23 * 23) <= TOL


SHAPES = [(1, 1, 1), (2, 3, 5), (4, 4, 4), (5, 5, 5), (8, 8, 8), (9, 9, 9), (13, 13, 13), (16, 16, 16), (22, 22, 22),
          (26, 26, 26), (32, 32, 32), (45, 45, 45), (64, 64, 64), (80, 80, 80), (23, 5, 64), (64, 4, 9), (7, 45, 13),
          (23, 23, 100), (80, 3, 80), (3, 80, 150)]


@pytest.mark.parametrize("shape", SHAPES, ids=[f"{m}x{n}x{k}" for m, n, k in SHAPES])
def test_shapes_parity(acc, shape):
    A, stream = acc
    m, n, k = shape
    case = W.stack_case(m, n, k, 1500, 97, 89, 31, seed=m * 10000 + n * 100 + k)
    c0 = W.rng(1).uniform(-1, 1, size=case.nc * m * n)  # C accumulates onto existing content
    got = run_device(A, stream, case, c0=c0)
    ref = oracle_c(case, c0=c0)
    assert oracle.block_relerr(got, ref, m * n) <= TOL


@pytest.mark.parametrize("chunk,mt,nt,kp,wpb", [(1, 3, 3, 2, 1), (2, 1, 1, 4, 4), (3, 2, 4, 2, 2), (7, 4, 4, 4, 3),
                                                 (64, 3, 2, 4, 4), (1000, 1, 3, 2, 1)])
def test_parameter_variants_parity(acc, chunk, mt, nt, kp, wpb):
    """Every kernel variant and chunk length gives the same result (pieces cross many chunks)."""
    A, stream = acc
    case = W.stack_case(23, 23, 23, 3000, 200, 200, 40, seed=chunk + mt)
    A.set_params(23, 23, 23, chunk, mt, nt, kp, wpb)
    try:
        got = run_device(A, stream, case)
    finally:
        A.lib().libxstream_b200_clear_params()
    assert oracle.block_relerr(got, oracle_c(case), 23 * 23) <= TOL


def test_single_hot_block(acc):
    """Every entry updates the same C block: one segment spans every chunk."""
    A, stream = acc
    case = W.stack_case(23, 23, 23, 20000, 300, 300, 1, seed=4)
    assert oracle.block_relerr(run_device(A, stream, case), oracle_c(case), 23 * 23) <= TOL


def test_grouped_stack_and_singletons(acc):
    A, stream = acc
    case = W.stack_case(16, 16, 16, 5000, 100, 100, 5000, seed=5, zipf_s=0.0, grouped=True)
    assert oracle.block_relerr(run_device(A, stream, case), oracle_c(case), 256) <= TOL


def test_single_entry_and_empty(acc):
    A, stream = acc
    case = W.stack_case(23, 23, 23, 1, 2, 2, 1, seed=6)
    assert oracle.block_relerr(run_device(A, stream, case), oracle_c(case), 529) <= TOL
    empty = np.zeros((0, 3), np.int32)
    got = run_device(A, stream, case, stack=empty)
    assert not np.any(got)


def test_reference_generator_parity(acc):
    """The acc_bench default problem built by the reference's own INIT_MAT/INIT_STACK."""
    A, stream = acc
    case = W.reference_case(23, S=30000)
    assert oracle.block_relerr(run_device(A, stream, case), oracle_c(case), 529) <= TOL


def test_deterministic_bitwise(acc):
    A, stream = acc
    case = W.stack_case(23, 23, 23, 30000, 4096, 4096, 1024, seed=9)
    r1 = run_device(A, stream, case)
    r2 = run_device(A, stream, case)
    assert np.array_equal(r1, r2)


def test_accumulates_on_repeated_calls(acc):
    """Two calls add twice (beta = 1 semantics of acc_bench's repeated timed loop)."""
    A, stream = acc
    case = W.stack_case(13, 13, 13, 2000, 50, 50, 20, seed=10)
    m, n, k = 13, 13, 13
    da = A.DevBuf.from_array(case.a, stream)
    db = A.DevBuf.from_array(case.b_rowmajor(), stream)
    dc = A.DevBuf(case.nc * m * n * 8)
    dc.zero(stream)
    ds = A.DevBuf.from_array(case.stack, stream)
    for _ in range(2):
        assert A.process(ds, case.S, da, db, dc, m, n, k, stream) == 0
    got = dc.download(np.zeros(case.nc * m * n), stream)
    stream.sync()
    ref = oracle_c(case)
    ref = oracle_c(case, c0=ref)
    for b in (da, db, dc, ds):
        b.free()
    assert oracle.block_relerr(got, ref, m * n) <= TOL


@pytest.mark.parametrize("m,n", [(23, 23), (5, 64), (64, 5), (80, 80), (7, 3), (1, 9), (45, 45)])
def test_transpose_bit_exact(acc, m, n):
    A, stream = acc
    g = W.rng(m * 100 + n)
    nblk = 333
    data = g.uniform(-1, 1, size=(nblk + 5) * m * n)
    trs = (g.permutation(nblk + 5)[:nblk] * (m * n)).astype(np.int32)
    offset = 3
    trs_full = np.concatenate([np.zeros(offset, np.int32), trs])
    dd = A.DevBuf.from_array(data, stream)
    dt = A.DevBuf.from_array(trs_full, stream)
    assert A.transpose(dt, offset, nblk, dd, m, n, stream) == 0
    got = dd.download(np.zeros_like(data), stream)
    stream.sync()
    ref = oracle.transpose(trs_full, offset, data.copy(), m, n)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    # transposing back restores the input bit for bit
    assert A.transpose(dt, offset, nblk, dd, n, m, stream) == 0
    back = dd.download(np.zeros_like(data), stream)
    stream.sync()
    assert np.array_equal(back.view(np.uint64), data.view(np.uint64))
    dd.free()
    dt.free()


def test_transpose_preserves_special_values(acc):
    A, stream = acc
    m, n = 4, 3
    vals = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1.0, -2.5, 1e308, -1e-308, 3.0, 7.0])
    nan_payload = np.array([0x7ff8000000000123], dtype=np.uint64).view(np.float64)
    vals[4] = nan_payload[0]
    dd = A.DevBuf.from_array(vals, stream)
    dt = A.DevBuf.from_array(np.zeros(1, np.int32), stream)
    assert A.transpose(dt, 0, 1, dd, m, n, stream) == 0
    got = dd.download(np.zeros_like(vals), stream)
    stream.sync()
    ref = oracle.transpose(np.zeros(1, np.int32), 0, vals.copy(), m, n)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    dd.free()
    dt.free()


def test_norms(acc):
    A, stream = acc
    g = W.rng(12)
    mat = g.uniform(-1, 1, size=50000)
    offs = np.sort(g.integers(0, 40000, size=500)).astype(np.int32)
    ne = g.integers(1, 5000, size=500).astype(np.int32)
    dm, do, dn = A.DevBuf.from_array(mat, stream), A.DevBuf.from_array(offs, stream), A.DevBuf.from_array(ne, stream)
    dout = A.DevBuf(500 * 4)
    assert A.norms(dm, 500, do, dn, dout, stream) == 0
    got = dout.download(np.zeros(500, np.float32), stream)
    stream.sync()
    np.testing.assert_allclose(got, oracle.norms(mat, offs, ne), rtol=2e-7)
    for b in (dm, do, dn, dout):
        b.free()


def test_unhandled_returns_minus_one_on_device(acc):
    A, stream = acc
    dummy = A.DevBuf(64)
    assert A.process(dummy, 4, dummy, dummy, dummy, 81, 81, 4, stream) == -1
    assert A.process(dummy, 4, dummy, dummy, dummy, 23, 23, 23, stream, def_mnk=0) == -1
    dummy.free()


def test_injected_allocation_failure_is_reported(acc):
    A, stream = acc
    case = W.stack_case(8, 8, 8, 100, 10, 10, 4, seed=13)
    da = A.DevBuf.from_array(case.a, stream)
    db = A.DevBuf.from_array(case.b_rowmajor(), stream)
    dc = A.DevBuf(case.nc * 64 * 8)
    ds = A.DevBuf.from_array(case.stack, stream)
    A.lib().libxstream_b200_inject_alloc_failure(1)
    assert A.process(ds, case.S, da, db, dc, 8, 8, 8, stream) != 0
    A.lib().libxstream_b200_inject_alloc_failure(0)
    A.lib().c_dbcsr_acc_clear_errors()
    assert A.process(ds, case.S, da, db, dc, 8, 8, 8, stream) == 0
    stream.sync()
    for b in (da, db, dc, ds):
        b.free()


def test_runtime_events_and_streams(acc):
    A, stream = acc
    lib = A.lib()
    import ctypes
    lo, hi = ctypes.c_int(), ctypes.c_int()
    assert lib.c_dbcsr_acc_stream_priority_range(ctypes.byref(lo), ctypes.byref(hi)) == 0
    s2 = A.Stream("calc", hi.value)
    ev = A.Event()
    buf = A.DevBuf(1 << 20)
    buf.zero(stream)
    ev.record(stream)
    assert lib.c_dbcsr_acc_stream_wait_event(s2.handle, ev.handle) == 0
    ev.sync()
    assert ev.query()
    fr, tot = ctypes.c_size_t(), ctypes.c_size_t()
    assert lib.c_dbcsr_acc_dev_mem_info(ctypes.byref(fr), ctypes.byref(tot)) == 0 and 0 < fr.value <= tot.value
    host = A.HostBuf((1000,), np.float64, stream)
    host.array[:] = np.arange(1000)
    b2 = A.DevBuf(8000)
    b2.upload(host.array, None)            # NULL stream: synchronous
    out = b2.download(np.zeros(1000), None)
    assert np.array_equal(out, np.arange(1000))
    assert lib.c_dbcsr_acc_memcpy_d2d(b2.ptr, buf.ptr, 8000, None) == 0
    out2 = buf.download(np.zeros(1000), None)
    assert np.array_equal(out2, np.arange(1000))
    host.free(stream)
    for b in (buf, b2):
        b.free()
    ev.destroy()
    s2.sync()
    s2.destroy()
    assert lib.c_dbcsr_acc_device_synchronize() == 0


def test_irregular_c_offsets_multipass_sort(acc):
    """C blocks at irregular, non-overlapping offsets (gap of 0..5 elements between blocks, so the
    gcd of offset differences is 1 and the bucket ids span several radix digits)."""
    A, stream = acc
    m, n, k = 9, 7, 5
    g = W.rng(21)
    nc = 3000
    gaps = g.integers(0, 6, size=nc)
    starts = np.concatenate([[0], np.cumsum(m * n + gaps)[:-1]])
    case = W.stack_case(m, n, k, 20000, 300, 300, nc, seed=22)
    cblk = (case.stack[:, 2] - 1) // (m * n)
    st = case.stack.copy()
    st[:, 2] = starts[cblk] + 1
    total = int(starts[-1] + m * n)
    case2 = W.StackCase(m, n, k, case.na, case.nb, nc, st, case.a, case.b)
    c0 = np.zeros(total)
    da = A.DevBuf.from_array(case.a, stream)
    db = A.DevBuf.from_array(case.b_rowmajor(), stream)
    dc = A.DevBuf.from_array(c0, stream)
    ds = A.DevBuf.from_array(st, stream)
    assert A.process(ds, case.S, da, db, dc, m, n, k, stream) == 0
    got = dc.download(np.zeros(total), stream)
    stream.sync()
    ref = np.zeros(total)
    oracle.smm(st, case.a, case.b, ref, m, n, k, b_rowmajor=False)
    for b in (da, db, dc, ds):
        b.free()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= TOL
    del case2


@pytest.mark.parametrize("S", [2048, 2049, 16385, 32768, 32769])
def test_grouping_cluster_and_cooperative_sizes(acc, S):
    """Stacks of up to 16 tiles of 2048 entries are grouped by one thread-block cluster, larger ones by
    the cooperative kernel; both sides of each size boundary agree with the oracle and are bitwise
    reproducible."""
    A, stream = acc
    case = W.stack_case(23, 23, 23, S, 500, 500, 300, seed=S)
    r1 = run_device(A, stream, case)
    r2 = run_device(A, stream, case)
    assert np.array_equal(r1, r2)
    assert oracle.block_relerr(r1, oracle_c(case), 529) <= TOL
