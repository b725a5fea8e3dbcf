"""Seeded synthetic stacks and block pools for the SMM stack path.

Two families:
  * the benchmark workloads (uniform[-1,1] entries, Zipf(1.1)-distributed c index), drawn from
    numpy's PCG64 generator with a fixed seed (default 25071975, the seed of the reference's
    samples/smm/acc_bench.c:146);
  * the reference's own deterministic generators INIT_MAT and INIT_STACK
    (samples/smm/acc_bench.h:30-79) driven by glibc rand() seeded like acc_bench.c:144-147,
    so that a stack built exactly as acc_bench builds it can be replayed.
All offsets are element offsets into flat pools; stacks hold 1-based (a, b, c) triples as int32.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
from dataclasses import dataclass, field

import numpy as np

SEED = 25071975
MIXED_SHAPE_SET = (4, 5, 9, 13, 16, 22, 23, 26, 32, 45, 64)


def rng(seed: int = SEED) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def uniform_pool(g: np.random.Generator, nblocks: int, rows: int, cols: int) -> np.ndarray:
    return g.uniform(-1.0, 1.0, size=nblocks * rows * cols)


def spread_pool(g: np.random.Generator, nblocks: int, rows: int, cols: int, emin: int = -20, emax: int = 20) -> np.ndarray:
    """Entries mantissa U[1,2) * 2^e, e uniform integer in [emin, emax], random sign."""
    size = nblocks * rows * cols
    mant = g.uniform(1.0, 2.0, size=size)
    e = g.integers(emin, emax + 1, size=size)
    sign = np.where(g.integers(0, 2, size=size) == 0, -1.0, 1.0)
    return sign * np.ldexp(mant, e)


def zipf_indices(g: np.random.Generator, n: int, count: int, s: float = 1.1) -> np.ndarray:
    """count draws from a Zipf(s) law over n items (rank r has weight r^-s); ranks are mapped to
    item ids through a random permutation so the hot blocks are scattered over the pool."""
    w = np.arange(1, n + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    ranks = np.searchsorted(cdf, g.random(count), side="right")
    ranks = np.minimum(ranks, n - 1)
    perm = g.permutation(n)
    return perm[ranks]


def make_stack(g: np.random.Generator, S: int, na: int, nb: int, nc: int, m: int, n: int, k: int,
               zipf_s: float = 1.1, grouped: bool = False) -> np.ndarray:
    """(S, 3) int32 triples: a, b uniform over the pools, c Zipf(zipf_s); 1-based element offsets.
    grouped=True sorts the stack by c (stably), as DBCSR generates its stacks."""
    a = g.integers(0, na, size=S)
    b = g.integers(0, nb, size=S)
    c = zipf_indices(g, nc, S, zipf_s) if zipf_s > 0 else g.integers(0, nc, size=S)
    if grouped:
        order = np.argsort(c, kind="stable")
        a, b, c = a[order], b[order], c[order]
    st = np.empty((S, 3), dtype=np.int64)
    st[:, 0] = a * (m * k) + 1
    st[:, 1] = b * (k * n) + 1
    st[:, 2] = c * (m * n) + 1
    assert st.max() < 2**31
    return st.astype(np.int32)


def transpose_blocks_rowmajor(bpool_colmajor: np.ndarray, nblocks: int, k: int, n: int) -> np.ndarray:
    """Host-side reference of what libsmm_acc_transpose(k, n) makes of a B pool: each k x n
    column-major block becomes n x k column-major (= k x n row-major)."""
    return bpool_colmajor.reshape(nblocks, n, k).transpose(0, 2, 1).copy().reshape(-1)


@dataclass
class StackCase:
    m: int
    n: int
    k: int
    na: int
    nb: int
    nc: int
    stack: np.ndarray            # (S, 3) int32, 1-based offsets
    a: np.ndarray                # A pool, m x k column-major blocks
    b: np.ndarray                # B pool, k x n column-major blocks (host layout, before transpose)
    meta: dict = field(default_factory=dict)

    @property
    def S(self) -> int:
        return int(self.stack.shape[0])

    @property
    def flops(self) -> int:
        return 2 * self.m * self.n * self.k * self.S

    @property
    def algo_bytes(self) -> int:
        """Bytes per the reference's work statement: S * 8 * (mk + kn + 2mn) (smm_kernel.c:504-506)."""
        return self.S * 8 * (self.m * self.k + self.k * self.n + 2 * self.m * self.n)

    def b_rowmajor(self) -> np.ndarray:
        return transpose_blocks_rowmajor(self.b, self.nb, self.k, self.n)


def stack_case(m: int, n: int, k: int, S: int, na: int, nb: int, nc: int, seed: int = SEED, zipf_s: float = 1.1,
               values: str = "uniform", grouped: bool = False) -> StackCase:
    g = rng(seed)
    if values == "uniform":
        a = uniform_pool(g, na, m, k)
        b = uniform_pool(g, nb, k, n)
    elif values == "spread":
        a = spread_pool(g, na, m, k)
        b = spread_pool(g, nb, k, n)
    else:
        raise ValueError(values)
    st = make_stack(g, S, na, nb, nc, m, n, k, zipf_s=zipf_s, grouped=grouped)
    return StackCase(m, n, k, na, nb, nc, st, a, b, {"seed": seed, "zipf": zipf_s, "values": values})


def config1(seed: int = SEED) -> StackCase:
    """Plain FP64 23x23x23 stack: A/B pools of 4096 blocks, C pool of 1024 blocks, 30000 triples,
    a/b uniform, c Zipf(1.1), entries uniform[-1,1]."""
    return stack_case(23, 23, 23, 30000, 4096, 4096, 1024, seed=seed)


def pool_sizes(S: int) -> tuple[int, int, int]:
    """Pool sizes used for the mixed-shape and Ozaki stacks (not fixed by the workload statement):
    A/B pools of clamp(S/8, 16, 8192) blocks, C pool of clamp(S/32, 8, 2048) blocks."""
    nab = int(min(8192, max(16, S // 8)))
    nc = int(min(2048, max(8, S // 32)))
    return nab, nab, nc


def mixed_shapes(seed: int = SEED, nstacks: int = 12, smin: int = 100, smax: int = 200000) -> list[StackCase]:
    """12 stacks with (m, n, k) drawn from MIXED_SHAPE_SET^3 and sizes log-uniform in [smin, smax]."""
    g = rng(seed)
    cases = []
    for i in range(nstacks):
        m, n, k = (int(x) for x in g.choice(MIXED_SHAPE_SET, size=3))
        S = int(round(math.exp(g.uniform(math.log(smin), math.log(smax)))))
        na, nb, nc = pool_sizes(S)
        cases.append(stack_case(m, n, k, S, na, nb, nc, seed=seed + 1 + i))
    return cases


def mixed_shapes_scaled(total: int = 2_000_000, seed: int = SEED) -> list[StackCase]:
    """The 12 mixed_shapes() stacks with every stack size multiplied by one common factor so that
    the batch holds about `total` triples (the relative log-uniform spread is kept)."""
    base = mixed_shapes(seed=seed)
    scale = total / sum(c.S for c in base)
    out = []
    for i, c in enumerate(base):
        S = max(1, int(round(c.S * scale)))
        na, nb, nc = pool_sizes(S)
        out.append(stack_case(c.m, c.n, c.k, S, na, nb, nc, seed=seed + 1 + i))
    return out


def transpose_workload(seed: int = SEED, nblocks: int = 100000, smin: int = 5, smax: int = 64):
    """Square blocks with sizes uniform in [smin, smax]: returns {size: count}."""
    g = rng(seed)
    sizes = g.integers(smin, smax + 1, size=nblocks)
    vals, counts = np.unique(sizes, return_counts=True)
    return {int(v): int(c) for v, c in zip(vals, counts)}


# ------------------------------------------------------------ reference-compatible generators

def _libc():
    return ctypes.CDLL(ctypes.util.find_library("c"))


def reference_rand_table(count: int, seed: int = SEED) -> np.ndarray:
    """glibc rand() values after srand(seed), as acc_bench.c:144-147 fills its table."""
    libc = _libc()
    libc.srand(ctypes.c_uint(seed))
    return np.array([libc.rand() for _ in range(count)], dtype=np.int64)


def reference_init_mat(seed: int, m: int, n: int, scale: float) -> np.ndarray:
    """INIT_MAT (acc_bench.h:30-40): column-major m x n, value (scale*seed + scale) * (idx + 1)."""
    s1 = scale * seed + scale
    return s1 * (np.arange(m * n, dtype=np.float64) + 1.0)


def reference_init_stack(S: int, rnd: np.ndarray, mn: int, mk: int, kn: int, nc: int, na: int, nb: int) -> np.ndarray:
    """INIT_STACK (acc_bench.h:48-79) with a supplied random table: runs of c of average length S/nc."""
    assert 0 < nc <= S
    rsize = max(1, rnd.size)
    navg = S // nc
    nimb = max(1, navg - 4)
    out = np.empty((S, 3), dtype=np.int64)
    i = c = ntop = 0
    while i < S:
        r = int(rnd[i % rsize])
        nxt = c + 1
        ntop += navg + (r % (2 * nimb) - nimb)
        ntop = min(ntop, S)
        while i < ntop:
            a = int(rnd[(2 * i + 0) % rsize]) % na
            b = int(rnd[(2 * i + 1) % rsize]) % nb
            out[i] = (a * mk + 1, b * kn + 1, c * mn + 1)
            i += 1
        if nxt < nc:
            c = nxt
    return out.astype(np.int32)


def reference_case(m: int = 23, n: int | None = None, k: int | None = None, S: int = 30000, nrepeat: int = 1,
                   nrand: int = 30000) -> StackCase:
    """The acc_bench default problem (acc_bench.c:167-277): nc = S/16, na = nb = 10*nc, INIT_MAT
    seeds i+42 (A) and i+24 (B), scale 1/(nrepeat*nc*na), unpadded block strides."""
    n = m if n is None else n
    k = m if k is None else k
    nc = max(S // 16, 1)
    na = nb = 10 * nc
    nr = nrepeat * nc
    rnd = reference_rand_table(nrand)
    st = reference_init_stack(S, rnd, m * n, m * k, k * n, nc, na, nb)
    a = np.concatenate([reference_init_mat(i + 42, m, k, 1.0 / (nr * na)) for i in range(na)])
    b = np.concatenate([reference_init_mat(i + 24, k, n, 1.0 / (nr * nb)) for i in range(nb)])
    return StackCase(m, n, k, na, nb, nc, st, a, b, {"generator": "acc_bench INIT_MAT/INIT_STACK"})
