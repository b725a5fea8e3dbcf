"""CPU restatement of the Ozaki scheme-2 (Chinese remainder) FP64 GEMM (test infrastructure only).

The reference's scheme 2 (samples/ozaki/kernels/ozaki2_int8.cl:13-45; moduli count and input
mantissa bits, samples/ozaki/ozaki_opencl.c:406-426): each row of A and each column of B is scaled
by its largest power of two and truncated to a signed integer of `mb` bits (the aligned significand
of samples/ozaki/kernels/ozaki_common.cl:789-806, cut to mb bits); the integer product is taken
modulo every modulus (one 8-bit GEMM each on the device), reconstructed exactly by the CRT, centred
to [-P/2, P/2) and scaled back. This restatement computes the residue products with numpy int64
and the reconstruction with Python integers, so it is the scheme's exact result (the device's
reconstruction, a 128-bit binary fraction of x / P times P, differs from it by rounding only). The moduli are this build's own
set (pairwise coprime, <= 256); the reference picks its own.
"""
from __future__ import annotations

import math

import numpy as np

MODULI = (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181, 179, 173)


def mantissa_bits(nmod: int, K: int) -> int:
    """Bits per input integer that nmod moduli hold for inner dimension K (at most 53)."""
    lgk = max(0, math.ceil(math.log2(K))) if K > 1 else 0
    lp = sum(math.log2(m) for m in MODULI[:nmod])
    return min(53, int(math.floor((lp - 2.0 - lgk) / 2.0)))


def default_moduli(K: int) -> int:
    for n in range(1, len(MODULI) + 1):
        if mantissa_bits(n, K) >= 53:
            return n
    return len(MODULI)


def _aligned(X: np.ndarray, mb: int, axis: int):
    """Integers of mb bits aligned to the largest exponent along `axis` (rows of A: axis 1 of an
    (M, K) array), and the exponents (biased, 0 for all-zero / non-finite lines)."""
    bits = X.view(np.uint64)
    be = ((bits >> np.uint64(52)) & np.uint64(2047)).astype(np.int64)
    mant = (bits & np.uint64((1 << 52) - 1)) | np.uint64(1 << 52)
    bad = (be == 0) | (be == 2047)
    be = np.where(bad, 0, be)
    mant = np.where(bad, np.uint64(0), mant)
    emax = be.max(axis=axis, keepdims=True)
    sh = emax - be + 53 - mb
    u = np.where(sh < 64, mant >> np.minimum(sh, 63).astype(np.uint64), np.uint64(0))
    sign = np.where((bits >> np.uint64(63)) != 0, -1, 1)
    return u.astype(object) * sign.astype(object), np.squeeze(emax, axis=axis)


def ozaki2_gemm(A: np.ndarray, B: np.ndarray, nmod: int) -> np.ndarray:
    """C = A @ B by the scheme with nmod moduli; A (M, K), B (K, N) float64 row-major numpy arrays."""
    M, K = A.shape
    N = B.shape[1]
    mb = mantissa_bits(nmod, K)
    ia, ea = _aligned(np.ascontiguousarray(A), mb, 1)
    ib, eb = _aligned(np.ascontiguousarray(B.T), mb, 1)
    mods = MODULI[:nmod]
    P = math.prod(mods)
    # residue products per modulus in int64 (residues < 256, K * 255^2 < 2^63)
    res = []
    for m in mods:
        ra = np.array([[int(x) % m for x in row] for row in ia], dtype=np.int64)
        rb = np.array([[int(x) % m for x in row] for row in ib], dtype=np.int64)
        res.append((ra @ rb.T) % m)
    out = np.zeros((M, N))
    for i in range(M):
        for j in range(N):
            x = 0
            for q, m in enumerate(mods):  # exact CRT
                Mi = P // m
                x += int(res[q][i, j]) * Mi * pow(Mi, -1, m)
            x %= P
            if 2 * x >= P:
                x -= P
            if ea[i] == 0 or eb[j] == 0:
                continue
            out[i, j] = math.ldexp(float(x), int(ea[i]) + int(eb[j]) - 2150 + 2 * (53 - mb))
    return out
