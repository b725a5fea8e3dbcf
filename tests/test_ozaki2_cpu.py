"""CPU tests of the Ozaki scheme-2 restatement (oracle/ozaki2.py) and of the arithmetic the device's
CRT reconstruction uses (a 128-bit binary fraction of x / P, centred by its two's-complement
reading, times P in double precision), restated here in Python integers and exact rationals."""
from __future__ import annotations

import math
import random
from fractions import Fraction

import numpy as np
import pytest

from oracle import ozaki2 as O


def test_moduli_pairwise_coprime_and_bytes():
    mods = O.MODULI
    assert all(2 <= m <= 256 for m in mods)
    for i, a in enumerate(mods):
        for b in mods[:i]:
            assert math.gcd(a, b) == 1


@pytest.mark.parametrize("K", [1, 17, 64, 65, 4096, 40000, 1 << 17])
def test_default_moduli_is_fewest_for_53_bits(K):
    n = O.default_moduli(K)
    assert O.mantissa_bits(n, K) == 53
    assert O.mantissa_bits(n - 1, K) < 53
    # P > 2 K 2^(2 mb): the centred integer products fit
    P = math.prod(O.MODULI[:n])
    assert P > 2 * K * (1 << (2 * O.mantissa_bits(n, K)))


def test_default_moduli_counts():
    assert O.default_moduli(64) == 15
    assert O.default_moduli(4096) == 16
    assert O.default_moduli(1 << 17) == 16


def test_integer_inputs_are_exact():
    """Small integers keep all their bits: the scheme returns the exact product."""
    g = np.random.default_rng(5)
    A = g.integers(-1000, 1000, size=(6, 40)).astype(np.float64)
    B = g.integers(-1000, 1000, size=(40, 5)).astype(np.float64)
    got = O.ozaki2_gemm(A, B, O.default_moduli(40))
    assert np.array_equal(got, A @ B)


def test_error_bound_against_exact_product():
    """Entries below their row's (column's) largest exponent lose the bits under 2^(e_max - 52):
    |C - AB| <= K 2^-51 max|a_i.| max|b_.j| element by element (plus the final rounding)."""
    g = np.random.default_rng(6)
    M, N, K = 5, 4, 24
    A = g.uniform(-1, 1, size=(M, K)) * np.exp2(g.integers(-8, 8, size=(M, K)))
    B = g.uniform(-1, 1, size=(K, N)) * np.exp2(g.integers(-8, 8, size=(K, N)))
    got = O.ozaki2_gemm(A, B, O.default_moduli(K))
    for i in range(M):
        for j in range(N):
            exact = sum(Fraction(A[i, k]) * Fraction(B[k, j]) for k in range(K))
            bound = K * 2.0 ** -51 * np.max(np.abs(A[i])) * np.max(np.abs(B[:, j])) + abs(float(exact)) * 2.0 ** -53
            assert abs(Fraction(got[i, j]) - exact) <= Fraction(bound)


def _fraction_words(nmod: int):
    """w_i = floor(2^128 y_i / m_i), y_i = (P / m_i)^-1 mod m_i; P as a double-double."""
    mods = O.MODULI[:nmod]
    P = math.prod(mods)
    W = []
    for m in mods:
        pm = (P // m) % m
        W.append((pow(pm, -1, m) << 128) // m)
    phi = float(P)
    plo = float(P - int(phi))
    return mods, P, W, phi, plo


def _fma(a: float, b: float, c: float) -> float:
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _reconstruct(res, W, phi, plo) -> float:
    """x as the device computes it: S = sum r_i w_i mod 2^128, T its signed upper and U its lower
    64 bits; th = round(T), tl = (T - th) + U 2^-64; x 2^64 = th phi + (th plo + tl phi)."""
    S = sum(r * w for r, w in zip(res, W)) % (1 << 128)
    T, U = S >> 64, S & ((1 << 64) - 1)
    if T >= 1 << 63:
        T -= 1 << 64
    th = float(T)
    tl = float(T - int(th)) + float(U) * 2.0 ** -64
    return _fma(th, phi, _fma(th, plo, tl * phi)) * 2.0 ** -64


@pytest.mark.parametrize("nmod", [8, 12, 14, 16])
def test_fraction128_reconstruction_matches_exact_crt(nmod):
    mods, P, W, phi, plo = _fraction_words(nmod)
    rnd = random.Random(nmod)
    xs = [0, 1, -1, 2, -2, P // 4 - 1, -(P // 4)]
    xs += [rnd.randrange(-P // 4, P // 4) for _ in range(300)]
    xs += [rnd.randrange(-(1 << 60), 1 << 60) for _ in range(300)]
    for x in xs:
        got = _reconstruct([x % m for m in mods], W, phi, plo)
        # one rounding of x, plus the 2^-128 truncation of the words (nmod * 255 * 2^-128 of P)
        assert abs(Fraction(got) - x) <= abs(x) * Fraction(2) ** -52 + Fraction(P) * Fraction(2) ** -115, (nmod, x)
