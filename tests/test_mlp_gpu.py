"""GPU tests of the learned parameter predictor's device kernels against the CPU oracle
(oracle/mlp_oracle.py, FP64): forward pass, loss gradients, inference; training reduces the loss;
the installed predictor drives the stack path's parameter lookup; the exhaustive tuner times every
candidate."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from libxstream_b200 import predictor as P
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def random_problem(N: int, seed: int):
    g = np.random.default_rng(seed)
    raw = np.stack([g.integers(4, 81, N), g.integers(4, 81, N), g.integers(4, 81, N), g.choice(P.SIZES, N),
                    g.choice(P.SPREADS, N)], 1).astype(np.int32)
    r = np.zeros((N, P.K), dtype=np.float32)
    for i in range(N):
        v = P.valid_mask(int(raw[i, 0]), int(raw[i, 1]))
        t = 1.0 + g.random(P.K)
        t[g.integers(0, v.sum())] = 1.0
        r[i] = np.where(v, t / t[v].min(), 0.0)
    z = g.choice([-1.0, 0.0, 1.0], N).astype(np.float32)
    return raw, r, z


def test_forward_matches_oracle(acc):
    w = P.init_weights(3) * 1.5
    raw, _, _ = random_problem(700, 1)
    y = P.device_forward(w, raw)
    _, _, _, ref = M.forward(w.astype(np.float64), raw)
    assert np.max(np.abs(y - ref)) <= 1e-4 * max(1.0, np.max(np.abs(ref)))


def test_gradients_match_oracle(acc):
    w = P.init_weights(5)
    raw, r, z = random_problem(1000, 2)
    g, loss = P.device_grad(w, raw, r, z)
    lref, losses, gref = M.loss_and_grad(w.astype(np.float64), raw, r.astype(np.float64), z.astype(np.float64))
    assert abs(float(loss.mean()) - lref) <= 1e-5 * max(1.0, abs(lref))
    assert np.max(np.abs(loss - losses)) <= 1e-4
    assert np.linalg.norm(g - gref) <= 1e-4 * np.linalg.norm(gref)


def test_training_reduces_loss_and_learns_rule(acc):
    """Targets where the best configuration follows a rule of the shape; the network learns it."""
    g = np.random.default_rng(9)
    N = 3000
    raw = np.stack([g.integers(4, 81, N), g.integers(4, 81, N), g.integers(4, 81, N), g.choice(P.SIZES, N),
                    np.zeros(N, dtype=int)], 1).astype(np.int32)
    r = np.zeros((N, P.K), dtype=np.float32)
    for i in range(N):
        m, n, k = (int(x) for x in raw[i, :3])
        v = P.valid_mask(m, n)
        mt, nt = min(4, (m + 7) // 8), min(4, (n + 7) // 8)
        best = P.config_index(mt, nt, 4 if k > 16 else 2)
        r[i] = np.where(v, 1.0 + 0.05 * np.array([abs(c - best) for c in range(P.K)]), 0.0)
    z = (raw[:, 2] > 40).astype(np.float32)
    w, hist = P.train(raw, r, z, steps=2500, lr=3e-3)
    assert hist[-1] < 0.5 * hist[0]
    cfg, _, pz = P.device_predict(w, raw)
    chosen = r[np.arange(N), cfg]
    assert np.mean(chosen <= 1.05 + 1e-6) >= 0.95  # within 5% of the best on almost every sample
    assert np.mean((pz >= 0.5) == (z > 0.5)) >= 0.9


def test_predict_kernel_matches_oracle(acc):
    w = P.init_weights(11) * 2.0
    raw, _, _ = random_problem(500, 4)
    cfg, conf, pz = P.device_predict(w, raw)
    fma_ok = np.array([P.fma_supported(int(m), int(n), int(k)) for m, n, k in raw[:, :3]])
    rcfg, rconf, rpz = M.predict(w.astype(np.float64), raw, fma_ok)
    assert np.mean(cfg == rcfg) >= 0.995  # ties within FP32 rounding may differ
    assert np.max(np.abs(conf - rconf)) <= 1e-4 and np.max(np.abs(pz - rpz)) <= 1e-4


def test_install_drives_parameter_lookup(acc):
    A, _ = acc
    lib = A.lib()
    w = P.init_weights(13) * 2.0
    P.install(w)
    try:
        for (m, n, k, S) in [(23, 23, 23, 30000), (40, 9, 70, 1000), (80, 80, 80, 100000), (5, 64, 13, 5000)]:
            out = (ctypes.c_int * 3)()
            conf = ctypes.c_float()
            assert lib.libxstream_b200_mlp_lookup(m, n, k, S, out, ctypes.byref(conf)) == 1
            bucket = 1000 if S < 3000 else (10000 if S < 30000 else 100000)
            rc, _, _ = M.predict(w.astype(np.float64), np.array([[m, n, k, bucket, 0]]), [P.fma_supported(m, n, k)])
            assert P.config_index(out[0], out[1], out[2]) == int(rc[0])
            p6 = (ctypes.c_int * 6)()
            lib.libxstream_b200_get_params(m, n, k, S, p6)
            if (m, n, k) == (23, 23, 23) and int(rc[0]) != P.FMA:  # a staged kernel exists: its whole-block
                assert (p6[1], p6[2], p6[3]) == (3, 3, 0)                # tile replaces a predicted DMMA tile
            else:
                assert (p6[1], p6[2], p6[3]) == (out[0], out[1], out[2])
    finally:
        assert lib.libxstream_b200_mlp_install(None, 0) == 0
    out = (ctypes.c_int * 3)()
    assert lib.libxstream_b200_mlp_lookup(23, 23, 23, 30000, out, None) == 0


def test_tuner_times_every_candidate(acc):
    A, _ = acc
    lib = A.lib()
    t = P.tune_one(lib, 20, 9, 13, 2000, reps=1, ozaki=7)
    cand = (ctypes.c_int * (3 * (P.K + 1)))()
    nc = lib.libxstream_b200_tune_candidates(20, 9, cand, P.K + 1)
    assert nc == 3 * 2 * 2 + 1 and len([c for c in t if c != "oz"]) == nc  # 12 DMMA tile classes + the FMA kernel
    assert (cand[3 * 12], cand[3 * 12 + 1], cand[3 * 12 + 2]) == (1, 1, -1) and P.FMA in t
    assert all(v > 0 for v in t.values()) and "oz" in t
