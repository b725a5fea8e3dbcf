"""CPU oracle (numpy, FP64) of the learned parameter predictor -- test infrastructure only: the same
features, forward pass, loss and gradients as the device kernels in libxstream_b200/csrc/mlp.cu, so
that the device's forward pass and gradients can be checked against it (and it against finite
differences).

Network: 27 features -> relu(64) -> relu(64) -> 34 outputs (33 configuration logits: 32 DMMA tile
classes and the FMA kernel, + 1 Ozaki logit).
Weights are one flat vector: W1[27][64], b1[64], W2[64][64], b2[64], W3[64][34], b3[34].
Loss per sample: cross-entropy of the masked softmax of the configuration logits against the soft
target q_c ~ exp(-(r_c - 1) / 0.02) over the applicable configurations (r_c > 0), plus the binary
cross-entropy of the Ozaki logit when its label z is 0 or 1; the total is the mean.
"""
from __future__ import annotations

import numpy as np

F, H, K = 27, 64, 33
TARGET_TEMP = 0.02
O = K + 1
SHAPES = [("W1", (F, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, O)), ("b3", (O,))]
NW = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(w: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(w[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(parts: dict) -> np.ndarray:
    return np.concatenate([np.asarray(parts[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def features(raw: np.ndarray) -> np.ndarray:
    """raw: int (N, 5) rows (m, n, k, S, spread) -> float64 (N, 27): one-hot ceil(m/8) and ceil(n/8)
    (1..10), log2 k / 6.5, (k mod 8)/8, log10 S / 5, spread / 40, log2(m n k S) / 40, (m mod 8)/8,
    (n mod 8)/8."""
    raw = np.asarray(raw, dtype=np.int64)
    m, n, k, S, sp = (raw[:, i].astype(np.float64) for i in range(5))
    S = np.maximum(S, 1.0)
    x = np.zeros((raw.shape[0], F))
    fm = np.clip((raw[:, 0] + 7) // 8, 1, 10)
    fn = np.clip((raw[:, 1] + 7) // 8, 1, 10)
    x[np.arange(raw.shape[0]), fm - 1] = 1.0
    x[np.arange(raw.shape[0]), 10 + fn - 1] = 1.0
    x[:, 20] = np.log2(k) / 6.5
    x[:, 21] = (raw[:, 2] & 7) / 8.0
    x[:, 22] = np.log10(S) / 5.0
    x[:, 23] = sp / 40.0
    x[:, 24] = (np.log2(m) + np.log2(n) + np.log2(k) + np.log2(S)) / 40.0
    x[:, 25] = (raw[:, 0] & 7) / 8.0
    x[:, 26] = (raw[:, 1] & 7) / 8.0
    return x


def forward(w: np.ndarray, raw: np.ndarray):
    p = unpack(w)
    x = features(raw)
    a1 = x @ p["W1"] + p["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ p["W2"] + p["b2"]
    h2 = np.maximum(a2, 0.0)
    y = h2 @ p["W3"] + p["b3"]
    return x, h1, h2, y


def loss_and_grad(w: np.ndarray, raw: np.ndarray, r: np.ndarray, z: np.ndarray):
    """Mean loss, per-sample losses and the gradient with respect to the flat weights."""
    p = unpack(w)
    x, h1, h2, y = forward(w, raw)
    N = x.shape[0]
    valid = r > 0
    yc = np.where(valid, y[:, :K], -np.inf)
    ymax = yc.max(axis=1, keepdims=True)
    logp = np.where(valid, yc - ymax - np.log(np.where(valid, np.exp(yc - ymax), 0.0).sum(axis=1, keepdims=True)), 0.0)
    eq = np.where(valid, np.exp(-(r - 1.0) / TARGET_TEMP), 0.0)
    q = eq / eq.sum(axis=1, keepdims=True)
    losses = -(q * logp).sum(axis=1)
    dy = np.zeros_like(y)
    dy[:, :K] = np.where(valid, np.exp(logp) - q, 0.0) / N
    known = z >= 0
    yk = y[:, K]
    bce = np.maximum(yk, 0) - yk * z + np.log1p(np.exp(-np.abs(yk)))
    losses = losses + np.where(known, bce, 0.0)
    dy[:, K] = np.where(known, (1.0 / (1.0 + np.exp(-yk)) - z) / N, 0.0)
    g = {"W3": h2.T @ dy, "b3": dy.sum(axis=0)}
    dh2 = (dy @ p["W3"].T) * (h2 > 0)
    g["W2"] = h1.T @ dh2
    g["b2"] = dh2.sum(axis=0)
    dh1 = (dh2 @ p["W2"].T) * (h1 > 0)
    g["W1"] = x.T @ dh1
    g["b1"] = dh1.sum(axis=0)
    return float(losses.mean()), losses, pack(g)


def predict(w: np.ndarray, raw: np.ndarray, fma_ok: np.ndarray | None = None):
    """Masked argmax configuration, its softmax probability and the Ozaki probability. The DMMA tile
    classes (c < 32) apply up to ceil(dim/8) fragments; the FMA kernel (c = 32) where fma_ok (per
    sample, the library's rule for its lane grids and ring; None: nowhere)."""
    _, _, _, y = forward(w, raw)
    raw = np.asarray(raw)
    mtmax = np.clip((raw[:, 0] + 7) // 8, 1, 4)
    ntmax = np.clip((raw[:, 1] + 7) // 8, 1, 4)
    c = np.arange(K)
    valid = ((c[None, :] >> 3) + 1 <= mtmax[:, None]) & ((((c[None, :] >> 1) & 3) + 1) <= ntmax[:, None]) & (c[None, :] < 32)
    fok = np.zeros(raw.shape[0], dtype=bool) if fma_ok is None else np.asarray(fma_ok, dtype=bool)
    valid[:, 32] = fok
    yc = np.where(valid, y[:, :K], -np.inf)
    best = yc.argmax(axis=1)
    e = np.where(valid, np.exp(yc - yc.max(axis=1, keepdims=True)), 0.0)
    conf = 1.0 / e.sum(axis=1)
    pz = 1.0 / (1.0 + np.exp(-y[:, K]))
    return best, conf, pz
