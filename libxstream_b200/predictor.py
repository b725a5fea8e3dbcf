"""Autotuner sweeps and the learned parameter predictor (host side).

The exhaustive tuner (libxstream_b200_tune) times every precompiled configuration of the plain stack
kernels -- the DMMA tile classes MT x NT (each <= ceil(dim/8), <= 4) with k-panel KP in {2, 4}, 32
classes c = (mt-1)*8 + (nt-1)*2 + (kp==4), and the register-blocked FMA kernel, c = 32, where its lane
grids cover the block -- and, for m, n, k <= 64, the Ozaki form, on synthetic stacks of a given shape
and size. A sweep over many shapes is the predictor's training set: every (shape, stack
size) becomes samples for the exponent spreads {0, 10, 40} with targets r_c = t_c / t_best and the
Ozaki label (Ozaki faster than the best plain configuration). The network (3 x FP32 width 64, see
csrc/mlp.cu) is trained on the device by the library's own kernels; the exhaustive tuner is its
fallback (shapes where the network is not confident are tuned) and its referee (held-out shapes are
scored by the measured time of the predicted configuration against the tuned optimum).

Command line (one GPU):
  python -m libxstream_b200.predictor sweep --out sweep.csv --shapes 4000 --heldout 300 --minutes 12
  python -m libxstream_b200.predictor sweep --fma-only --out sweep_fma.csv   # re-tune the shapes the
        FMA kernel takes, with every candidate; train/eval --override sweep_fma.csv replace those rows
  python -m libxstream_b200.predictor train --sweep sweep.csv --out mlp.txt
  python -m libxstream_b200.predictor eval --sweep sweep.csv --weights mlp.txt
"""
from __future__ import annotations

import argparse
import ctypes
import gzip
import json
import math
import time
from pathlib import Path

import numpy as np

K = 33  # configurations: 32 DMMA tile classes, then the FMA kernel
FMA = 32
NFEAT = 27
SPREADS = (0, 10, 40)
SIZES = (1000, 10000, 100000)
PARAMS_DIR = Path(__file__).resolve().parent / "params"
DEFAULT_WEIGHTS = PARAMS_DIR / "mlp_b200.txt"
DEFAULT_SWEEP = PARAMS_DIR / "sweep_b200.csv.gz"
DEFAULT_SWEEP_FMA = PARAMS_DIR / "sweep_fma_b200.csv.gz"  # the FMA kernel's shapes re-tuned with every candidate


def config_index(mt: int, nt: int, kp: int) -> int:
    if kp < 0:  # the FMA kernel (kp = -1)
        return FMA
    return (mt - 1) * 8 + (nt - 1) * 2 + (1 if kp == 4 else 0)


def config_of(c: int) -> tuple[int, int, int]:
    if c == FMA:
        return 1, 1, -1
    return (c >> 3) + 1, ((c >> 1) & 3) + 1, 4 if (c & 1) else 2


def fma_supported(m: int, n: int, k: int) -> bool:
    """The FMA kernel takes m x n x k (its lane grids cover the block, its ring fits shared memory):
    the library's own rule (a host function, no device call)."""
    from . import lib as _lib
    f = _lib().xs_smm_fma_supported
    f.restype, f.argtypes = ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    return bool(f(m, n, k))


def valid_mask(m: int, n: int, k: int | None = None) -> np.ndarray:
    """Configurations that apply to m x n (x k): the DMMA tile classes up to ceil(dim/8) fragments,
    the FMA kernel where it takes the shape (only when k is given)."""
    mtmax, ntmax = min(4, max(1, (m + 7) // 8)), min(4, max(1, (n + 7) // 8))
    v = [config_of(c)[0] <= mtmax and config_of(c)[1] <= ntmax for c in range(FMA)]
    return np.array(v + [k is not None and fma_supported(m, n, k)])


def random_shapes(count: int, seed: int, lo: int = 4, hi: int = 80, exclude: set | None = None) -> list[tuple[int, int, int]]:
    g = np.random.Generator(np.random.PCG64(seed))
    out, seen = [], set(exclude or ())
    while len(out) < count:
        s = tuple(int(x) for x in g.integers(lo, hi + 1, size=3))
        if s not in seen:
            seen.add(s)
            out.append(s)
    return out


# ------------------------------------------------------------------------------------- sweep

def tune_one(lib, m: int, n: int, k: int, S: int, reps: int = 2, ozaki: int = 7, seed: int = 12345) -> dict:
    """Times of every applicable configuration {c: ms} and the Ozaki time (key 'oz') when measured."""
    cand = (ctypes.c_int * (3 * (K + 1)))()
    nc = lib.libxstream_b200_tune_candidates(m, n, cand, K + 1)
    ms = (ctypes.c_float * (K + 2))()
    got = lib.libxstream_b200_tune(m, n, k, S, reps, ozaki, seed, ms, K + 2, None)
    if got < nc:
        raise RuntimeError(f"tune {m}x{n}x{k} S={S} failed ({got}, last error {lib.libxstream_b200_last_error()})")
    out = {}
    for i in range(nc):  # configuration index -> ms (the FMA kernel, kp = -1, is index FMA)
        if ms[i] < 0:
            continue  # the candidate does not take this shape
        out[config_index(cand[3 * i], cand[3 * i + 1], cand[3 * i + 2])] = float(ms[i])
    if got > nc:
        out["oz"] = float(ms[nc])
    return out


def sweep(out: Path, shapes: list, heldout: list, minutes: float, reps: int = 2, header: bool = True,
          fma_only: bool = False) -> int:
    """Tunes held-out shapes first, then training shapes, until the time budget is spent; one CSV row
    per (shape, stack size): split,m,n,k,S,t_0..t_32 (ms, empty = not applicable; t_32 is the FMA
    kernel),t_oz. fma_only: only the shapes the FMA kernel takes (every candidate is still timed)."""
    from . import lib as _lib
    lib = _lib()
    t_end = time.time() + 60.0 * minutes
    rows = 0
    opener = gzip.open if str(out).endswith(".gz") else open
    with opener(out, "wt") as f:
        if header:
            f.write("split,m,n,k,S," + ",".join(f"t{c}" for c in range(K)) + ",t_oz\n")
        for split, group in (("heldout", heldout), ("train", shapes)):
            for (m, n, k) in group:
                if time.time() > t_end:
                    break
                if fma_only and not fma_supported(m, n, k):
                    continue
                for S in SIZES:
                    t = tune_one(lib, m, n, k, S, reps)
                    cells = [f"{t[c]:.5f}" if c in t else "" for c in range(K)]
                    f.write(f"{split},{m},{n},{k},{S}," + ",".join(cells) + "," + (f"{t['oz']:.5f}" if "oz" in t else "") + "\n")
                    rows += 1
                f.flush()
    return rows


def load_sweep(path: Path, override: Path | None = None) -> list[dict]:
    """Sweep records; a file with 32 configuration columns (before the FMA kernel) has no FMA time.
    override: a second sweep whose rows replace the rows of the same (m, n, k, S)."""
    opener = gzip.open if str(path).endswith(".gz") else open
    recs = []
    with opener(path, "rt") as f:
        cols = next(f).rstrip("\n").split(",")
        nk = sum(1 for c in cols if c.startswith("t") and c[1:].isdigit())
        for line in f:
            p = line.rstrip("\n").split(",")
            t = np.full(K, np.nan)
            t[:nk] = [float(x) if x else np.nan for x in p[5:5 + nk]]
            recs.append({"split": p[0], "m": int(p[1]), "n": int(p[2]), "k": int(p[3]), "S": int(p[4]), "t": t,
                         "oz": float(p[5 + nk]) if p[5 + nk] else None})
    if override is not None:
        newer = {(r["m"], r["n"], r["k"], r["S"]): r for r in load_sweep(override)}
        recs = [newer.pop((r["m"], r["n"], r["k"], r["S"]), r) for r in recs] + list(newer.values())
    return recs


def build_dataset(recs: list[dict], spreads=SPREADS):
    """raw (N, 5) int32, r (N, K) float32 (t_c / t_best, 0 = not applicable), z (N,) float32."""
    raw, r, z = [], [], []
    for rec in recs:
        t = rec["t"]
        best = np.nanmin(t)
        ratio = np.where(np.isnan(t), 0.0, t / best)
        zi = -1.0 if rec["oz"] is None else (1.0 if rec["oz"] < best else 0.0)
        for sp in spreads:
            raw.append((rec["m"], rec["n"], rec["k"], rec["S"], sp))
            r.append(ratio)
            z.append(zi)
    return (np.ascontiguousarray(raw, dtype=np.int32), np.ascontiguousarray(r, dtype=np.float32),
            np.ascontiguousarray(z, dtype=np.float32))


# ----------------------------------------------------------------------------------- training

def nweights() -> int:
    from . import lib as _lib
    return int(_lib().libxstream_b200_mlp_nweights())


def init_weights(seed: int = 7) -> np.ndarray:
    """He-normal weights, zero biases (layout W1[F][64], b1, W2[64][64], b2, W3[64][K + 1], b3: K
    configuration logits and the Ozaki logit)."""
    g = np.random.Generator(np.random.PCG64(seed))
    out = K + 1
    parts = [g.normal(0, math.sqrt(2 / NFEAT), NFEAT * 64), np.zeros(64), g.normal(0, math.sqrt(2 / 64), 64 * 64), np.zeros(64),
             g.normal(0, math.sqrt(1 / 64), 64 * out), np.zeros(out)]
    return np.concatenate(parts).astype(np.float32)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def train(raw: np.ndarray, r: np.ndarray, z: np.ndarray, steps: int = 3000, lr: float = 3e-3,
          weights: np.ndarray | None = None, seed: int = 7):
    """Trains on the device; returns (weights, loss per step)."""
    from . import lib as _lib
    w = (init_weights(seed) if weights is None else np.array(weights, dtype=np.float32)).copy()
    if w.size != nweights():  # the device copies exactly nweights() floats in and out of w
        raise ValueError(f"weights hold {w.size} floats, the network {nweights()}")
    hist = np.zeros(max(steps, 1), dtype=np.float32)
    rc = _lib().libxstream_b200_mlp_train(_ptr(raw), _ptr(r), _ptr(z), raw.shape[0], steps, lr, _ptr(w), _ptr(hist))
    if rc != 0:
        raise RuntimeError(f"mlp_train failed ({rc})")
    return w, hist[:steps]


def device_grad(w: np.ndarray, raw: np.ndarray, r: np.ndarray, z: np.ndarray):
    from . import lib as _lib
    w = np.ascontiguousarray(w, dtype=np.float32)
    g = np.zeros_like(w)
    loss = np.zeros(raw.shape[0], dtype=np.float32)
    rc = _lib().libxstream_b200_mlp_grad(_ptr(w), _ptr(raw), _ptr(r), _ptr(z), raw.shape[0], _ptr(g), _ptr(loss))
    if rc != 0:
        raise RuntimeError(f"mlp_grad failed ({rc})")
    return g, loss


def device_forward(w: np.ndarray, raw: np.ndarray) -> np.ndarray:
    from . import lib as _lib
    w = np.ascontiguousarray(w, dtype=np.float32)
    y = np.zeros((raw.shape[0], K + 1), dtype=np.float32)
    if _lib().libxstream_b200_mlp_forward(_ptr(w), _ptr(raw), raw.shape[0], _ptr(y)) != 0:
        raise RuntimeError("mlp_forward failed")
    return y


def device_predict(w: np.ndarray, raw: np.ndarray):
    from . import lib as _lib
    w = np.ascontiguousarray(w, dtype=np.float32)
    n = raw.shape[0]
    cfg = np.zeros(n, dtype=np.uint8)
    conf = np.zeros(n, dtype=np.float32)
    pz = np.zeros(n, dtype=np.float32)
    if _lib().libxstream_b200_mlp_predict(_ptr(w), _ptr(raw), n, _ptr(cfg), _ptr(conf), _ptr(pz)) != 0:
        raise RuntimeError("mlp_predict failed")
    return cfg.astype(np.int64), conf, pz


def install(w: np.ndarray) -> None:
    from . import lib as _lib
    w = np.ascontiguousarray(w, dtype=np.float32)
    if _lib().libxstream_b200_mlp_install(_ptr(w), w.size) != 0:
        raise RuntimeError("mlp_install failed")


def save_weights(path: Path, w: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write(f"XS_MLP {w.size}\n")
        for v in np.asarray(w, dtype=np.float32):
            f.write(f"{float(v):.9g}\n")


def load_weights(path: Path = DEFAULT_WEIGHTS) -> np.ndarray:
    with open(path) as f:
        hdr = f.readline().split()
        vals = np.array([float(x) for x in f.read().split()], dtype=np.float32)
    if hdr[0] != "XS_MLP" or int(hdr[1]) != vals.size:
        raise ValueError(f"{path}: not a predictor weight file")
    return vals


# --------------------------------------------------------------------------------- evaluation

def default_config(m: int, n: int, k: int) -> int:
    """The library's default heuristic (the method without the predictor), restated: least padded
    split of ceil(dim/8) fragments into <= 4 per warp; KP = 2 when k <= 8 else 4, or the KP of the
    shape-specialised kernel with those tiles when one exists (queried from the library). Removes an
    installed predictor first (the library installs the shipped one when it initialises), since the
    library's lookup would otherwise return the predictor's choice."""
    from . import lib as _lib
    _lib().libxstream_b200_mlp_install(None, 0)
    out = (ctypes.c_int * 6)()
    _lib().libxstream_b200_get_params(m, n, k, 10000, out)
    return config_index(out[1], out[2], out[3])


def evaluate(recs: list[dict], predict_fn, default_fn=default_config, minconf: float = 0.0) -> dict:
    """Scores predictions on sweep records by the measured time of the chosen configuration over the
    tuned optimum; predictions below minconf confidence fall back to the exhaustive tuner (ratio 1)."""
    raw = np.array([(r["m"], r["n"], r["k"], r["S"], 40) for r in recs], dtype=np.int32)
    cfg, conf, pz = predict_fn(raw)
    ratios, dratios, fallbacks, choice_ok, choice_n = [], [], 0, 0, 0
    for rec, c, cf, p in zip(recs, cfg, conf, pz):
        t = rec["t"]
        best = np.nanmin(t)
        if cf < minconf:
            fallbacks += 1
            ratios.append(1.0)
        else:
            ratios.append(float(t[c] / best) if not np.isnan(t[c]) else float("inf"))
        dc = default_fn(rec["m"], rec["n"], rec["k"])
        dratios.append(float(t[dc] / best) if not np.isnan(t[dc]) else float("inf"))
        if rec["oz"] is not None:
            choice_n += 1
            choice_ok += int((p >= 0.5) == (rec["oz"] < best))
    ratios, dratios = np.array(ratios), np.array(dratios)
    return {"samples": len(recs), "within_5pct": float(np.mean(ratios <= 1.05)),
            "mean_ratio": float(np.mean(ratios)), "geomean_ratio": float(np.exp(np.mean(np.log(ratios)))),
            "max_ratio": float(np.max(ratios)), "fallback_rate": fallbacks / max(1, len(recs)),
            "default_within_5pct": float(np.mean(dratios <= 1.05)), "default_mean_ratio": float(np.mean(dratios)),
            "default_geomean_ratio": float(np.exp(np.mean(np.log(dratios)))),
            "choice_accuracy": (choice_ok / choice_n) if choice_n else None, "choice_samples": choice_n}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("sweep")
    s.add_argument("--out", type=Path, default=DEFAULT_SWEEP)
    s.add_argument("--shapes", type=int, default=4000)
    s.add_argument("--heldout", type=int, default=300)
    s.add_argument("--minutes", type=float, default=12.0)
    s.add_argument("--seed", type=int, default=2025)
    s.add_argument("--start", type=int, default=0, help="first training shape (continue an earlier sweep)")
    s.add_argument("--no-heldout", action="store_true", help="skip the held-out shapes (tuned by an earlier sweep)")
    s.add_argument("--fma-only", action="store_true", help="only the shapes the FMA kernel takes")
    t = sub.add_parser("train")
    t.add_argument("--sweep", type=Path, default=DEFAULT_SWEEP)
    t.add_argument("--override", type=Path, default=DEFAULT_SWEEP_FMA, help="rows replacing the sweep's (none: '')")
    t.add_argument("--out", type=Path, default=DEFAULT_WEIGHTS)
    t.add_argument("--steps", type=int, default=3000)
    t.add_argument("--lr", type=float, default=3e-3)
    e = sub.add_parser("eval")
    e.add_argument("--sweep", type=Path, default=DEFAULT_SWEEP)
    e.add_argument("--override", type=Path, default=DEFAULT_SWEEP_FMA, help="rows replacing the sweep's (none: '')")
    e.add_argument("--weights", type=Path, default=DEFAULT_WEIGHTS)
    e.add_argument("--minconf", type=float, default=0.0)
    a = ap.parse_args(argv)
    if a.cmd == "sweep":
        held = random_shapes(a.heldout, a.seed + 1)
        train_shapes = random_shapes(a.shapes, a.seed, exclude=set(held))
        rows = sweep(a.out, train_shapes[a.start:], [] if a.no_heldout else held, a.minutes, fma_only=a.fma_only)
        print(json.dumps({"rows": rows, "out": str(a.out)}))
    elif a.cmd == "train":
        ov = a.override if a.override and str(a.override) and Path(a.override).exists() else None
        recs = [r for r in load_sweep(a.sweep, ov) if r["split"] == "train"]
        # choose steps / learning rate on a validation tenth of the training shapes, then retrain on all
        shapes = sorted({(r["m"], r["n"], r["k"]) for r in recs})
        g = np.random.Generator(np.random.PCG64(99))
        val = {shapes[i] for i in g.choice(len(shapes), len(shapes) // 10, replace=False)}
        fit = [r for r in recs if (r["m"], r["n"], r["k"]) not in val]
        vrecs = [r for r in recs if (r["m"], r["n"], r["k"]) in val]
        raw, r, z = build_dataset(fit)
        search = []
        for steps, lr in ((a.steps, a.lr), (2 * a.steps, a.lr), (2 * a.steps, a.lr / 3)):
            w, hist = train(raw, r, z, steps, lr)
            sc = evaluate(vrecs, lambda q, w=w: device_predict(w, q), default_fn=lambda m, n, k: 0)
            search.append({"steps": steps, "lr": lr, "loss_last": float(hist[-1]), "val_within_5pct": sc["within_5pct"],
                           "val_geomean_ratio": sc["geomean_ratio"]})
        best = max(search, key=lambda e: (e["val_within_5pct"], -e["val_geomean_ratio"]))
        raw, r, z = build_dataset(recs)
        w, hist = train(raw, r, z, best["steps"], best["lr"])
        save_weights(a.out, w)
        print(json.dumps({"samples": int(raw.shape[0]), "search": search, "chosen": best, "loss_first": float(hist[0]),
                          "loss_last": float(hist[-1]), "out": str(a.out)}))
    else:
        ov = a.override if a.override and str(a.override) and Path(a.override).exists() else None
        recs = [r for r in load_sweep(a.sweep, ov) if r["split"] == "heldout"]
        w = load_weights(a.weights)
        print(json.dumps(evaluate(recs, lambda raw: device_predict(w, raw), minconf=a.minconf)))


if __name__ == "__main__":
    main()
