"""Generates the golden fixtures of the stack path from the reference's own kernels
(samples/smm/kernels/multiply.cl and transpose.cl compiled as host C by oracle/ref_build.py).

Each fixture stores the case parameters, the SHA-256 of its generated inputs (the inputs themselves
are regenerated from the seeded generator in libxstream_b200/workloads.py, which is deterministic) and
the reference kernel's output. Run in the build container, where the reference tree is present:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from libxstream_b200 import workloads as W  # noqa: E402
from oracle import ref_build as R  # noqa: E402

# (m, n, k, S, pool blocks, C blocks, seed, zipf, values, reference kernel configuration)
SMM_CASES = [
    (23, 23, 23, 3000, 64, 32, 11, 1.1, "uniform", {"bs": 8}),
    (5, 13, 7, 2000, 48, 16, 12, 1.1, "uniform", {"bs": 4, "reg_b": True}),
    (45, 32, 9, 1000, 40, 20, 13, 1.1, "spread", {"bm": 8, "bn": 4, "bs": 16, "reg_a": True, "reg_b": True}),
    (64, 64, 64, 300, 24, 12, 14, 2.0, "uniform", {"bs": 8}),
    (1, 1, 1, 500, 30, 10, 15, 1.1, "uniform", {}),
    (16, 9, 33, 2500, 60, 8, 16, 1.1, "spread", {"bm": 4, "bn": 3, "bs": 4}),
]
TRANSPOSE_CASES = [(23, 23, 50, 21), (13, 7, 40, 22), (64, 64, 8, 23), (5, 80, 30, 24)]


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def smm_case(spec):
    m, n, k, S, npool, nc, seed, zipf, values, _ = spec
    return W.stack_case(m, n, k, S, npool, npool, nc, seed=seed, zipf_s=zipf, values=values)


def transpose_input(spec):
    m, n, nblk, seed = spec
    g = W.rng(seed)
    data = g.uniform(-1, 1, size=nblk * m * n)
    data[:: 7] = np.nan  # NaN payloads must survive the bit copy
    trs = (g.permutation(nblk) * (m * n)).astype(np.int32)
    return data, trs


def main():
    meta = {"smm": [], "transpose": []}
    arrays = {}
    for i, spec in enumerate(SMM_CASES):
        case = smm_case(spec)
        m, n, k = case.m, case.n, case.k
        f = R.multiply(m, n, k, **spec[-1])
        c = np.zeros(case.nc * m * n)
        st = np.ascontiguousarray(case.stack, dtype=np.int32)
        bt = case.b_rowmajor()
        f(st.ctypes.data, case.S, 0, case.a.ctypes.data, bt.ctypes.data, c.ctypes.data)
        arrays[f"smm{i}_c"] = c
        meta["smm"].append({"spec": list(spec[:-1]), "kernel": spec[-1], "inputs_sha256": digest(case.stack, case.a, case.b)})
    for i, spec in enumerate(TRANSPOSE_CASES):
        data, trs = transpose_input(spec)
        out = data.copy()
        R.transpose(spec[0], spec[1])(trs.ctypes.data, 0, spec[2], out.ctypes.data)
        arrays[f"tr{i}_out"] = out
        meta["transpose"].append({"spec": list(spec), "inputs_sha256": digest(data, trs)})
    np.savez_compressed(HERE / "stack_path_reference.npz", **arrays)
    (HERE / "stack_path_reference.json").write_text(json.dumps(meta, indent=1) + "\n")
    print(f"{len(SMM_CASES)} stack cases, {len(TRANSPOSE_CASES)} transpose cases")


if __name__ == "__main__":
    main()
