"""Concurrent LIBSMM calls from several host threads, each on its own stream (run by
tests/test_threads_gpu.py in a fresh process, so that the threads also race on the library's lazy
initialisation and on first-time parameter lookups of their shapes).

libsmm_acc_is_thread_safe() returns 1, as the reference does under OpenMP
(samples/smm/smm_acc.c:484-491), where DBCSR's threads call libsmm_acc_process and
libsmm_acc_transpose concurrently on different streams and the reference serialises argument
binding with per-key locks (samples/smm/smm_kernel.c:91-113). Here every thread:
  - uploads its pools, transposes its B pool with libsmm_acc_transpose (checked bit for bit),
  - runs libsmm_acc_process on stacks of several shapes (some shared with other threads, some its
    own, none looked up before in this process), accumulating twice into the same C,
  - downloads C; the main thread then checks every C against the CPU oracle (relative max-norm error
    per C block <= 1e-13).
Prints one JSON line with the worst error and exits 0 when every check passed.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from libxstream_b200 import acc as A  # noqa: E402
from libxstream_b200 import workloads as W  # noqa: E402

TOL = 1e-13
SHARED = [(23, 23, 23), (5, 7, 9), (13, 4, 16), (32, 32, 32), (9, 9, 9)]
OWN = [(7, 11, 3), (45, 45, 45), (16, 26, 5), (64, 3, 80), (22, 22, 23), (4, 4, 4), (26, 13, 40), (80, 80, 5)]


def plan(nthreads: int) -> list[list[tuple[int, int, int, int, int]]]:
    """Per thread: (m, n, k, S, seed) of its stacks; every thread sees the shared shapes in a rotated
    order, so several threads ask for the same new shape at about the same time."""
    out = []
    for t in range(nthreads):
        shapes = SHARED[t % len(SHARED):] + SHARED[: t % len(SHARED)] + [OWN[t % len(OWN)]]
        out.append([(m, n, k, 1500 + 700 * ((t + i) % 5), 9000 + 100 * t + i) for i, (m, n, k) in enumerate(shapes)])
    return out


def worker(t, work, cases, results, errors, start):
    try:
        stream = A.Stream(f"thread{t}")
        start.wait()
        for idx, (m, n, k, S, seed) in enumerate(work):
            case = cases[(t, idx)]
            da = A.DevBuf.from_array(case.a, stream)
            db = A.DevBuf.from_array(case.b, stream)
            trs = A.DevBuf.from_array(np.arange(case.nb, dtype=np.int32) * (k * n), stream)
            ds = A.DevBuf.from_array(case.stack, stream)
            dc = A.DevBuf(case.nc * m * n * 8)
            dc.zero(stream)
            rc_t = A.transpose(trs, 0, case.nb, db, k, n, stream)
            rc_p = A.process(ds, case.S, da, db, dc, m, n, k, stream)
            rc_q = A.process(ds, case.S, da, db, dc, m, n, k, stream)  # accumulate a second time
            bt = db.download(np.zeros(case.b.size), stream)
            got = dc.download(np.zeros(case.nc * m * n), stream)
            stream.sync()
            results[(t, idx)] = (rc_t, rc_p, rc_q, bt, got)
            for b in (da, db, trs, ds, dc):
                b.free()
        stream.destroy()
    except Exception as exc:  # reported by the main thread
        errors.append(f"thread {t}: {exc!r}")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=6)
    args = ap.parse_args()
    L = A.lib()
    if L.c_dbcsr_acc_init() != 0:  # as DBCSR: LIBSMM itself initialises on the first stack call
        print(json.dumps({"ok": False, "error": "c_dbcsr_acc_init failed"}))
        return 1
    work = plan(args.threads)
    cases = {}
    for t, items in enumerate(work):
        for idx, (m, n, k, S, seed) in enumerate(items):
            cases[(t, idx)] = W.stack_case(m, n, k, S, 97, 89, 23, seed=seed)
    results, errors = {}, []
    start = threading.Barrier(args.threads)
    threads = [threading.Thread(target=worker, args=(t, work[t], cases, results, errors, start)) for t in range(args.threads)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    worst, bad = 0.0, list(errors)
    for key, case in cases.items():
        if key not in results:
            bad.append(f"{key}: no result")
            continue
        rc_t, rc_p, rc_q, bt, got = results[key]
        m, n, k = case.m, case.n, case.k
        if (rc_t, rc_p, rc_q) != (0, 0, 0):
            bad.append(f"{key} {m}x{n}x{k}: return codes {(rc_t, rc_p, rc_q)}")
            continue
        want_bt = case.b.reshape(case.nb, n, k).transpose(0, 2, 1).reshape(-1)  # k x n col-major -> row-major
        if not np.array_equal(bt.view(np.uint64), np.ascontiguousarray(want_bt).view(np.uint64)):
            bad.append(f"{key} {m}x{n}x{k}: transposed B differs")
        ref = np.zeros(case.nc * m * n)
        oracle.smm(case.stack, case.a, case.b, ref, m, n, k, b_rowmajor=False)
        oracle.smm(case.stack, case.a, case.b, ref, m, n, k, b_rowmajor=False)
        err = oracle.block_relerr(got, ref, m * n)
        worst = max(worst, err)
        if not err <= TOL:
            bad.append(f"{key} {m}x{n}x{k}: relative error {err:.3e}")
    L.c_dbcsr_acc_finalize()
    print(json.dumps({"ok": not bad, "threads": args.threads, "calls": 2 * len(cases), "worst_relerr": worst,
                      "autotune": os.environ.get("LIBXSTREAM_B200_AUTOTUNE", "0"), "problems": bad[:20]}))
    return 0 if not bad else 1


if __name__ == "__main__":
    sys.exit(main())
