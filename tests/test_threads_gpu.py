"""Thread safety of the LIBSMM ABI (libsmm_acc_is_thread_safe() == 1): several host threads issue
libsmm_acc_process and libsmm_acc_transpose at once on their own streams, with shapes that are new to
the process, with the exhaustive autotuner off and on (LIBXSTREAM_B200_AUTOTUNE, read once per
process, hence a fresh process per setting). Every C is checked against the CPU oracle at <= 1e-13
and every transposed B bit for bit (tests/threaded_calls.py). Reference: samples/smm/smm_acc.c:484-491,
samples/smm/smm_kernel.c:91-113."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent


@pytest.mark.parametrize("autotune", ["0", "1"])
def test_concurrent_calls_from_host_threads(acc, autotune):
    env = dict(os.environ, LIBXSTREAM_B200_AUTOTUNE=autotune, LIBXSTREAM_B200_NOBUILD="1")
    proc = subprocess.run([sys.executable, str(HERE / "threaded_calls.py"), "--threads", "8"], env=env,
                          capture_output=True, text=True, timeout=900)
    lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
    assert lines, proc.stdout[-2000:] + proc.stderr[-2000:]
    out = json.loads(lines[-1])
    assert proc.returncode == 0 and out["ok"], out
    assert out["worst_relerr"] <= 1e-13
