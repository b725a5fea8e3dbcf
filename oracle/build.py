"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/smm_oracle.c`` into ``oracle/_build/liboracle.so`` with OpenMP and
``-ffp-contract=off`` so sums and products round exactly as written in the C source.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "smm_oracle.c"
OUT = HERE / "_build" / "liboracle.so"


def build(force: bool = False) -> Path:
    if OUT.exists() and not force and OUT.stat().st_mtime >= max(SRC.stat().st_mtime, Path(__file__).stat().st_mtime):
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = ["gcc", "-O3", "-march=native", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-Wall", "-o", str(tmp), str(SRC), "-lm"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + proc.stdout + proc.stderr)
        raise RuntimeError("oracle build failed")
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
