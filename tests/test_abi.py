"""CPU tests of the C-ABI library: it loads, exports every declared symbol, and its host-side rules
(suitability, no-op cases, parameter table) behave like the reference without touching a GPU."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import pytest

import libxstream_b200 as xs

ROOT = Path(__file__).resolve().parent.parent


def declared_functions() -> set[str]:
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"^\s*typedef[^;]*;", "", text, flags=re.M | re.S)  # function-pointer types are not symbols
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_builds_and_loads():
    lib = xs.lib()
    assert xs.LIB_PATH.exists()
    assert lib.libsmm_acc_is_thread_safe() == 1


def test_exports_every_declared_symbol():
    declared = declared_functions()
    # the 26 DBCSR ACC names of the reference (.abi.txt:1-26) and the LIBSMM entry points
    for name in ("c_dbcsr_acc_init", "c_dbcsr_acc_memset_zero", "c_dbcsr_acc_stream_wait_event", "libsmm_acc_process",
                 "libsmm_acc_transpose", "libsmm_acc_init", "libsmm_acc_finalize", "libsmm_acc_is_thread_safe",
                 "c_calculate_norms"):
        assert name in declared
    assert len([d for d in declared if d.startswith("c_dbcsr_acc_")]) == 26
    out = subprocess.run(["nm", "-D", "--defined-only", str(xs.LIB_PATH)], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    missing = sorted(declared - exported)
    assert not missing, missing
    # and the ctypes binding table covers them all
    assert declared <= set(xs.SIGNATURES)


def test_suitability_rules():
    lib = xs.lib()
    f = lib.libxstream_b200_process_suitable
    assert f(1, 3, 30000, 23, 23, 23, 80) == 1
    assert f(0, 3, 30000, 23, 23, 23, 80) == 0      # inhomogeneous
    assert f(1, 3, 30000, 81, 80, 23, 80) == 0      # m*n > max_kernel_dim^2
    assert f(1, 3, 30000, 80, 80, 200, 80) == 1     # k may exceed max_kernel_dim
    assert f(1, 1, 30000, 23, 23, 23, 80) == 0      # FP32: host fallback
    assert f(1, 3, 0, 23, 23, 23, 80) == 0


def test_process_returns_minus_one_for_unhandled_stacks_without_gpu():
    lib = xs.lib()
    # inhomogeneous, too large, FP32, complex: -1 (host fallback) for non-empty stacks
    assert lib.libsmm_acc_process(None, None, 10, 3, None, None, None, 23, 23, 23, 80, 0, None, None) == -1
    assert lib.libsmm_acc_process(None, None, 10, 3, None, None, None, 90, 90, 23, 80, 1, None, None) == -1
    assert lib.libsmm_acc_process(None, None, 10, 1, None, None, None, 23, 23, 23, 80, 1, None, None) == -1
    assert lib.libsmm_acc_process(None, None, 10, 7, None, None, None, 23, 23, 23, 80, 1, None, None) == -1
    # an empty stack is a successful no-op
    assert lib.libsmm_acc_process(None, None, 0, 3, None, None, None, 23, 23, 23, 80, 1, None, None) == 0


def test_transpose_noop_cases_without_gpu():
    lib = xs.lib()
    assert lib.libsmm_acc_transpose(None, 0, 10, None, 3, 1, 1, 80, None) == 0    # 1x1 block
    assert lib.libsmm_acc_transpose(None, 0, 0, None, 3, 23, 23, 80, None) == 0   # empty
    assert lib.libsmm_acc_transpose(None, 0, 10, None, 7, 23, 23, 80, None) == 0  # complex: not handled, no-op
    assert lib.libsmm_acc_transpose(None, 0, 10, None, 3, 90, 90, 80, None) == 0  # too large: no-op
    assert lib.libsmm_acc_transpose(None, -1, 10, None, 3, 23, 23, 80, None) != 0  # negative offset


def test_null_arguments_are_rejected():
    lib = xs.lib()
    assert lib.c_dbcsr_acc_dev_mem_set_ptr(None, None, 0) != 0
    assert lib.c_dbcsr_acc_get_ndevices(None) != 0
    assert lib.c_dbcsr_acc_stream_create(None, b"s", 0) != 0
    assert lib.c_dbcsr_acc_event_create(None) != 0
    assert lib.c_calculate_norms(None, 0, None, None, None, None) == 0
    assert lib.c_calculate_norms(None, 3, None, None, None, None) != 0


def test_set_ptr_is_pointer_arithmetic():
    import ctypes
    lib = xs.lib()
    p = ctypes.c_void_p()
    assert lib.c_dbcsr_acc_dev_mem_set_ptr(ctypes.byref(p), ctypes.c_void_p(0x1000), 0x28) == 0
    assert p.value == 0x1028


def test_parameter_table_roundtrip(tmp_path):
    from libxstream_b200 import acc as A
    lib = xs.lib()
    lib.libxstream_b200_clear_params()
    assert lib.libxstream_b200_mlp_install(None, 0) == 0  # default heuristic, not the learned predictor
    d = A.get_params(23, 23, 23, 30000)
    assert d["mt"] == 3 and d["nt"] == 3 and d["chunk"] == 0  # open: sized per stack by the launcher
    A.set_params(23, 23, 23, 16, 2, 3, 2, 2)
    assert A.get_params(23, 23, 23, 30000) == {"chunk": 16, "mt": 2, "nt": 3, "kp": 2, "wpb": 2, "sorted": 0}
    csv = tmp_path / "params.csv"
    csv.write_text("DEVICE;TYPEID;M;N;K;S;GFLOPS;L;MT;NT;KP;WPB\n"
                   "NVIDIA B200;3;13;13;13;30000;1000.0;8;2;2;4;4\n"
                   "NVIDIA B200;3;45;45;45;30000;1000.0;0;3;3;4;2\n")
    assert lib.libxstream_b200_load_params(str(csv).encode()) == 2
    assert A.get_params(13, 13, 13, 100)["chunk"] == 8
    p45 = A.get_params(45, 45, 45, 30000)
    assert p45["mt"] == 3 and p45["chunk"] == 0      # L=0 in the file: sized per stack by the launcher
    assert lib.libxstream_b200_load_params(b"/nonexistent.csv") == -1
    lib.libxstream_b200_clear_params()


C_CALLER = r"""
#include "dbcsr_acc.h"
#include "libsmm_acc.h"
#include "libxstream_b200.h"
#include <stdio.h>

/* the calling sequence of a DBCSR-side C caller, limited to the calls that need no GPU */
int main(void) {
  void* p = NULL;
  int (*process)(const int*, const int*, int, libsmm_acc_data_t, const void*, const void*, void*, int, int, int, int,
    c_dbcsr_acc_bool_t, void*, void*) = libsmm_acc_process; /* the reference's exact signature */
  if (1 != libsmm_acc_is_thread_safe()) return 1;
  if (0 != c_dbcsr_acc_dev_mem_set_ptr(&p, (void*)0x1000, 0x28) || (char*)p != (char*)0x1028) return 2;
  /* inhomogeneous stack: not handled, DBCSR runs its host path */
  if (-1 != process(NULL, NULL, 10, dbcsr_type_real_8, NULL, NULL, NULL, 23, 23, 23, 80, 0, NULL, NULL)) return 3;
  /* FP32: not handled either */
  if (-1 != process(NULL, NULL, 10, dbcsr_type_real_4, NULL, NULL, NULL, 23, 23, 23, 80, 1, NULL, NULL)) return 4;
  /* an empty stack and a 1x1 transpose are successful no-ops */
  if (0 != process(NULL, NULL, 0, dbcsr_type_real_8, NULL, NULL, NULL, 23, 23, 23, 80, 1, NULL, NULL)) return 5;
  if (0 != libsmm_acc_transpose(NULL, 0, 10, NULL, dbcsr_type_real_8, 1, 1, 80, NULL)) return 6;
  c_dbcsr_timeset(NULL, 0, NULL); /* weak no-op when DBCSR does not provide it */
  c_dbcsr_timestop(NULL);
  printf("ok\n");
  return 0;
}
"""


def test_c_caller_compiles_links_and_runs(tmp_path):
    """A C program built against include/*.h and linked with -lxstream_b200 (as DBCSR links it)
    compiles without warnings, resolves every symbol it uses and behaves like the reference on the
    calls that need no GPU."""
    import os
    import shutil

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    xs.lib()
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    libdir = xs.LIB_PATH.parent
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                    "-L", str(libdir), "-lxstream_b200", "-Wl,-rpath," + str(libdir)], check=True)
    env = dict(os.environ, LD_LIBRARY_PATH=str(libdir))
    out = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", (out.returncode, out.stdout, out.stderr)
