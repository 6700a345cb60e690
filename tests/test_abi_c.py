"""The C ABI from plain C: `include/sck.h` and `include/sck_made.h` compile as C99 with every warning an error,
a C program links `libsckb200.so`, and the struct sizes it sees (sizeof in C) are the library's own and the
Python binding's — the check a cgo, JNI or N-API binding does at load time. No GPU call is made."""

from __future__ import annotations

import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from spin_colour_kernel_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]

PROGRAM = r"""
#include <stdio.h>
#include "sck.h"
#include "sck_made.h"

int main(void) {
  int64_t d = 0, s = 0, b = 0, u = 0;
  if (sck_struct_sizes(&d, &s, &b, &u) != SCK_OK) return 2;
  if (d != (int64_t)sizeof(sck_system_desc) || s != (int64_t)sizeof(sck_sublattice) ||
      b != (int64_t)sizeof(sck_bond) || u != (int64_t)sizeof(sck_buffers)) return 3;
  if (sck_abi_version() != SCK_ABI_VERSION) return 4;
  if (sck_plan_create(NULL, 1, SCK_MODE_F32, NULL) == SCK_OK) return 5;        /* refused on the host */
  printf("%lld %lld %lld %lld %s\n", (long long)d, (long long)s, (long long)b, (long long)u, sck_last_error());
  return 0;
}
"""


@pytest.fixture(scope="module", autouse=True)
def _built():
    from spin_colour_kernel_b200 import build
    build.build()


def test_headers_compile_as_c_and_sizes_agree(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "abi"
    libdir = L.LIB_PATH.parent
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", f"-I{ROOT / 'include'}", str(src),
                        f"-L{libdir}", "-lsckb200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)
    d, s, b, u = (int(v) for v in run.stdout.split()[:4])
    assert [d, s, b, u] == [ctypes.sizeof(L.SystemDesc), ctypes.sizeof(L.Sublattice), ctypes.sizeof(L.Bond),
                            ctypes.sizeof(L.Buffers)]
    assert run.stdout.split(maxsplit=4)[4].strip()            # the refusal left a message
