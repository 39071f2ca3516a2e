"""The ctypes mirrors of the C-ABI structs (cbc_b200/_lib.py) have the same
size and field offsets as the structs in include/cbc_b200.h, as compiled by
the host C compiler.  A field added on one side only would silently shift
every later field of every call; this catches it without a GPU."""
import ctypes
import os
import shutil
import subprocess

import pytest

from cbc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = [_lib.cbc_spec, _lib.cbc_buffers, _lib.cbc_solve_stats, _lib.cbc_ensemble, _lib.cbc_work,
           _lib.cbc_env_io, _lib.cbc_precompute_consts]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_ctypes_structs_match_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cbc_b200.h"', "int main(void) {"]
    for st in STRUCTS:
        name = st.__name__
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for fname, _ in st._fields_:
            lines.append(f'  printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                              check=True).stdout.splitlines())
    for st in STRUCTS:
        name = st.__name__
        assert int(out[f"{name} size"]) == ctypes.sizeof(st), name
        for fname, _ in st._fields_:
            assert int(out[f"{name}.{fname}"]) == getattr(st, fname).offset, f"{name}.{fname}"
