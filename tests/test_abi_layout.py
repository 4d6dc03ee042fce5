"""The ctypes mirrors of the C ABI's structs (bachelors_b200/_lib.py) have the header's layout:
a small C program built against include/fmmcuda.h prints every field's offset and each struct's
size, and they must equal the ctypes ones (no GPU, gcc only)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from bachelors_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {"fmm_config": _lib.FmmConfig, "fmm_stats": _lib.FmmStats, "fmm_tuning": _lib.FmmTuning}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_struct_layouts_match_header(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "fmmcuda.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'   printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'   printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["   return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        parts = line.split()
        got[tuple(parts[:-1])] = int(parts[-1])
    for cname, cls in STRUCTS.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
