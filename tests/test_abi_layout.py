"""The ctypes mirrors of the C ABI's structs (vnlbgpu_lib.py) against the
headers themselves: a small C program, compiled here with gcc against
include/vnlbgpu.h and include/vnlbgpu_diag.h, prints each struct's size and
every field's offset, and the mirrors must agree field by field (a struct
that grows in the header and not in the binding would shift every later
argument a plugin passes)."""
import ctypes
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "vapoursynth-vnlb_b200"))

import vnlbgpu_lib as lib  # noqa: E402

MIRRORS = {
    "vnlbgpu_params": lib.Params,
    "vnlbgpu_stats": lib.Stats,
    "vnlbgpu_mvtools_analysis": lib.MVToolsAnalysis,
    "vnlbgpu_diag_row": lib.DiagRow,
}


def c_layout(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "vnlbgpu.h"', '#include "vnlbgpu_diag.h"',
             "int main(void) {"]
    for cname, mirror in MIRRORS.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in mirror._fields_:
            lines.append(f'    printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {tuple(line.split()[:2]): int(line.split()[2]) for line in out.splitlines()}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is needed to read the header layout")
def test_ctypes_mirrors_match_the_headers(tmp_path):
    layout = c_layout(tmp_path)
    for cname, mirror in MIRRORS.items():
        assert layout[(cname, "size")] == ctypes.sizeof(mirror), cname
        for field, _ in mirror._fields_:
            assert layout[(cname, field)] == getattr(mirror, field).offset, (cname, field)
