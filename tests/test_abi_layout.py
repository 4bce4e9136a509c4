"""The ctypes mirrors of the C-ABI structs (qmbcuda_b200/_capi.py) against
include/qmb_b200.h: a C program compiled here prints each struct's size and
each field's offset, which must equal the ctypes layout (no GPU needed)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from qmbcuda_b200 import _capi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PAIRS = [("Geometry", "qmb_geometry"), ("SectorDesc", "qmb_sector_desc"), ("SectorInfo", "qmb_sector_info"),
         ("Terms", "qmb_terms"), ("HamInfo", "qmb_ham_info"), ("LanczosOpts", "qmb_lanczos_opts"),
         ("LanczosResult", "qmb_lanczos_result"), ("BatchDesc", "qmb_batch_desc"), ("BatchInfo", "qmb_batch_info")]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_struct_layouts_match_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "qmb_b200.h"', 'int main(void) {']
    want = {}
    for py, c in PAIRS:
        cls = getattr(A, py)
        lines.append(f'    printf("{py} size %zu\\n", sizeof({c}));')
        want[f"{py} size"] = C.sizeof(cls)
        for f in cls._fields_:
            name = f[0]
            lines.append(f'    printf("{py}.{name} %zu\\n", offsetof({c}, {name}));')
            want[f"{py}.{name}"] = getattr(cls, name).offset
    lines += ['    return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        k, v = line.rsplit(" ", 1)
        got[k] = int(v)
    assert got == want
