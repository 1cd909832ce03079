"""The ctypes mirrors of the C-ABI's structures have the layout include/subfv.h gives
them: a small C program built with the host compiler prints each field's offset and the
structure's size, and the Python mirror must agree field by field."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _c_layout(tmp_path, struct, fields):
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "subfv.h"', 'int main(void) {',
             f'  printf("size %zu\\n", sizeof({struct}));']
    lines += [f'  printf("{f} %zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ['  return 0;', '}']
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    return {k: int(v) for k, v in (line.split() for line in out if line)}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
@pytest.mark.parametrize("struct,mirror", [("subfv_ns_cfg", "NsCfgC"), ("subfv_implicit_stats", "ImplicitStats")])
def test_struct_layout_matches_header(tmp_path, struct, mirror):
    from subfv_b200 import ns
    cls = getattr(ns, mirror)
    names = [f[0] for f in cls._fields_]
    lay = _c_layout(tmp_path, struct, names)
    assert lay["size"] == C.sizeof(cls)
    for n in names:
        assert lay[n] == getattr(cls, n).offset, n
