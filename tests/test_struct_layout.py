"""The ctypes mirrors in gpsm_b200/_lib.py have the C structs' layout: every
field at the same offset and every struct the same size, as a C compiler
lays out include/gpsm.h. A mismatch would make Python read or pass the
wrong bytes without any error."""
import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import ROOT
from gpsm_b200 import _lib

STRUCTS = {
    "gpsm_match_opts": _lib.MatchOpts,
    "gpsm_match_info": _lib.MatchInfo,
    "gpsm_batch_info": _lib.BatchInfo,
    "gpsm_request_info": _lib.RequestInfo,
    "gpsm_tuning": _lib.Tuning,
}


def _c_layout(tmp_path):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "gpsm.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    return {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_mirrors_match_the_c_layout(tmp_path):
    c = _c_layout(tmp_path)
    for cname, py in STRUCTS.items():
        assert c[(cname, "size")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert c[(cname, field)] == getattr(py, field).offset, (cname, field)
