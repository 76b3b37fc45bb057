"""The ctypes mirrors of the C-ABI structs (xfluid_b200/_lib.py) match
include/xfp.h field for field: a probe compiled against the header with the
host C compiler prints every field's offset and each struct's size, and those
must equal the ctypes layout.  A mismatch would let the library write past a
Python-allocated stats buffer."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

from xfluid_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]

STRUCTS = {"xfp_options": _lib.XfpOptions, "xfp_stats": _lib.XfpStats, "xfp_scene": _lib.XfpScene}


def _probe_source():
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "xfp.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    return "\n".join(lines) + "\n"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_ctypes_structs_match_the_header(tmp_path):
    src = tmp_path / "probe.c"
    exe = tmp_path / "probe"
    src.write_text(_probe_source())
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line.strip():
            cname, key, val = line.split()
            got[(cname, key)] = int(val)
    for cname, py in STRUCTS.items():
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
