"""include/olb_b200.h compiles as C99 and as C++17 (the language of OpenLB's host
side), and the ctypes mirrors in openlb_b200/_abi.py have the header's struct
sizes and field offsets, so a binding written from either agrees byte for byte."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from openlb_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "olb_b200.h"

STRUCTS = {
    "olb_b200_desc": _abi.Desc,
    "olb_b200_dyn_params": _abi.DynParams,
    "olb_b200_stats": _abi.Stats,
    "olb_b200_tuning": _abi.Tuning,
    "olb_b200_ensemble_desc": _abi.EnsembleDesc,
    "olb_b200_instance_desc": _abi.InstanceDesc,
}


def layout_program() -> str:
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "olb_b200.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("  return 0;\n}")
    return "\n".join(lines) + "\n"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_mirrors_match_the_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(layout_program())
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{HEADER.parent}", str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in STRUCTS.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_header_compiles_as_cxx17(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text('#include "olb_b200.h"\n'
                   "static_assert(sizeof(olb_b200_dyn_params) == 112, \"ABI v3 dynamics entry\");\n"
                   "int probe() { olb_b200_desc d{}; d.q = 19; return olb_b200_abi_version() + d.q; }\n")
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", f"-I{HEADER.parent}", str(src)],
                   check=True, capture_output=True, text=True)
