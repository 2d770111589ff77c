"""The public header compiles as C99 and as C++, and the ctypes structures of the Python
binding have the C structures' layout (every field's offset, every struct's size), as gcc
lays them out on this host. A binding whose layout drifted from the header would pass
wrong values to the library without any error."""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from cfd_solver_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]

STRUCTS = {
    "cfd_grid": _lib.CfdGrid,
    "cfd_grid_spec": _lib.CfdGridSpec,
    "cfd_params": _lib.CfdParams,
    "cfd_step_stats": _lib.CfdStepStats,
    "cfd_request": _lib.CfdRequest,
    "cfd_result": _lib.CfdResult,
    "cfd_serve_config": _lib.CfdServeConfig,
    "cfd_serve_stats": _lib.CfdServeStats,
}

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None,
                                reason="no host compiler")


def _layout_program():
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "cfd_b200.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} . %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    return "\n".join(lines) + "\n"


def test_header_compiles_as_c_and_cxx(tmp_path):
    src_c = tmp_path / "h.c"
    src_c.write_text('#include "cfd_b200.h"\nint cfd_header_probe;\n')
    src_cc = tmp_path / "h.cc"
    src_cc.write_text('#include "cfd_b200.h"\nint (*probe)(cfd_batch*, int) = cfd_batch_step;\n')
    inc = f"-I{ROOT / 'include'}"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", inc, "-c",
                    str(src_c), "-o", str(tmp_path / "h_c.o")], check=True)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", inc, "-c", str(src_cc),
                    "-o", str(tmp_path / "h_cc.o")], check=True)


def test_ctypes_structures_match_the_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(_layout_program())
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    c_layout = {}
    for line in out.splitlines():
        s, f, v = line.split()
        c_layout[(s, f)] = int(v)
    bad = []
    for cname, cls in STRUCTS.items():
        if ctypes.sizeof(cls) != c_layout[(cname, ".")]:
            bad.append(f"sizeof {cname}: ctypes {ctypes.sizeof(cls)}, C {c_layout[(cname, '.')]}")
        for fname, _ in cls._fields_:
            off = getattr(cls, fname).offset
            if off != c_layout[(cname, fname)]:
                bad.append(f"{cname}.{fname}: ctypes {off}, C {c_layout[(cname, fname)]}")
    assert not bad, bad


def test_every_header_struct_has_a_binding():
    txt = (ROOT / "include" / "cfd_b200.h").read_text()
    defined = set(re.findall(r"typedef struct (cfd_[a-z_]+) \{", txt))
    assert defined == set(STRUCTS), defined ^ set(STRUCTS)
