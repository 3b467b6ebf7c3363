"""The ctypes mirrors of the C-ABI structures (angstromcube_b200/_lib.py) have the sizes and field
offsets that a C compiler gives the declarations in include/a43g.h: a small C program built with
gcc against the header prints them.  No GPU, no library call."""
import ctypes
import os
import shutil
import subprocess

import pytest

from angstromcube_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MIRRORS = [("a43g_geometry_t", _lib.Geometry), ("a43g_plan_sizes_t", _lib.PlanSizes),
           ("a43g_plan_export_t", _lib.PlanExport), ("a43g_solve_options_t", _lib.SolveOptions),
           ("a43g_solve_stats_t", _lib.SolveStats)]


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("layout")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "a43g.h"', 'int main(void) {']
    for cname, mirror in MIRRORS:
        lines.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for field, _ in mirror._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, field, cname, field))
    lines += ['return 0;', '}']
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        cname, field, value = line.split()
        table[(cname, field)] = int(value)
    return table


@pytest.mark.parametrize("cname,mirror", MIRRORS, ids=[m[0] for m in MIRRORS])
def test_struct_layout_matches_header(c_layout, cname, mirror):
    assert ctypes.sizeof(mirror) == c_layout[(cname, "sizeof")]
    for field, _ in mirror._fields_:
        assert getattr(mirror, field).offset == c_layout[(cname, field)], field
