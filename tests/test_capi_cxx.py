"""The C ABI from C++ (tests/cxx/plan_from_cxx.cpp, compiled with g++ against include/a43g.h
and the library): a plan built and exported and a grid Hamiltonian written and read back, with
the same plan sizes as the Python mirror gives.  No GPU."""
import json
import os
import shutil
import subprocess

import pytest

from angstromcube_b200 import _lib, green_function as gf, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_plan_and_hamiltonian_from_cxx(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "plan_from_cxx"
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cxx", "plan_from_cxx.cpp"), "-o", str(exe),
                           "-L", libdir, "-langstromcube_b200", "-Wl,-rpath," + libdir])
    out = subprocess.run([str(exe), str(tmp_path / "Hmt.xml")], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["rows_ok"] == 1 and r["mats_ok"] == 1 and r["natoms"] == 1 and r["ng"] == [16, 16, 16]
    # the same geometry through the Python mirror
    atoms = [[0.0, 0.0, 0.0, 13, 0, 3, 0.5, 0]]
    import numpy as np
    g = workloads.Geometry((16, 16, 16), (1, 1, 1), (0.25, 0.25, 0.25), 3.0, (1, 1, 1), 4, 6.0, np.array(atoms))
    p = gf.construct_Green_function(g)
    for k in ("nnzb", "nRows", "nCols", "nAtoms"):
        assert r[k] == p.sizes[k], k
