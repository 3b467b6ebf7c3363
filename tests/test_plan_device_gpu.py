"""Plan construction with the dyadic plan's atom-image x target-row test on the GPU
(a43g_plan_build_device) gives every array of the host construction (a43g_plan_build), which
the plan parity tests pin to the reference: the test geometries, the workloads and the two
benchmark cells (the 16^3 cell of the contour and the wrapped 32^3 cell with 256 atoms)."""
import time

import numpy as np
import pytest

from helpers import GEOMETRIES
from angstromcube_b200 import green_function as gf, workloads

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def same_plans(g):
    a = gf.construct_Green_function(g).export()
    b = gf.construct_Green_function(g, on_device=True).export()
    assert sorted(a) == sorted(b)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    return a


@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_device_plan_matches_host_plan(name):
    same_plans(GEOMETRIES[name]())


@pytest.mark.parametrize("name", ["periodic4_1atom", "periodic16_64atoms_s2x2x2", "wrapped32_256atoms"])
def test_device_plan_matches_host_plan_workloads(name):
    g = workloads.make(name).geometry
    t0 = time.perf_counter()
    gf.construct_Green_function(g)
    t1 = time.perf_counter()
    gf.construct_Green_function(g, on_device=True)
    t2 = time.perf_counter()
    e = same_plans(g)
    assert len(e["AtomImageIndex"]) > 0
    print("%s: host %.3f s, device test %.3f s" % (name, t1 - t0, t2 - t1))
