"""The product's C++ plan builder against the reference's own plan construction
(src/green_function.cxx:357-1068, src/kinetic_plan.cxx:38-322, src/dyadic_plan.cxx:159-583):
every array bit-identical.  CPU only: plans are host data."""
import os

import numpy as np
import pytest

import oracle
from helpers import GEOMETRIES, inputs_for, product_plan, reference_plan
from angstromcube_b200 import green_function as gf
from angstromcube_b200 import workloads

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU build (oracle/_ref) not built")


def compare(ra, pa):
    keys = sorted(set(ra) & set(pa))
    assert len(keys) >= 30
    bad = [k for k in keys if not (ra[k].shape == pa[k].shape and np.array_equal(ra[k], pa[k]))]
    assert not bad, "arrays differ from the reference plan: %s" % bad


@needs_ref
@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_plan_matches_reference(name):
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    ref = reference_plan(g, Vc, mats, offs, E, k, dVol)
    pl = product_plan(g, Vc, mats, offs, E, k, dVol)
    assert ref.sizes["nnzb"] == pl.sizes["nnzb"] > 0
    compare(ref.export(), pl.export())


@needs_ref
@pytest.mark.parametrize("name", ["periodic4_1atom", "periodic4_1atom_iso", "periodic4_noatom"])
def test_plan_matches_reference_workloads(name):
    w = workloads.make(name)
    ref = oracle.RefGreen(w.geometry)
    pl = gf.construct_Green_function(w.geometry)
    compare(ref.export(), pl.export())


@needs_ref
@pytest.mark.parametrize("name", ["periodic16_64atoms", "periodic16_64atoms_s1x1x1", "wrapped32_256atoms"])
def test_plan_matches_reference_benchmark_cells(name):
    """The benchmark cells themselves: the dense periodic 16^3-cube cell with 64 atoms (16 and
    one source cubes) and the wrapped 32^3-cube cell with 256 atoms and 32 source cubes
    (300,960 blocks, the truncation sphere with the 8/27-corner test of the reference's
    default build)."""
    w = workloads.make(name)
    ref = oracle.RefGreen(w.geometry)
    pl = gf.construct_Green_function(w.geometry)
    assert ref.sizes["nnzb"] == pl.sizes["nnzb"]
    if name == "wrapped32_256atoms":
        assert pl.sizes["nnzb"] == 300960 and pl.sizes["nCols"] == 32
    compare(ref.export(), pl.export())


def test_plan_matches_golden():
    """Committed plan arrays generated by the reference (tests/golden/make_golden.py)."""
    path = os.path.join(GOLDEN, "plan_wrap6.npz")
    gold = dict(np.load(path))
    g = GEOMETRIES_GOLDEN()
    pl = gf.construct_Green_function(g)
    pa = pl.export()
    for k, v in gold.items():
        if k.startswith("plan_"):
            kk = k[len("plan_"):]
            assert np.array_equal(pa[kk], v), kk


def GEOMETRIES_GOLDEN():
    from helpers import geometry
    return geometry((6, 6, 6), (1, 1, 1), 2.4, (2, 2, 1), 4, 3, seed=11)


def test_dense_periodic_sizes():
    """A periodic direction whose cell is shorter than the truncation diameter is not truncated
    (src/green_function.cxx:515-532): the 16^3-cube cell with 16 sources is dense."""
    g = workloads.make("periodic16_64atoms").geometry
    pl = gf.construct_Green_function(g)
    assert pl.sizes["nnzb"] == 16 ** 3 * 16
    assert pl.sizes["nRows"] == 16 ** 3 and pl.sizes["nCols"] == 16
    assert pl.sizes["FD_range0"] == 4


def test_source_count_limit():
    """65535 source cubes are the most a plan takes (uint16 column indices, one CTA row per
    source in the per-column kernels): 65536 are refused when the plan is built."""
    g = workloads.Geometry((4 * 256, 4 * 256, 4), (1, 1, 1), (0.25,) * 3, 0.5, (-1, -1, -1))
    with pytest.raises(RuntimeError, match="65535"):
        gf.construct_Green_function(g)


def test_invalid_geometry_is_an_error():
    g = workloads.Geometry((6, 8, 8), (1, 1, 1), (0.25,) * 3, 3.0, (1, 1, 1))
    with pytest.raises(RuntimeError, match="multiples of 4"):
        gf.construct_Green_function(g)
    g = workloads.Geometry((8, 8, 8), (1, 1, 1), (0.25,) * 3, 3.0, (1, 1, 1))
    p = gf.construct_Green_function(g)
    with pytest.raises(RuntimeError, match="0.503"):
        gf.update_phases(p, [0.6, 0, 0])
