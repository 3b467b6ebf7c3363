"""Pins of the restated oracle (oracle/green_oracle.c) before it is trusted as the checker:
  * the reference's analytic finite-difference known answers with its RMS thresholds
    (src/green_kinetic.cxx:59-226, thresholds :107-108),
  * the 15-degree phase purification, exact to 3e-16 (src/green_kinetic.cxx:228-235),
  * the reference's own action on identical inputs (oracle/_ref) and the committed golden output.
"""
import os

import numpy as np
import pytest

import oracle
from helpers import GEOMETRIES, geometry, inputs_for, reference_plan, rel_err
from angstromcube_b200 import workloads

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU build (oracle/_ref) not built")


def chain_plan(nnzb, dd, periodic, nFD, phase):
    """Plan arrays of a 1D chain of nnzb cubes along dd with unit grid spacing."""
    nh = 4
    lst = [0] * nh + list(range(1, nnzb + 1)) + [0] * nh
    if periodic:
        for i in range(nh):
            lst[nh + nnzb + i] = -(i + 1)
            lst[i] = -(nnzb - nh + i + 1)
    a = {"colindx": np.zeros(nnzb, np.uint16), "rowstart": np.array([0, nnzb], np.uint32),
         "subset": np.zeros(1, np.uint32), "rowindx": np.zeros(nnzb, np.uint32),
         "veff_index": -np.ones(nnzb, np.int32), "kinetic_prefactor": np.full(3, -0.5),
         "FD_range": np.full(3, nFD, np.int32), "phase": phase,
         "AtomStarts": np.zeros(1, np.uint32), "AtomLmax": np.zeros(0, np.int8), "AtomMatrices": np.zeros(0),
         "AtomImageStarts": np.zeros(1, np.uint32), "AtomImagePos": np.zeros((0, 4)),
         "AtomImageLmax": np.zeros(0, np.int8), "AtomImagePhase": np.zeros((0, 4)),
         "grid_spacing_dyadic": np.ones(4), "rowCubePos": np.zeros((1, 4), np.float32),
         "SHOprj_start": np.zeros(1, np.uint32), "SHOprj_col": np.zeros(0, np.uint32),
         "SHOadd_start": np.zeros(nnzb + 1, np.uint32), "SHOadd_col": np.zeros(0, np.uint32),
         "SHOsum_start": np.zeros(1, np.uint32), "SHOsum_col": np.zeros(0, np.uint32)}
    for d in range(3):
        a["lists_start%d" % d] = np.array([0, len(lst)] if d == dd else [0], np.uint32)
        a["lists%d" % d] = np.array(lst if d == dd else [], np.int32)
    return a


@pytest.mark.parametrize("dd", [0, 1, 2])
@pytest.mark.parametrize("itest", [0, 1, 2])
def test_finite_difference_known_answers(dd, itest):
    """8th order isolated (Gauss-Hermite), 16th order isolated, 8th order periodic (Bloch wave)."""
    nnzb, n1 = 35, 35 * 4
    periodic = itest > 1
    nFD = 8 if itest == 1 else 4
    border = (itest + 1) * (itest < 2)
    ph = np.zeros((3, 2, 2)); ph[:, :, 0] = 1
    if periodic:
        angles = [0.25, -1 / 3.0, 0.5]
        for d in range(3):
            ph[d], _ = oracle.restated_set_phase(angles[d])
        kvec = 2 * np.pi * angles[dd] / n1
        arg = kvec * (np.arange(n1) + 0.5)
        f = np.stack([np.cos(arg), np.sin(-arg)])
        res = 0.5 * kvec ** 2 * f
    else:
        kvec = 14.0 / n1
        xx = kvec * (np.arange(n1) - 0.5 * (n1 - 1))
        G = np.exp(-0.5 * xx * xx)
        f = np.stack([G, G * xx])
        res = 0.5 * kvec ** 2 * np.stack([G * (1 - xx * xx), G * (3 - xx * xx) * xx])
    o = oracle.RestatedOracle(chain_plan(nnzb, dd, periodic, nFD, ph), np.zeros((1, 64)), 0)
    x = np.zeros((nnzb, 2, 64, 64))
    stride = 1 << (2 * dd)
    for b in range(nnzb):
        for i4 in range(4):
            x[b, :, i4 * stride, 0] = f[:, 4 * b + i4]
    y = o.kinetic(x, dd)
    got = np.array([[y[b, ri, i4 * stride, 0] for b in range(border, nnzb - border) for i4 in range(4)] for ri in range(2)])
    ref = res[:, 4 * border: 4 * (nnzb - border)]
    dev = np.sqrt(((got - ref) ** 2).sum() / (ref ** 2).sum())
    threshold = [5.5e-9, 4.0e-14, 8e-12][itest]
    assert dev <= threshold, (dev, threshold)


def test_set_phase_purified():
    gold = np.load(os.path.join(GOLDEN, "phase.npz"))
    maxdev = 0.0
    for a, ph_ref in zip(gold["angles"], gold["phase"]):
        ph, dev = oracle.restated_set_phase(a)
        assert np.array_equal(ph, ph_ref), a
        maxdev = max(maxdev, dev)
    assert maxdev <= 3e-16


def test_action_matches_golden():
    """The restated action against the reference's output committed in tests/golden."""
    gold = np.load(os.path.join(GOLDEN, "action_p2.npz"))
    g = geometry((2, 2, 2), (1, 1, 1), 6.0, (1, 1, 1), 4, 1, seed=12, sigma=0.5, numax=2)
    from angstromcube_b200 import green_function as gf
    p = gf.construct_Green_function(g)
    gf.update_potential(p, gold["Vc"], gold["mats"], gold["offs"], layout="cells")
    gf.update_energy_parameter(p, complex(gold["E"]), float(gold["dVol"]))
    gf.update_phases(p, gold["k"])
    o = oracle.RestatedOracle(p.export(), gold["Vc"], complex(gold["E"]))
    x = np.random.default_rng(int(gold["x_seed"])).standard_normal((p.nnzb, 2, 64, 64))
    y = o.action(x)
    assert rel_err(y[:2], gold["y_blocks"]) < 1e-13
    w = np.arange(1, 8193, dtype=np.float64).reshape(2, 64, 64) / 8192.0
    cs = np.stack([y.sum(axis=(1, 2, 3)), (w * y * y).sum(axis=(1, 2, 3))], axis=1)
    assert np.allclose(cs, gold["checksums"], rtol=1e-11, atol=1e-11 * np.abs(gold["checksums"]).max())


@needs_ref
@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_restated_action_matches_reference(name):
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    ref = reference_plan(g, Vc, mats, offs, E, k, dVol)
    o = oracle.RestatedOracle(ref.export(), Vc, E)
    x = np.random.default_rng(1).standard_normal((ref.sizes["nnzb"], 2, 64, 64))
    assert rel_err(o.action(x), ref.action(x)) < 1e-13


@needs_ref
def test_sho_prefactors_match_reference():
    for numax, sigma in [(3, 0.5), (5, 0.6), (7, 1.3)]:
        assert np.allclose(workloads.sho_prefactors(numax, sigma), oracle.ref_sho_prefactors(numax, sigma),
                           rtol=1e-15, atol=0)
