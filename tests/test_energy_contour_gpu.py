"""Contour integration with the GPU solver: the density summed by energy_contour.integrate equals
the weighted sum of the individual solves (FP64, periodic 4^3 cell with one atom, two k-points)."""
import numpy as np
import pytest

from angstromcube_b200 import energy_contour as ec, green_action, green_function as gf, workloads

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_integrate_matches_individual_solves():
    w = workloads.make("periodic4_1atom")
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    E, W = ec.get_energy_mesh(5e-2, -1.0, 2, 3, 2, 1)     # lowest point at Im E = pi kT = 0.16
    ks = [np.zeros(3), np.array([0.25, 0.0, 0.0])]
    kw = [0.5, 0.5]
    opts = dict(tolerance=1e-9, max_iterations=4000, precision="float64", check_every=5)
    rho, resp, stats = ec.integrate(p, E, W, ks, kw, w.dVol, fermi_level=-0.1, **opts)
    assert len(stats) == len(E) * len(ks) and all(s["converged"] for s in stats), stats
    total = 0
    for e, we in zip(E, W):
        for k, wk in zip(ks, kw):
            gf.update_energy_parameter(p, complex(e) - 0.1, w.dVol)
            gf.update_phases(p, k)
            st, r = green_action.solve(p, **opts)
            total = total + we * wk * r
    assert np.abs(rho - total.real).max() <= 1e-8 * np.abs(total.real).max()
    assert np.all(np.isfinite(resp))
