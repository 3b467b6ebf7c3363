"""Energy contour (src/energy_contour.cxx): the computed quadratures and mesh against the
reference's own tables and mesh (oracle/_ref), and the integration over energies and k-points
(host logic with a stand-in solver; the GPU solver in test_energy_contour_gpu)."""
import numpy as np
import pytest

import oracle
from angstromcube_b200 import energy_contour as ec

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("n", list(range(1, 33)))
def test_gauss_legendre_matches_reference(n):
    x, w = ec.gauss_legendre(n)
    xr, wr = oracle.ref_quadrature("legendre", n)
    assert np.abs(x - xr).max() < 1e-14 and np.abs(w - wr).max() < 1e-14


@needs_ref
@pytest.mark.parametrize("n", list(range(1, 11)))
def test_gauss_fermi_dirac_matches_reference(n):
    """Up to 10 points the reference's table is the Gauss rule of 1/(1+exp(30x)) on [-1, inf)
    to 1e-12; its larger tables drift from it (1e-6 at 16 points), ours are converged."""
    x, w = ec.gauss_fermi_dirac(n)
    xr, wr = oracle.ref_quadrature("fermi_dirac", n)
    assert np.abs(x - xr).max() < 1e-12 and np.abs(w - wr).max() < 1e-12


@pytest.mark.parametrize("n", [4, 9, 16])
def test_gauss_fermi_dirac_is_exact_on_polynomials(n):
    # moments of the weight by a fine composite rule against the n-point Gauss rule (degree 2n-1)
    x, w = ec.gauss_fermi_dirac(n)
    gx, gw = np.polynomial.legendre.leggauss(64)
    edges = np.linspace(-1, 2, 301)
    X = np.concatenate([0.5 * (b - a) * gx + 0.5 * (a + b) for a, b in zip(edges[:-1], edges[1:])])
    Wt = np.concatenate([0.5 * (b - a) * gw for a, b in zip(edges[:-1], edges[1:])]) / (1 + np.exp(30 * X))
    for k in range(2 * n):
        assert abs(np.sum(w * x ** k) - np.sum(Wt * X ** k)) < 1e-12


@needs_ref
@pytest.mark.parametrize("args", [(1e-2, -1.0, 5, 15, 9, 3), (2e-2, -0.7, 4, 12, 6, 2), (1e-2, -1.0, 5, 15, 9, -2),
                                  (1e-2, -1.0, 0, 11, 0, 0)])
def test_energy_mesh_matches_reference(args):
    E, W = ec.get_energy_mesh(*args)
    Er, Wr = oracle.ref_energy_mesh(*args)
    assert len(E) == len(Er)
    assert np.abs(E - Er).max() < 1e-12 and np.abs(W - Wr).max() < 1e-12


def test_integrate_host_logic():
    E, W = ec.get_energy_mesh(1e-2, -1.0, 2, 3, 2, 1)
    ks = [np.zeros(3), np.array([0.25, 0.0, 0.0])]
    kw = [0.5, 0.5]

    def fake(Ep, k):
        i = np.arange(2 * 64).reshape(2, 64)
        return np.exp(1j * (i * Ep.real + k.sum())) / (1 + abs(Ep)) + 1j * Ep.imag

    rho, resp, _ = ec.integrate(None, E, W, ks, kw, 1.0, solve=fake)
    rho_c = sum(wE * sum(wk * fake(complex(e), np.asarray(k)) for k, wk in zip(ks, kw)) for e, wE in zip(E, W))
    assert np.allclose(rho, rho_c.real, rtol=1e-13, atol=1e-13)
    n = len(E)
    res = -sum(sum(wk * fake(complex(e), np.asarray(k)) for k, wk in zip(ks, kw)) for e in E[:n - 2])
    res_point = -sum(complex(e) for e in E[:n - 2])
    assert np.allclose(resp, (res / res_point).real, rtol=1e-12, atol=1e-13)
