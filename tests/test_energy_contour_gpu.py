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


def test_integrate_matches_reference_cpu_solves():
    """The contour density with the GPU solver against the same contour with every (E, k) point
    solved by the reference's own CPU action (oracle/_ref) driven by the numpy tfQMR restatement:
    two atoms in a periodic 4^3 cell, truncation radius 3 Bohr, four energy points at one k-point
    (each reference solve takes seconds: the reference's CPU action on 64 blocks is ~80 ms)."""
    import oracle
    from oracle import tfqmr
    from helpers import geometry, inputs_for, product_plan, reference_plan
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    g = geometry((4, 4, 4), (1, 1, 1), 3.0, (1, 1, 1), 4, 2, seed=17, sigma=0.5, numax=3)
    Vc, mats, offs, E0, k0, dVol, na = inputs_for(g, seed=23)
    E, W = ec.get_energy_mesh(5e-2, -1.0, 1, 1, 1, 1)
    ks = [np.array([0.2, -0.1, 0.3])]
    kw = [1.0]

    def ref_solve(e, k):
        r = reference_plan(g, Vc, mats, offs, e, k, dVol)
        ex = r.export()
        X, info = tfqmr.solve_blocks_torch(lambda z: torch.from_numpy(r.action(z.cpu().numpy())).to(z.device),
                                           ex["subset"], ex["colindx"], r.sizes["nnzb"], r.sizes["nCols"],
                                           tol=1e-11, maxiter=3000)
        assert info["converged"], (e, k, info)
        X = X.cpu().numpy()
        d = X[ex["subset"]][:, :, np.arange(64), np.arange(64)] / np.pi      # [nCols, 2, 64]
        return d[:, 0] + 1j * d[:, 1]

    rho_ref, resp_ref, _ = ec.integrate(None, E, W, ks, kw, dVol, fermi_level=-0.1, solve=ref_solve)
    p = product_plan(g, Vc, mats, offs, E0, k0, dVol)
    rho, resp, stats = ec.integrate(p, E, W, ks, kw, dVol, fermi_level=-0.1, tolerance=1e-11, max_iterations=3000,
                                    precision="float64", check_every=5)
    assert all(s["converged"] for s in stats), stats
    assert np.abs(rho - rho_ref).max() <= 1e-8 * np.abs(rho_ref).max()
    assert np.abs(resp - resp_ref).max() <= 1e-8 * max(np.abs(resp_ref).max(), 1e-300)
