"""tfQMR solves on the GPU.  Solver parity is anchored on the operator: the true residual
|B - A X| / |B| of the returned solution is recomputed with the oracle's FP64 action on the
CPU, and the solution is compared with the numpy tfQMR restatement (oracle/tfqmr.py)."""
import numpy as np
import pytest

import oracle
from angstromcube_b200 import green_action, green_function as gf, workloads

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def setup(name):
    w = workloads.make(name)
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(p, w.E, w.dVol)
    return w, p


def true_residual(p, w, X):
    a = p.export()
    o = oracle.RestatedOracle(a, w.Vcell, w.E)
    AX = o.action(X)
    B = np.zeros_like(X)
    for c, b in enumerate(a["subset"]):
        B[b, 0][np.arange(64), np.arange(64)] = 1.0
    R = (B - AX)
    Rc = (R[:, 0] + 1j * R[:, 1])
    colres = np.zeros((p.nCols, 64))
    np.add.at(colres, a["colindx"].astype(np.int64), (np.abs(Rc) ** 2).sum(axis=1))
    return np.sqrt(colres.max())


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_solve_periodic4_1atom(precision):
    w, p = setup("periodic4_1atom")
    X = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    # the mixed solver restarts tfQMR once per FP32 sweep (about 3 digits each): larger budget
    maxit = w.max_iterations if precision == "float64" else 3*w.max_iterations
    stats, rho = green_action.solve(p, X=X, tolerance=w.tolerance, max_iterations=maxit,
                                    precision=precision, check_every=5, max_refinements=6)
    assert stats["converged"] == 1, stats
    assert stats["residual_max"] <= w.tolerance
    Xn = X.cpu().numpy()
    res = true_residual(p, w, Xn)
    assert res <= 2 * w.tolerance, res
    a = p.export()
    d = np.array([Xn[b, 0][np.arange(64), np.arange(64)] + 1j * Xn[b, 1][np.arange(64), np.arange(64)]
                  for b in a["subset"]]) / np.pi
    assert np.allclose(rho, d, rtol=0, atol=1e-14)


def test_fp64_and_mixed_agree():
    w, p = setup("periodic4_1atom")
    X1 = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    X2 = torch.zeros_like(X1)
    s1, _ = green_action.solve(p, X=X1, tolerance=1e-10, max_iterations=800, precision="float64")
    s2, _ = green_action.solve(p, X=X2, tolerance=1e-10, max_iterations=2000, precision="float32")
    assert s1["converged"] and s2["converged"], (s1, s2)
    err = ((X1 - X2).abs().max() / X1.abs().max()).item()
    assert err < 1e-7


def test_solve_matches_numpy_tfqmr():
    """Same problem solved by the numpy restatement of tfQMR around the oracle action."""
    from oracle import tfqmr
    w, p = setup("periodic4_1atom")
    a = p.export()
    o = oracle.RestatedOracle(a, w.Vcell, w.E)
    X = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    stats, _ = green_action.solve(p, X=X, tolerance=1e-9, max_iterations=500, precision="float64")
    Xo, info = tfqmr.solve_blocks(o.action, a["subset"], a["colindx"], p.nnzb, p.nCols, tol=1e-9, maxiter=500)
    assert info["converged"]
    Xg = X.cpu().numpy()
    assert np.abs(Xg - Xo).max() / np.abs(Xo).max() < 1e-6


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_graph_replay_matches_direct_launches(precision):
    """On a non-default stream every tfQMR iteration is one replay of a captured CUDA graph; on
    the default stream the kernels are launched one by one.  Both converge to the same solution
    (the per-column reductions use atomics, so agreement is to the solve tolerance, not bits)."""
    from angstromcube_b200 import _lib
    w, p = setup("periodic4_1atom")
    X0 = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    X1 = torch.zeros_like(X0)
    maxit = 800 if precision == "float64" else 2400
    s0, _ = green_action.solve(p, X=X0, tolerance=1e-10, max_iterations=maxit, precision=precision)
    stream = torch.cuda.Stream()
    n0 = _lib.lib().a43g_kernel_launches()
    s1, _ = green_action.solve(p, X=X1, tolerance=1e-10, max_iterations=maxit, precision=precision, stream=stream)
    torch.cuda.synchronize()
    assert _lib.lib().a43g_kernel_launches() - n0 > 10 * s1["iterations"]   # replays are counted
    assert s0["converged"] and s1["converged"], (s0, s1)
    err = ((X0 - X1).abs().max() / X0.abs().max()).item()
    assert err < 1e-8


def test_solve_concurrent_matches_sequential():
    """Batched solves of several (E, k) pairs on worker plans and streams give the densities of
    the same solves done one after the other."""
    w = workloads.make("periodic4_1atom")
    energies = [complex(-0.3 + 0.05 * i, 0.05 + 0.05 * i) for i in range(6)]
    kpoints = [np.zeros(3) if i % 2 == 0 else np.array([0.1, 0.0, 0.2]) for i in range(6)]
    opts = dict(tolerance=1e-10, max_iterations=1500, precision="float64")
    out = green_action.solve_concurrent(w.geometry, w.Vcell, w.mats, w.offsets, energies, kpoints, w.dVol,
                                        workers=3, **opts)
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    for (st, rho), E, k in zip(out, energies, kpoints):
        assert st["converged"], st
        gf.update_energy_parameter(p, E, w.dVol)
        gf.update_phases(p, k)
        st0, rho0 = green_action.solve(p, **opts)
        assert np.abs(rho - rho0).max() <= 1e-8 * np.abs(rho0).max()


@pytest.mark.parametrize("name", ["iso6_fd16", "mixed_iso_peri_vac", "repeat_aniso", "wrap8"])
@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_solve_geometries_true_residual(name, precision):
    """Solves on every kind of boundary condition and both stencil orders: the true residual of
    the returned solution, recomputed with the oracle's FP64 action, meets the tolerance."""
    from helpers import GEOMETRIES, inputs_for, product_plan
    g = GEOMETRIES[name]()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g)
    E = complex(E.real, 0.3)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    X = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    stats, _ = green_action.solve(p, X=X, tolerance=1e-9, max_iterations=4000, precision=precision,
                                  stream=torch.cuda.Stream())
    assert stats["converged"], stats
    a = p.export()
    o = oracle.RestatedOracle(a, Vc, E)
    Xn = X.cpu().numpy()
    B = np.zeros_like(Xn)
    for c, b in enumerate(a["subset"]):
        B[b, 0][np.arange(64), np.arange(64)] = 1.0
    R = B - o.action(Xn)
    Rc = R[:, 0] + 1j * R[:, 1]
    colres = np.zeros((p.nCols, 64))
    np.add.at(colres, a["colindx"].astype(np.int64), (np.abs(Rc) ** 2).sum(axis=1))
    assert np.sqrt(colres.max()) <= 2e-9
