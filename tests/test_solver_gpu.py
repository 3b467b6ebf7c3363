"""tfQMR solves on the GPU.  Solver parity is anchored on the operator: the true residual
|B - A X| / |B| of the returned solution is recomputed with the oracle's FP64 action on the
CPU, and the solution is compared with the numpy tfQMR restatement (oracle/tfqmr.py).
Reductions are in a fixed order, so repeated solves are bit-identical; retiring finished source
cubes changes no bit of the result; batched solves match one-by-one solves."""
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
    maxit = w.max_iterations if precision == "float64" else 2*w.max_iterations
    stats, rho = green_action.solve(p, X=X, tolerance=w.tolerance, max_iterations=maxit,
                                    precision=precision, check_every=5)
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
    the default stream the kernels are launched one by one.  Both give the same bits (the
    per-column reductions run in a fixed order)."""
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
    assert s0["iterations"] == s1["iterations"]
    assert torch.equal(X0, X1)


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_solve_is_deterministic_and_retirement_changes_no_bit(precision):
    """Two solves of the same problem give identical bits and iteration counts; solving without
    retirement (finished source cubes keep being computed, as the reference's solver does) gives
    the same bits again, since finished columns are frozen."""
    w = workloads.make("periodic8_8atoms_s2x2x1")
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(p, complex(-0.3, 0.25), w.dVol)
    stream = torch.cuda.Stream()
    Xs, ss = [], []
    # (the FP32 recurrences always retire finished sources: the third solve repeats the first)
    for retire in (True, True, False):
        X = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
        st, _ = green_action.solve(p, X=X, tolerance=1e-9, max_iterations=3000, precision=precision,
                                   check_every=1, retire=retire, stream=stream)
        torch.cuda.synchronize()
        # FP64 tfQMR stops on its QMR bound: the true residual may end a little above it
        assert st["iterations"] < 3000 and st["residual_max"] <= 1e-8, st
        Xs.append(X); ss.append(st)
    assert ss[0]["iterations"] == ss[1]["iterations"] == ss[2]["iterations"]
    assert torch.equal(Xs[0], Xs[1])
    assert torch.equal(Xs[0], Xs[2])


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_solve_batched_matches_individual_solves(precision):
    """Five (E, k) pairs in waves of two (the last wave padded): the densities and the true
    residuals of every pair match its own solve."""
    w = workloads.make("periodic4_1atom")
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    energies = [complex(-0.4 + 0.1 * i, 0.08 + 0.04 * i) for i in range(5)]
    kpoints = [np.array([0.0, 0.0, 0.0]), np.array([0.1, 0.0, 0.2]), np.array([0.25, 0.25, 0.0]),
               np.array([0.0, -0.2, 0.1]), np.array([0.3, 0.1, -0.1])]
    opts = dict(tolerance=1e-10, max_iterations=2000, precision=precision, check_every=1)
    stream = torch.cuda.Stream()
    stats, rho = green_action.solve_batched(p, energies, kpoints, w.dVol, want_rho=True, batch=2,
                                            stream=stream, **opts)
    for i, (E, k) in enumerate(zip(energies, kpoints)):
        assert stats[i]["converged"] and stats[i]["residual_max"] <= 1e-10, (i, stats[i])
        gf.update_energy_parameter(p, E, w.dVol)
        gf.update_phases(p, k)
        X = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
        st, rho0 = green_action.solve(p, X=X, stream=stream, **opts)
        assert st["converged"], (i, st)
        assert np.abs(rho[i] - rho0).max() <= 1e-8 * np.abs(rho0).max()
        # and the single solve against the oracle
        we = workloads.Workload(w.name, w.geometry, w.Vcell, w.mats, w.offsets, E, k, w.dVol, 1e-10, 2000)
        assert true_residual(p, we, X.cpu().numpy()) <= 2e-10


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


def test_slow_convergence_at_the_single_energy_is_the_algorithms():
    """At E = -0.2 + 0.02i (the energy of the single-energy configuration of the 16^3-cube cell)
    tfQMR converges slowly, and that is the algorithm's behaviour, not this library's: after 400
    iterations the true residual of this library's FP64 solve and that of the restated tfQMR
    (oracle/tfqmr.py, on torch tensors, around this library's FP64 action, which matches the
    reference's action on this cell to 1e-12) both lie between 1e-3 and 1."""
    from oracle import tfqmr
    w = workloads.make("periodic16_64atoms_s1x1x1")
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    E = complex(-0.2, 0.02)
    gf.update_energy_parameter(p, E, w.dVol)
    st, _ = green_action.solve(p, precision="float64", tolerance=1e-8, max_iterations=400, check_every=10,
                               want_rho=False, stream=torch.cuda.Stream())
    assert not st["converged"] and 1e-3 < st["residual_max"] < 1.0, st
    a = p.export()
    ci = torch.from_numpy(a["colindx"].astype(np.int16)).cuda()
    op = green_action.action_t(p, "float64")

    def action(x):
        y = torch.empty_like(x)
        op.multiply(y, x.contiguous(), ci, p.nnzb, p.nCols)
        return y

    B = torch.zeros((p.nnzb, 2, 64, 64), dtype=torch.float64, device="cuda")
    for c, b in enumerate(a["subset"]):
        B[int(b), 0, torch.arange(64), torch.arange(64)] = 1.0

    def true_residual(X):
        R = B - action(X)
        return float(torch.sqrt((R ** 2).sum(dim=(0, 1, 2))).max())   # one source cube: per-column norms

    X, info = tfqmr.solve_blocks_torch(action, a["subset"], a["colindx"], p.nnzb, p.nCols, tol=1e-8, maxiter=400)
    r = true_residual(X)
    assert not info["converged"] and 1e-3 < r < 1.0, (r, info)


def test_solve_traced_error_of_G():
    """a43g_solve_traced: against the plain FP64 solution, the FP64 solve's own trace ends at
    exactly zero (the solver is deterministic) and the mixed solve's error of G falls to the
    level of the tolerance."""
    w = workloads.make("periodic4_1atom")
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(p, complex(-0.3, 0.1), w.dVol)
    stream = torch.cuda.Stream()
    Xref = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    st, _ = green_action.solve(p, X=Xref, stream=stream, want_rho=False, precision="float64", tolerance=1e-10,
                               max_iterations=2000, check_every=1)
    assert st["iterations"] < 2000 and st["residual_max"] <= 1e-9
    st2, _, tr = green_action.solve_traced(p, Xref, every=1, stream=stream, precision="float64", tolerance=1e-10,
                                           max_iterations=2000, check_every=1)
    # one row per iteration and the final row
    assert st2["iterations"] == st["iterations"] and len(tr) == st["iterations"] + 1
    assert np.array_equal(tr[:-1, 0], np.arange(1, len(tr))) and tr[-1, 0] == st["iterations"]
    assert tr[-2, 1] == 0.0 and tr[-1, 1] == 0.0 and tr[-1, 2] == 0
    st3, _, tr3 = green_action.solve_traced(p, Xref, every=5, stream=stream, precision="float32", tolerance=1e-10,
                                            max_iterations=2000)
    assert st3["converged"] and len(tr3) >= 2
    assert np.all(np.diff(tr3[:-1, 0]) == 5) and tr3[0, 1] > 1e-3 and tr3[-1, 1] < 1e-6


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_vector_kernels_16_byte_and_scalar_agree(precision, monkeypatch):
    """The tfQMR vector kernels with 16-byte accesses (the default) and the scalar ones
    (A43G_VEC16=0) give the same densities to the tolerance of the solve."""
    w = workloads.make("periodic4_1atom")
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("A43G_VEC16", flag)
        p = gf.construct_Green_function(w.geometry)
        gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
        gf.update_energy_parameter(p, complex(-0.3, 0.1), w.dVol)
        gf.update_phases(p, np.array([0.1, 0.0, 0.2]))
        st, rho = green_action.solve(p, stream=torch.cuda.Stream(), tolerance=1e-10, max_iterations=2000,
                                     precision=precision, check_every=1)
        assert st["converged"], (flag, st)
        out.append(rho)
    assert np.abs(out[0] - out[1]).max() <= 1e-8 * np.abs(out[1]).max()


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_preconditioned_solve_same_solution_fewer_iterations(precision):
    """Right preconditioning by the cube-diagonal local operator (A43G_SOLVE_PRECONDITION): the
    returned X is the solution of the original system (its true residual with the oracle's FP64
    action at the tolerance's level) and its densities equal the unpreconditioned solve's.  (On
    this cell, eight atoms in deep wells, it takes more iterations than the plain solve: the
    cube's mean potential is a poor model of the wells.)"""
    w = workloads.make("periodic8_8atoms_s2x2x1")
    E, k = complex(-0.3, 0.25), np.array([0.1, 0.0, 0.2])
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    gf.update_energy_parameter(p, E, w.dVol)
    gf.update_phases(p, k)
    stream = torch.cuda.Stream()
    opts = dict(tolerance=1e-9, max_iterations=3000, precision=precision, check_every=1, stream=stream)
    st0, rho0 = green_action.solve(p, **opts)
    X = torch.zeros((p.nnzb, 2, 64, 64), device="cuda", dtype=torch.float64)
    st1, rho1 = green_action.solve(p, X=X, precondition=True, **opts)
    # (FP64 tfQMR stops on its QMR bound: the true residual may end a little above the tolerance)
    assert st0["residual_max"] <= 1e-8 and st1["residual_max"] <= 1e-8, (st0, st1)
    assert np.abs(rho1 - rho0).max() <= 1e-7 * np.abs(rho0).max()
    we = workloads.Workload(w.name, w.geometry, w.Vcell, w.mats, w.offsets, E, k, w.dVol, 1e-9, 3000)
    assert true_residual(p, we, X.cpu().numpy()) <= 1e-8


def test_preconditioned_batched_matches_individual():
    """Batched and individual preconditioned solves (each pair with its own energy in the
    preconditioner's scaling) give the same densities."""
    w = workloads.make("periodic4_1atom")
    p = gf.construct_Green_function(w.geometry)
    gf.update_potential(p, w.Vcell, w.mats, w.offsets, layout="cells")
    energies = [complex(-0.4, 0.08), complex(-0.2, 0.2), complex(0.1, 0.15)]
    kpoints = [np.zeros(3), np.array([0.1, 0.0, 0.2]), np.array([0.25, 0.25, 0.0])]
    opts = dict(tolerance=1e-10, max_iterations=2000, precision="float64", check_every=1, precondition=True)
    stream = torch.cuda.Stream()
    stats, rho = green_action.solve_batched(p, energies, kpoints, w.dVol, want_rho=True, batch=2, stream=stream, **opts)
    for i, (E, k) in enumerate(zip(energies, kpoints)):
        assert stats[i]["residual_max"] <= 1e-9, (i, stats[i])
        gf.update_energy_parameter(p, E, w.dVol)
        gf.update_phases(p, k)
        st, rho0 = green_action.solve(p, stream=stream, **opts)
        assert st["residual_max"] <= 1e-9, (i, st)
        assert np.abs(rho[i] - rho0).max() <= 1e-8 * np.abs(rho0).max()
