"""Vector-Jacobian products (a43g_vjp).  The reference has no derivatives, so the gradients are
checked against finite differences: of the action's bilinear form F = sum L^T (H - E S) G
(linear in the potential and the atom matrices: exact up to rounding; central differences with
a 1e-4 Bohr step for the atom positions), and of a functional of FP64 solves,
J = Im(w sum_i W_i G_ii), whose gradient uses the adjoint Green function (the solve at conj(E),
conjugated).  Tolerances: 1e-9 relative for the linear parts, 1e-6 for finite differences of
positions and of solves.
"""
import copy

import numpy as np
import pytest

from helpers import geometry, inputs_for, product_plan
from angstromcube_b200 import green_action, workloads

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def small_geometry():
    # 4^3 periodic cubes, two atoms numax 3 (20 projectors), dense truncation.  The projection
    # radius is 8 sigma instead of 6: the functions are cut off where they are below 1e-11, so
    # moving an atom by the finite-difference step changes no value by more than that when a
    # point crosses the cut-off sphere (at 6 sigma such a crossing jumps by about 3e-6)
    g = geometry((4, 4, 4), (1, 1, 1), 3.0, (1, 1, 1), 4, 2, seed=11, sigma=0.5, numax=3)
    g.proj_radius = 8.0
    return g


def colindx(p):
    return torch.from_numpy(p.export()["colindx"].astype(np.int16)).cuda()


def bilinear(p, L, G):
    y = torch.empty_like(G)
    green_action.action_t(p, "float64").multiply(y, G, colindx(p), p.nnzb, p.nCols)
    torch.cuda.synchronize()
    Lc = torch.complex(L[:, 0], L[:, 1])
    yc = torch.complex(y[:, 0], y[:, 1])
    return complex((Lc * yc).sum().item())


def atom_slot(p, atom_id):
    ids = list(p.export()["global_atom_ids"])
    return ids.index(atom_id)


@pytest.fixture(scope="module")
def setup():
    g = small_geometry()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g, seed=21)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    gen = torch.Generator().manual_seed(3)
    L = torch.randn((p.nnzb, 2, 64, 64), generator=gen, dtype=torch.float64)
    G = torch.randn((p.nnzb, 2, 64, 64), generator=gen, dtype=torch.float64)
    return g, (Vc, mats, offs, E, k, dVol), p, L, G      # host tensors: moved to the GPU in the tests


def test_vjp_potential_and_matrices_exact(setup):
    g, (Vc, mats, offs, E, k, dVol), p, L, G = setup
    L, G = L.cuda(), G.cuda()
    out = green_action.vjp(p, L, G)
    F0 = bilinear(p, L, G)
    rng = np.random.default_rng(7)
    # potential: F is linear in V
    D = rng.standard_normal(Vc.shape)
    F1 = bilinear(product_plan(g, Vc + D, mats, offs, E, k, dVol), L, G)
    pred = np.sum(D * out["V"])
    assert abs((F1 - F0) - pred) <= 1e-9 * abs(pred)
    # atom matrices: M = dVol (dH - E dS); perturb dH and dS of atom 1
    nc = 20
    o = int(offs[1])
    for plane, factor in ((0, dVol), (1, -E * dVol)):
        m2 = mats.copy()
        Dm = rng.standard_normal((nc, nc))
        m2[o + plane * nc * nc:o + (plane + 1) * nc * nc] += Dm.ravel()
        F2 = bilinear(product_plan(g, Vc, m2, offs, E, k, dVol), L, G)
        pred = factor * np.sum(Dm * out["M"][atom_slot(p, 1)])
        assert abs((F2 - F0) - pred) <= 1e-9 * abs(pred)


def test_vjp_positions_central_differences(setup):
    g, (Vc, mats, offs, E, k, dVol), p, L, G = setup
    L, G = L.cuda(), G.cuda()
    out = green_action.vjp(p, L, G, potential=False, matrices=False)
    h = 1e-4
    for atom in (0, 1):
        for d in range(3):
            F = []
            for s in (+1, -1):
                g2 = copy.deepcopy(g)
                g2.xyzZinso = g.xyzZinso.copy()
                g2.xyzZinso[atom, d] += s * h
                F.append(bilinear(product_plan(g2, Vc, mats, offs, E, k, dVol), L, G))
            fd = (F[0] - F[1]) / (2 * h)
            an = out["R"][atom_slot(p, atom), d]
            assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-3 * np.abs(out["R"]).max()), (atom, d, fd, an)


def _solve(p):
    X = torch.zeros((p.nnzb, 2, 64, 64), dtype=torch.float64, device="cuda")
    st, rho = green_action.solve(p, X=X, precision="float64", tolerance=1e-13, max_iterations=4000, check_every=5)
    assert st["residual_max"] < 1e-11, st
    return X, rho


def _functional(rho, W, w):
    # J = Im(w sum_i W_i G_ii), G_ii = pi rho_i (rho exported as diag(G)/pi)
    return float(np.imag(w * np.pi * np.sum(W * rho)))


def test_vjp_solve_gradient_vs_finite_differences():
    """Gradient of J = Im(w sum_i W_i G_ii(E)) at k != 0 through the adjoint solve."""
    g = small_geometry()
    Vc, mats, offs, E, k, dVol, na = inputs_for(g, seed=21)
    rng = np.random.default_rng(9)
    W = rng.uniform(0.5, 1.5, size=(1, 64))
    w = complex(0.3, -0.2)
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    G, rho = _solve(p)
    # adjoint Green function: A(E)^T = conj(A(conj E)), so A^-T B = conj(G(conj E))
    pa = product_plan(g, Vc, mats, offs, E.conjugate(), k, dVol)
    Ga, _ = _solve(pa)
    Gt = torch.stack([Ga[:, 0], -Ga[:, 1]], dim=1)
    Wt = torch.from_numpy(W[0]).cuda()
    Lam = Gt * Wt                                   # scale every source column by its weight
    out = green_action.vjp(p, Lam, G)
    # dJ/dp = Im(w * (-dF/dp))
    gV = np.imag(-w * out["V"])
    gM = np.imag(-w * out["M"][atom_slot(p, 0)])
    gR = np.imag(-w * out["R"][atom_slot(p, 0)])
    # finite differences of J along one random direction of V, one of dH (atom 0), one position
    D = rng.standard_normal(Vc.shape)
    dv = 1e-5
    Jp = _functional(_solve(product_plan(g, Vc + dv * D, mats, offs, E, k, dVol))[1], W, w)
    Jm = _functional(_solve(product_plan(g, Vc - dv * D, mats, offs, E, k, dVol))[1], W, w)
    fd = (Jp - Jm) / (2 * dv)
    an = float(np.sum(D * gV))
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)
    nc = 20
    Dm = rng.standard_normal((nc, nc))
    o = int(offs[0])
    J = []
    for s in (+1, -1):
        m2 = mats.copy()
        m2[o:o + nc * nc] += s * 1e-5 * Dm.ravel()
        J.append(_functional(_solve(product_plan(g, Vc, m2, offs, E, k, dVol))[1], W, w))
    fd = (J[0] - J[1]) / 2e-5
    an = float(dVol * np.sum(Dm * gM))
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)
    J = []
    for s in (+1, -1):
        g2 = copy.deepcopy(g)
        g2.xyzZinso = g.xyzZinso.copy()
        g2.xyzZinso[0, 2] += s * 1e-4
        J.append(_functional(_solve(product_plan(g2, Vc, mats, offs, E, k, dVol))[1], W, w))
    fd = (J[0] - J[1]) / 2e-4
    assert abs(fd - gR[2]) <= 1e-6 * max(abs(gR[2]), 1e-3 * np.abs(gR).max()), (fd, gR)


def test_vjp_matches_reference_cpu_solves():
    """The gradient from solves with the reference's own action (oracle/_ref, its CPU build,
    driven by the numpy tfQMR restatement) agrees with the GPU adjoint gradient: dJ/dV and dF/dM
    assembled on the CPU, dF/dR through the vector-Jacobian products of the CPU solutions."""
    import oracle
    from oracle import tfqmr
    from helpers import reference_plan
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    g = geometry((4, 4, 4), (1, 1, 1), 3.0, (1, 1, 1), 4, 2, seed=11, sigma=0.5, numax=3)
    Vc, mats, offs, E, k, dVol, na = inputs_for(g, seed=21)
    E = complex(-0.3, 0.5)                            # broad enough for short CPU solves
    rng = np.random.default_rng(13)
    W = rng.uniform(0.5, 1.5, size=64)
    w = complex(0.3, -0.2)
    # reference CPU solves at E and at conj(E)
    sol = []
    for e in (E, E.conjugate()):
        r = reference_plan(g, Vc, mats, offs, e, k, dVol)
        ex = r.export()
        X, info = tfqmr.solve_blocks(r.action, ex["subset"], ex["colindx"], r.sizes["nnzb"], r.sizes["nCols"],
                                     tol=1e-11, maxiter=1500)
        assert info["converged"], info
        sol.append(X[:, 0] + 1j * X[:, 1])
        veff = ex["veff_index"]
    Gc, Gac = sol
    Lam = np.conj(Gac) * W[None, None, :]
    dV_cpu = np.zeros((len(Vc), 64), complex)
    prod = (Lam * Gc).sum(axis=2)                     # [nnzb, 64 points]
    for b, cell in enumerate(veff):
        if cell >= 0:
            dV_cpu[cell] += prod[b]
    gV_cpu = np.imag(-w * dV_cpu)
    # the same on the GPU: solves, adjoint, vector-Jacobian product
    p = product_plan(g, Vc, mats, offs, E, k, dVol)
    G, _ = _solve(p)
    Ga, _ = _solve(product_plan(g, Vc, mats, offs, E.conjugate(), k, dVol))
    Lt = torch.stack([Ga[:, 0], -Ga[:, 1]], dim=1) * torch.from_numpy(W).cuda()
    out_gpu = green_action.vjp(p, Lt, G)
    gV_gpu = np.imag(-w * out_gpu["V"])
    assert np.abs(gV_gpu - gV_cpu).max() <= 1e-7 * np.abs(gV_cpu).max()
    # dF/dM_A = sum over columns of l_A g_A^T with g_A = sum_i ph_i P_i^T G and
    # l_A = sum_i conj(ph_i) P_i^T Lambda over the images i of atom A, assembled on the CPU from the
    # reference solves with the oracle's projection (P^T x per image, pinned to the reference)
    e = p.export()
    o = oracle.RestatedOracle(e, Vc, E)
    Gr = np.stack([Gc.real, Gc.imag], axis=1)
    Lr = np.stack([Lam.real, Lam.imag], axis=1)
    _, apcG, _ = o.dyadic(Gr, want_coefficients=True)
    _, apcL, _ = o.dyadic(Lr, want_coefficients=True)
    aG = apcG[:, 0] + 1j * apcG[:, 1]                  # [coefficients of all images (nCols = 1), 64 columns]
    aL = apcL[:, 0] + 1j * apcL[:, 1]
    ph = e["AtomImagePhase"][:, 0] + 1j * e["AtomImagePhase"][:, 1]
    starts = e["AtomImageStarts"]
    for slot in range(len(e["AtomLmax"])):
        nc = workloads.nsho(int(e["AtomLmax"][slot]))
        gA = np.zeros((nc, 64), complex); lA = np.zeros((nc, 64), complex)
        for k in range(e["SHOsum_start"][slot], e["SHOsum_start"][slot + 1]):
            i = e["SHOsum_col"][k]
            gA += ph[i] * aG[starts[i]:starts[i] + nc]
            lA += np.conj(ph[i]) * aL[starts[i]:starts[i] + nc]
        dM_cpu = lA @ gA.T
        assert np.abs(out_gpu["M"][slot] - dM_cpu).max() <= 1e-7 * np.abs(dM_cpu).max()
    # positions: the vector-Jacobian products of the reference CPU solutions against those of the
    # GPU solutions (the same kernels, different solves)
    Gcu = torch.from_numpy(Gr).cuda()
    Lcu = torch.from_numpy(Lr).cuda()
    dR_ref = green_action.vjp(p, Lcu, Gcu, potential=False, matrices=False)["R"]
    assert np.abs(out_gpu["R"] - dR_ref).max() <= 1e-7 * np.abs(dR_ref).max()
