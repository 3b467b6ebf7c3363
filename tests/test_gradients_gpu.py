"""Gradients of the contour density objective through torch.autograd (tests/green_autograd.py):

    L = Im sum_E w_E sum_{i in the source cube} W_i G_ii(E)

on the differentiation cell (the periodic 16^3-cube cell with 64 atoms, numax 5, sigma 0.6, its
potential and atom matrices; one source cube, 4,096 blocks) at 8 energies of the contour with
their quadrature weights (the top arc of the 32-point semicircle from -1 to 0 Ha, Im E 0.43 to
0.5 Ha), W a seeded positive weight of the 64 points of the source cube.  The adjoint gradient
(backward pass: solves at conj(E) and a43g_vjp) is checked by central finite differences along
seeded random directions of V (step 1e-5 Ha), of H and of S of one atom (symmetric directions,
step 1e-5 Ha) and of the atom positions (step 1e-4 Bohr, projection radius 8 sigma), to 1e-6
relative; every solve is FP64 to 1e-12.  The reference has no derivatives.
"""
import copy

import numpy as np
import pytest

from angstromcube_b200 import workloads

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def differentiation_problem():
    import green_autograd as ga
    w = workloads.make("periodic16_64atoms_s1x1x1")
    E, wE = workloads.contour_semicircle(32)
    top = np.argsort(-E.imag)[:8]
    rng = np.random.default_rng(2)
    W = rng.uniform(0.5, 1.5, size=(1, 64))
    prob = ga.Problem(w.geometry, E[top], wE[top], W, w.dVol)
    nsho = [workloads.nsho(int(l)) for l in w.geometry.xyzZinso[:, 5]]
    H, S = [], []
    for a, n in enumerate(nsho):
        o = int(w.offsets[a])
        H.append(w.mats[o:o + n * n].reshape(n, n).copy())
        S.append(w.mats[o + n * n:o + 2 * n * n].reshape(n, n).copy())
    R = w.geometry.xyzZinso[:, :3].copy()
    return prob, w.Vcell.copy(), H, S, R


def test_autograd_gradient_vs_central_differences():
    import green_autograd as ga
    prob, V, H, S, R = differentiation_problem()
    tV = torch.from_numpy(V).requires_grad_()
    tH = torch.from_numpy(np.concatenate([h.ravel() for h in H])).requires_grad_()
    tS = torch.from_numpy(np.concatenate([s.ravel() for s in S])).requires_grad_()
    tR = torch.from_numpy(R).requires_grad_()
    L = ga.objective(prob, tV, tH, tS, tR)
    gV, gH, gS, gR = torch.autograd.grad(L, [tV, tH, tS, tR])
    assert abs(L.item() - prob.value(V, H, S, R)) <= 1e-12 * abs(L.item())
    rng = np.random.default_rng(32)
    nsho = [h.shape[0] for h in H]
    # the atom whose matrices are varied: the one nearest the source cube (the derivatives of the
    # farther atoms are orders of magnitude smaller, below what central differences of solves to
    # 1e-12 resolve to 1e-6)
    from angstromcube_b200 import green_function as gf
    cc = gf.construct_Green_function(prob.geometry).export()["colCubePos"].reshape(-1, 4)[0, :3]
    centre = (cc.astype(np.float64) * 4 + 2) * np.asarray(prob.geometry.hg)
    a = int(np.argmin(np.linalg.norm(R - centre, axis=1)))
    off = sum(n * n for n in nsho[:a])
    n = nsho[a]

    def central(step, perturb):
        Lp = prob.value(*perturb(+step))
        Lm = prob.value(*perturb(-step))
        return (Lp - Lm) / (2 * step)

    # potential
    D = rng.standard_normal(V.shape)
    fd = central(1e-5, lambda h: (V + h * D, H, S, R))
    an = float(np.sum(D * gV.numpy()))
    assert abs(fd - an) <= 1e-6 * abs(an), ("V", fd, an)
    # atom matrices (symmetric directions)
    for which, grad in (("H", gH), ("S", gS)):
        Dm = rng.standard_normal((n, n)); Dm = 0.5 * (Dm + Dm.T)

        def perturb(h, which=which, Dm=Dm):
            H2 = [x.copy() for x in H]; S2 = [x.copy() for x in S]
            (H2 if which == "H" else S2)[a] += h * Dm
            return V, H2, S2, R
        fd = central(1e-5, perturb)
        an = float(np.sum(Dm * grad.numpy()[off:off + n * n].reshape(n, n)))
        assert abs(fd - an) <= 1e-6 * abs(an), (which, fd, an)
    # positions of all atoms: on the same cell with the projection radius at 8 sigma instead of
    # 6, where the functions are below 1e-11, so that no grid point crossing the cut-off sphere
    # during the 1e-4 Bohr steps changes a value by more than that (at 6 sigma a crossing jumps by
    # about 3e-6 of the function's scale, which central differences would turn into 1e-2)
    prob.geometry = copy.deepcopy(prob.geometry)
    prob.geometry.proj_radius = 8.0
    tR8 = torch.from_numpy(R).requires_grad_()
    gR8, = torch.autograd.grad(ga.objective(prob, tV.detach(), tH.detach(), tS.detach(), tR8), [tR8])
    Dr = rng.standard_normal(R.shape)
    fd = central(1e-4, lambda h: (V, H, S, R + h * Dr))
    an = float(np.sum(Dr * gR8.numpy()))
    assert abs(fd - an) <= 1e-6 * abs(an), ("R", fd, an)
