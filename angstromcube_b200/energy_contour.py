"""Energy contour of the Green-function density: mesh, quadratures and the integration over
energy points and k-points (the caller of the solver, src/energy_contour.cxx).

    E, w = get_energy_mesh(kBT, eBot, nBot, nPar, nFer, nPol)    # src/energy_contour.cxx:139-240
    rho, response, stats = integrate(plan, E, w, kpoints, kweights, dVol, ...)   # :273-451

The quadrature rules are computed, not tabulated: Gauss-Legendre nodes from numpy, and the
Gauss rule for the Fermi-Dirac weight w(x) = 1/(1 + exp(30 x)) on [-1, inf) (the Fermi function
over 30 kT above and below the Fermi level, the weight the reference's table is built for) by
the discretized Stieltjes procedure and the Golub-Welsch eigenvalue problem.
"""
import numpy as np

__all__ = ["gauss_legendre", "gauss_fermi_dirac", "get_energy_mesh", "integrate"]


def _node_count(n):
    # the reference rounds large rules up: multiples of 4 above 32 points, of 8 above 64
    n = max(int(n), 1)
    if n > 64:
        return ((n - 1) // 8 + 1) * 8
    if n > 32:
        return ((n - 1) // 4 + 1) * 4
    return n


def gauss_legendre(n):
    """Nodes (ascending) and weights on [-1, 1]; n = 0 gives empty arrays."""
    if n == 0:
        return np.zeros(0), np.zeros(0)
    x, w = np.polynomial.legendre.leggauss(_node_count(n))
    return x, w


def _fermi_dirac_discretization():
    # panels on [-1, 2]: the weight is 1 below -0.5 and below 1e-26 above 2
    edges = np.concatenate([np.linspace(-1.0, -0.5, 6), np.linspace(-0.5, 0.5, 101)[1:], np.linspace(0.5, 2.0, 16)[1:]])
    gx, gw = np.polynomial.legendre.leggauss(24)
    xs, ws = [], []
    for a, b in zip(edges[:-1], edges[1:]):
        xs.append(0.5 * (b - a) * gx + 0.5 * (a + b))
        ws.append(0.5 * (b - a) * gw)
    x = np.concatenate(xs)
    return x, np.concatenate(ws) / (1.0 + np.exp(30.0 * x))


def gauss_fermi_dirac(n):
    """Gauss rule for the weight 1/(1 + exp(30 x)) on [-1, inf): nodes (ascending) and weights."""
    if n == 0:
        return np.zeros(0), np.zeros(0)
    x, w = _fermi_dirac_discretization()
    # Stieltjes: three-term recurrence of the monic orthogonal polynomials in the discrete measure
    a = np.zeros(n); b = np.zeros(n)
    p_prev = np.zeros_like(x); p = np.ones_like(x)
    norm_prev = 1.0
    for k in range(n):
        norm = np.sum(w * p * p)
        a[k] = np.sum(w * x * p * p) / norm
        if k > 0:
            b[k] = norm / norm_prev
        p_next = (x - a[k]) * p - (b[k] if k > 0 else 0.0) * p_prev
        p_prev, p, norm_prev = p, p_next, norm
    J = np.diag(a) + np.diag(np.sqrt(b[1:]), 1) + np.diag(np.sqrt(b[1:]), -1)
    nodes, vecs = np.linalg.eigh(J)
    weights = np.sum(w) * vecs[0] ** 2
    return nodes, weights


def get_energy_mesh(kBT=1e-2, eBot=-1.0, nBot=5, nPar=15, nFer=9, nPol=3):
    """Energy points and complex weights of the contour relative to the Fermi level 0.

    nPol > 0: open contour with nPol Matsubara poles (bottom path up from eBot, a path parallel
    to the real axis at 2 nPol pi kT, the Fermi-Dirac tail, the poles); nPol < 0: closed contour
    without poles; nPol == 0: a density-of-states path at height pi kT."""
    assert kBT > 0
    pikT = np.pi * kBT
    E, W = [], []
    if nPol != 0:
        x, w = gauss_legendre(nBot)
        dE = abs(nPol) * pikT
        for xi, wi in zip(x, w):
            E.append(complex(eBot, (xi + 1.0) * dE)); W.append(complex(0.0, wi * dE))
        x, w = gauss_legendre(nPar)
        dE = (0.0 - 30 * kBT * (nPol > 0) - eBot) * 0.5
        for xi, wi in zip(x, w):
            E.append(complex(eBot + (xi + 1.0) * dE, abs(nPol) * 2 * pikT)); W.append(complex(wi * dE, 0.0))
    else:
        assert nPar > 0
        dE = 1.0 if nPar < 2 else (60 * kBT - eBot) / (nPar - 1.0)
        mFer = int(30 * kBT / dE)
        for i in range(mFer - nPar, mFer):
            E.append(complex(i * dE, pikT)); W.append(complex(dE, 0.0))
    if nPol > 0:
        x, w = gauss_fermi_dirac(nFer)
        dE = 30 * kBT
        for xi, wi in zip(x, w):
            E.append(complex(xi * dE, nPol * 2 * pikT)); W.append(complex(wi * dE, 0.0))
    if nPol >= 0:
        for i in range(nPol, 0, -1):
            E.append(complex(0.0, (2 * i - 1) * pikT)); W.append(complex(0.0, -2 * pikT))
    else:
        x, w = gauss_legendre(nFer)
        dE = abs(nPol) * pikT
        for xi, wi in zip(x, w):
            E.append(complex(0.0, (1.0 - xi) * dE)); W.append(complex(0.0, -wi * dE))
    return np.array(E), np.array(W)


def integrate(plan, energies, eweights, kpoints, kweights, dVol, fermi_level=0.0, solve=None, **options):
    """Density of the source cubes integrated over the contour and the k-points:
    rho = Re sum_E w_E sum_k w_k rho_Ek with rho_Ek = diag(G(E, k))/pi from each solve, and the
    response density accumulated as src/energy_contour.cxx:393-399 does (weight -1 for every
    energy point but the last two, normalized by the same sum of energies).
    `solve(E, k)` returns rho_Ek [nCols, 64] (complex); by default the GPU solver on `plan`.
    Returns (rho [nCols, 64], response [nCols, 64], list of per-solve statistics)."""
    from angstromcube_b200 import green_action, green_function as gf
    stats = []
    if solve is None:
        def solve(E, k):
            gf.update_energy_parameter(plan, E, dVol)
            gf.update_phases(plan, k)
            st, r = green_action.solve(plan, **options)
            stats.append(st)
            return r
    nE = len(energies)
    rho_c = None; res_c = None; res_point = 0.0
    for iE, (E0, wE) in enumerate(zip(energies, eweights)):
        E = complex(E0) + fermi_level
        rho_E = None
        for k, wk in zip(kpoints, kweights):
            r = np.asarray(solve(E, np.asarray(k, dtype=float)))
            rho_E = r * wk if rho_E is None else rho_E + r * wk
        rho_c = rho_E * wE if rho_c is None else rho_c + rho_E * wE
        if iE < nE - 2:                      # as the reference accumulates it (its ToDo)
            wgt = 1.0 if iE == nE - 1 else -1.0
            res_c = rho_E * wgt if res_c is None else res_c + rho_E * wgt
            res_point += E * wgt
    res_point = 1.0 / res_point if res_point != 0 else 1.0
    response = (res_c * res_point).real if res_c is not None else np.zeros_like(rho_c.real)
    return rho_c.real, response, stats
