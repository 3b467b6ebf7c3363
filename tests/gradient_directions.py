"""Adjoint gradients of the contour density objective against central finite differences along
32 seeded directions (8 each for the potential V, the atom Hamiltonian matrices H, the overlap
matrices S and the atom positions R), on the differentiation cell of tests/test_gradients_gpu.py
(the periodic 16^3-cube cell with 64 atoms, numax 5, sigma 0.6, one source cube; 8 energies of
the top arc of the contour with their quadrature weights):

    L = Im sum_E w_E sum_{i in the source cube} W_i G_ii(E).

The gradient is the backward pass of tests/green_autograd.py (adjoint solves at conj(E) and the
vector-Jacobian products of a43g_vjp); each finite difference takes 16 FP64 solves to 1e-12.
Steps: 1e-5 Ha for V, H and S (H and S directions symmetric, every atom's matrices at once),
1e-4 Bohr for R (with the projection radius at 8 sigma, so that no grid point crosses the
cut-off sphere by a visible jump).  A standalone GPU script (about 15 minutes on a B200), not a
pytest case:

    python tests/gradient_directions.py > gradient_directions.log
"""
import copy
import json
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import green_autograd as ga  # noqa: E402
from angstromcube_b200 import workloads  # noqa: E402


def problem():
    w = workloads.make("periodic16_64atoms_s1x1x1")
    E, wE = workloads.contour_semicircle(32)
    top = np.argsort(-E.imag)[:8]
    W = np.random.default_rng(2).uniform(0.5, 1.5, size=(1, 64))
    prob = ga.Problem(w.geometry, E[top], wE[top], W, w.dVol)
    nsho = [workloads.nsho(int(l)) for l in w.geometry.xyzZinso[:, 5]]
    H, S = [], []
    for a, n in enumerate(nsho):
        o = int(w.offsets[a])
        H.append(w.mats[o:o + n * n].reshape(n, n).copy())
        S.append(w.mats[o + n * n:o + 2 * n * n].reshape(n, n).copy())
    return prob, w.Vcell.copy(), H, S, w.geometry.xyzZinso[:, :3].copy()


def main(ndir=8):
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    prob, V, H, S, R = problem()
    L, gV, gH, gS, gR = prob.gradient(V, H, S, R)
    rng = np.random.default_rng(32)
    rows = []

    def central(step, perturb):
        return (prob.value(*perturb(+step)) - prob.value(*perturb(-step))) / (2 * step)

    def report(kind, k, fd, an):
        r = {"kind": kind, "direction": k, "fd": fd, "adjoint": an, "rel_err": abs(fd - an) / abs(an)}
        rows.append(r)
        print(json.dumps(r), flush=True)

    for k in range(ndir):
        D = rng.standard_normal(V.shape)
        report("V", k, central(1e-5, lambda h: (V + h * D, H, S, R)), float(np.sum(D * gV)))
    for kind, grad in (("H", gH), ("S", gS)):
        for k in range(ndir):
            Ds = []
            for m in H:
                d = rng.standard_normal(m.shape)
                Ds.append(0.5 * (d + d.T))

            def perturb(h, kind=kind, Ds=Ds):
                H2 = [x + h * d for x, d in zip(H, Ds)] if kind == "H" else H
                S2 = [x + h * d for x, d in zip(S, Ds)] if kind == "S" else S
                return V, H2, S2, R
            report(kind, k, central(1e-5, perturb), float(sum(np.sum(d * g) for d, g in zip(Ds, grad))))
    prob.geometry = copy.deepcopy(prob.geometry)
    prob.geometry.proj_radius = 8.0
    _, _, _, _, gR8 = prob.gradient(V, H, S, R)
    for k in range(ndir):
        D = rng.standard_normal(R.shape)
        report("R", k, central(1e-4, lambda h: (V, H, S, R + h * D)), float(np.sum(D * gR8)))
    summary = {kind: max(r["rel_err"] for r in rows if r["kind"] == kind) for kind in ("V", "H", "S", "R")}
    print(json.dumps({"max_rel_err": summary, "directions": len(rows), "L": L,
                      "seconds": time.perf_counter() - t0}), flush=True)
    return 0 if max(summary.values()) <= 1e-6 else 1


if __name__ == "__main__":
    sys.exit(main())
