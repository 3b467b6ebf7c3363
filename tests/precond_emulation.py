"""The cube-diagonal preconditioner in a CPU emulation: FP64 tfQMR (numpy, per column) with the
reference's own FP64 action (oracle/_ref), without and with right preconditioning, on the
CPU-runnable cell (periodic 4^3 cubes, one atom, one source cube) at five energies, or with
--cell NAME --energy E [--kpoint kx,ky,kz] on another workload at one energy (the 8^3 cell with
eight atoms and one source cube: hours, at some 0.6 s per action).  Two
preconditioners: the exact local operator of each cube (finite differences inside the cube plus
its potential minus E, inverted densely) and the separable one the solver uses (the cube's mean
potential, applied through the eigenbases of the 4-point difference matrices).  Prints the
iterations to 1e-9 and the true residuals.  No GPU; a few minutes:

    python tests/precond_emulation.py
    python tests/precond_emulation.py --cell periodic8_8atoms_s1x1x1 --energy=-0.3+0.25j --kpoint 0.1,0,0.2
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from fp32_floor_emulation import setup, to_c, to_r  # noqa: E402
from angstromcube_b200 import workloads  # noqa: E402


def cell_setup(name, E, k):
    import oracle
    w = workloads.make(name)
    r = oracle.RefGreen(w.geometry)
    r.set_potential(w.Vcell)
    r.set_atom_matrices(w.mats, w.offsets)
    r.set_energy(E, w.dVol)
    r.set_kpoint(np.asarray(k, dtype=np.float64))
    ex = r.export()
    ci = np.asarray(ex["colindx"], np.int64)
    B = np.zeros((r.sizes["nnzb"], 64, 64), np.complex128)
    for b in ex["subset"]:
        B[b][np.arange(64), np.arange(64)] = 1.0
    return w, r, ci, r.sizes["nCols"], B


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cell", default=None)
    ap.add_argument("--energy", type=complex, default=None)
    ap.add_argument("--kpoint", default="0,0,0")
    a = ap.parse_args()
    energies = (complex(-0.3, 0.05), complex(-0.0066, 0.081), complex(-0.6, 0.49), complex(-0.99, 0.117),
                complex(-0.2, 0.02))
    kpt = [float(v) for v in a.kpoint.split(",")]
    if a.cell:
        energies = (a.energy if a.energy is not None else complex(-0.3, 0.05),)
        w, r, ci, ncols, B = cell_setup(a.cell, energies[0], kpt)
    else:
        r, ci, ncols, B = setup()
        w = workloads.make("periodic4_1atom")
    ex = r.export()
    veff = ex["veff_index"]
    A64 = lambda z: to_c(r.action(to_r(z, np.float64)))

    def dot(a, b):
        out = np.zeros((ncols, 64), np.complex128)
        np.add.at(out, ci, (np.conj(a) * b).sum(axis=1))
        return out

    def col(s):
        return s[ci][:, None, :]

    c8 = np.array([-14350, 8064, -1008, 128]) / 5040.
    D1 = [np.array([[pf * c8[abs(i - j)] for j in range(4)] for i in range(4)]) for pf in ex["kinetic_prefactor"]]
    I4 = np.eye(4)
    T = np.kron(np.kron(I4, I4), D1[0]) + np.kron(np.kron(I4, D1[1]), I4) + np.kron(np.kron(D1[2], I4), I4)
    lam, Q = zip(*[np.linalg.eigh(d) for d in D1])
    Lsum = (lam[2][:, None, None] + lam[1][None, :, None] + lam[0][None, None, :]).reshape(64)
    Qfull = np.kron(np.kron(Q[2], Q[1]), Q[0])

    def tfqmr(A, tol=1e-9, maxit=1500):
        rng = np.random.default_rng(7)
        rt = rng.uniform(-1, 1, B.shape) + 1j * rng.uniform(-1, 1, B.shape)
        X = np.zeros_like(B); wv = B.copy(); y1 = B.copy(); v = A(y1); Ay1 = v.copy(); d = np.zeros_like(B)
        tau = np.sqrt(dot(B, B).real); theta = np.zeros_like(tau); eta = np.zeros((ncols, 64), complex)
        rho = dot(rt, wv); m = 0
        for it in range(1, maxit + 1):
            alpha = rho / dot(rt, v); y2 = y1 - col(alpha) * v; Ay2 = None
            for y, Ay in ((y1, Ay1), (y2, None)):
                if Ay is None:
                    Ay = Ay2 = A(y2)
                m += 1; wv = wv - col(alpha) * Ay
                th = np.sqrt(dot(wv, wv).real) / tau; c2 = 1 / (1 + th ** 2)
                d = y + col(theta ** 2 * eta / alpha) * d; eta = c2 * alpha; X = X + col(eta) * d
                tau = tau * th * np.sqrt(c2); theta = th
            if (tau * np.sqrt(m + 1)).max() <= tol:
                return it, X
            rho_new = dot(rt, wv); beta = rho_new / rho; rho = rho_new
            y1 = wv + col(beta) * y2; Ay1 = A(y1); v = Ay1 + col(beta) * (Ay2 + col(beta) * v)
        return maxit, X

    def true_res(X):
        R = B - A64(X)
        return float(np.sqrt(dot(R, R).real).max())

    for E in energies:
        r.set_energy(E, w.dVol)
        Minv = {}

        def exact(z):
            out = np.empty_like(z)
            for b in range(z.shape[0]):
                c = int(veff[b])
                if c not in Minv:
                    V = w.Vcell[c] if c >= 0 else np.zeros(64)
                    Minv[c] = np.linalg.inv(T + np.diag(V) - E * np.eye(64))
                out[b] = Minv[c] @ z[b]
            return out

        def separable(z):
            out = np.empty_like(z)
            for b in range(z.shape[0]):
                c = int(veff[b]); vbar = w.Vcell[c].mean() if c >= 0 else 0.0
                out[b] = Qfull @ ((Qfull.T @ z[b]) / (Lsum + vbar - E)[:, None])
            return out

        res = {"E": [E.real, E.imag]}
        it, X = tfqmr(A64)
        res["plain"] = [it, true_res(X)]
        for name, P in (("exact", exact), ("separable", separable)):
            it, Y = tfqmr(lambda z: A64(P(z)))
            res[name] = [it, true_res(P(Y))]
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
