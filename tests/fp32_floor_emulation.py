"""How far FP32 Krylov recurrences get on their own: tfQMR and BiCGStab with every vector
stored and updated in FP32 (complex64), inner products accumulated in FP64, and the
reference's own FP32 action (oracle/_ref, its CPU build), on the CPU-runnable cell (periodic
4^3 cubes, one atom, one source cube, E = -0.3 + 0.05i).  Every 10 iterations the true relative
residual |B - A X| / |B| of the FP32 iterate is computed with the reference's FP64 action and
printed beside the recurrence's own estimate (tfQMR: its QMR bound tau sqrt(m + 1); BiCGStab:
its recursive residual).  Where the true residual stops while the estimate keeps falling, the
recurrence has lost accuracy: the floor that residual replacement and the FP64 continuation of
the mixed solver work around.  With --variants: tfQMR with only the action or only the
vectors in FP32.  No GPU; a minute or two:

    python tests/fp32_floor_emulation.py [--variants]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from angstromcube_b200 import workloads  # noqa: E402


def setup():
    w = workloads.make("periodic4_1atom")
    r = oracle.RefGreen(w.geometry)
    r.set_potential(w.Vcell)
    r.set_atom_matrices(w.mats, w.offsets)
    r.set_energy(w.E, w.dVol)
    ex = r.export()
    ci = np.asarray(ex["colindx"], np.int64)
    nnzb, ncols = r.sizes["nnzb"], r.sizes["nCols"]
    B = np.zeros((nnzb, 64, 64), np.complex128)
    for b in ex["subset"]:
        B[b][np.arange(64), np.arange(64)] = 1.0
    return r, ci, ncols, B


def to_r(z, dtype):
    return np.ascontiguousarray(np.stack([z.real, z.imag], axis=1).astype(dtype))


def to_c(x):
    return x[:, 0] + 1j * x[:, 1]


def run(kind, maxit=300, vec=np.complex64, op32=True):
    """kind "tfqmr" or "bicgstab"; vec: the vectors' type; op32: the FP32 (else FP64) action."""
    r, ci, ncols, B = setup()
    A64 = lambda z: to_c(r.action(to_r(z, np.float64)))
    if op32:
        A32 = lambda z: to_c(r.action(to_r(z, np.float32))).astype(vec)
    else:
        A32 = lambda z: A64(z).astype(vec)

    def dot(a, b):                          # per column, FP64 accumulation
        out = np.zeros((ncols, 64), np.complex128)
        np.add.at(out, ci, (np.conj(a.astype(np.complex128)) * b.astype(np.complex128)).sum(axis=1))
        return out

    def col(s):
        return s[ci][:, None, :].astype(vec)

    def true_res(X):
        R = B - A64(X.astype(np.complex128))
        return float(np.sqrt(dot(R, R).real).max())      # |b| = 1 per column

    rng = np.random.default_rng(7)
    rt = (rng.uniform(-1, 1, B.shape) + 1j * rng.uniform(-1, 1, B.shape)).astype(vec)
    b32 = B.astype(vec)
    X = np.zeros_like(b32)
    hist = []
    if kind == "tfqmr":
        w = b32.copy(); y1 = b32.copy(); v = A32(y1); Ay1 = v.copy(); d = np.zeros_like(b32)
        tau = np.sqrt(dot(b32, b32).real); theta = np.zeros_like(tau); eta = np.zeros((ncols, 64), np.complex128)
        rho = dot(rt, w); m = 0
        for it in range(1, maxit + 1):
            alpha = rho / dot(rt, v)
            y2 = y1 - col(alpha) * v
            Ay2 = None
            for y, Ay in ((y1, Ay1), (y2, None)):
                if Ay is None:
                    Ay = Ay2 = A32(y2)
                m += 1
                w = w - col(alpha) * Ay
                th = np.sqrt(dot(w, w).real) / tau
                c2 = 1.0 / (1.0 + th ** 2)
                d = y + col(theta ** 2 * eta / alpha) * d
                eta = c2 * alpha
                X = X + col(eta) * d
                tau = tau * th * np.sqrt(c2); theta = th
            if it % 10 == 0:
                hist.append((it, true_res(X), float((tau * np.sqrt(m + 1)).max())))
            rho_new = dot(rt, w); beta = rho_new / rho; rho = rho_new
            y1 = w + col(beta) * y2
            Ay1 = A32(y1)
            v = Ay1 + col(beta) * (Ay2 + col(beta) * v)
    else:
        R = b32.copy(); P = R.copy(); rho = dot(rt, R)
        for it in range(1, maxit + 1):
            V = A32(P)
            alpha = rho / dot(rt, V)
            S = R - col(alpha) * V
            T = A32(S)
            omega = dot(T, S) / dot(T, T).real
            X = X + col(alpha) * P + col(omega) * S
            R = S - col(omega) * T
            rho_new = dot(rt, R)
            beta = (rho_new / rho) * (alpha / omega)
            rho = rho_new
            P = R + col(beta) * (P - col(omega) * V)
            if it % 10 == 0:
                hist.append((it, true_res(X), float(np.sqrt(dot(R, R).real).max())))
    return hist


if __name__ == "__main__":
    if "--variants" in sys.argv:
        # which rounding sets the floor: FP64 vectors with the FP32 action, FP32 vectors with the
        # FP64 action, everything FP64
        for name, vec, op32 in (("fp64 vectors, fp32 action", np.complex128, True),
                                ("fp32 vectors, fp64 action", np.complex64, False),
                                ("fp64 vectors, fp64 action", np.complex128, False)):
            h = run("tfqmr", vec=vec, op32=op32)
            print(json.dumps({"variant": name, "floor": min(t for _, t, _ in h),
                              "history": [(it, tr) for it, tr, _ in h]}), flush=True)
        sys.exit(0)
    out = {}
    for kind in ("tfqmr", "bicgstab"):
        h = run(kind)
        out[kind] = h
        for it, tr, est in h:
            print(json.dumps({"solver": kind, "iteration": it, "true_residual": tr, "estimate": est}), flush=True)
    print(json.dumps({"floor": {k: min(t for _, t, _ in h) for k, h in out.items()}}))
