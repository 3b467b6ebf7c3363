"""Mixed precision by flexible GMRES: an FP64 FGMRES(m) outer iteration whose preconditioner is
k iterations of FP32 tfQMR (vectors in complex64, FP64 inner products, the reference's FP32
action), on the CPU-runnable cell (periodic 4^3 cubes, one atom, one source cube,
E = -0.3 + 0.05i), every column with its own outer Krylov space.  Prints the true residual
after every restart cycle with the operator applications spent so far, FP32 and FP64, to
compare with plain FP64 tfQMR (216 iterations, 432 FP64 applications, to 1e-9 on this cell).
No GPU; a few minutes:

    python tests/fgmres_fp32_inner_emulation.py 50x4
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from fp32_floor_emulation import setup, to_c, to_r  # noqa: E402


def main(specs):
    r, ci, ncols, B = setup()
    cnt = {"f32": 0, "f64": 0}

    def A32(z):
        cnt["f32"] += 1
        return to_c(r.action(to_r(z, np.float32))).astype(np.complex64)

    def A64(z):
        cnt["f64"] += 1
        return to_c(r.action(to_r(z, np.float64)))

    def dot(a, b):
        out = np.zeros((ncols, 64), np.complex128)
        np.add.at(out, ci, (np.conj(a.astype(np.complex128)) * b.astype(np.complex128)).sum(axis=1))
        return out

    def col(s, dt=np.complex128):
        return s[ci][:, None, :].astype(dt)

    rng = np.random.default_rng(7)
    rt = (rng.uniform(-1, 1, B.shape) + 1j * rng.uniform(-1, 1, B.shape)).astype(np.complex64)

    def tfqmr32(b, k):
        b32 = b.astype(np.complex64)
        X = np.zeros_like(b32)
        w = b32.copy(); y1 = b32.copy(); v = A32(y1); Ay1 = v.copy(); d = np.zeros_like(b32)
        tau = np.sqrt(dot(b32, b32).real); theta = np.zeros_like(tau); eta = np.zeros((ncols, 64), np.complex128)
        rho = dot(rt, w)
        for _ in range(k):
            alpha = rho / dot(rt, v)
            y2 = y1 - col(alpha, np.complex64) * v
            Ay2 = None
            for y, Ay in ((y1, Ay1), (y2, None)):
                if Ay is None:
                    Ay = Ay2 = A32(y2)
                w = w - col(alpha, np.complex64) * Ay
                th = np.sqrt(dot(w, w).real) / tau
                c2 = 1.0 / (1.0 + th ** 2)
                d = y + col(theta ** 2 * eta / alpha, np.complex64) * d
                eta = c2 * alpha
                X = X + col(eta, np.complex64) * d
                tau = tau * th * np.sqrt(c2); theta = th
            rho_new = dot(rt, w); beta = rho_new / rho; rho = rho_new
            y1 = w + col(beta, np.complex64) * y2
            Ay1 = A32(y1)
            v = Ay1 + col(beta, np.complex64) * (Ay2 + col(beta, np.complex64) * v)
        return X

    for k, m in specs:
        cnt["f32"] = cnt["f64"] = 0
        X = np.zeros_like(B)
        hist = []
        for cycle in range(60):
            R = B - A64(X)
            beta = np.sqrt(dot(R, R).real)
            hist.append({"cycle": cycle, "fp32_applications": cnt["f32"], "fp64_applications": cnt["f64"],
                         "true_residual": float(beta.max())})
            if beta.max() <= 1e-9:
                break
            V = [R / col(np.where(beta == 0, 1, beta))]
            Z = []
            H = np.zeros((ncols, 64, m + 1, m), np.complex128)
            for j in range(m):
                z = tfqmr32(V[j], k).astype(np.complex128)
                Z.append(z)
                wv = A64(z)
                for i in range(j + 1):
                    h = dot(V[i], wv)
                    H[:, :, i, j] = h
                    wv = wv - col(h) * V[i]
                hn = np.sqrt(dot(wv, wv).real)
                H[:, :, j + 1, j] = hn
                V.append(wv / col(np.where(hn == 0, 1, hn)))
            Y = np.zeros((ncols, 64, m), np.complex128)
            for c in range(ncols):
                for jj in range(64):
                    e1 = np.zeros(m + 1, np.complex128); e1[0] = beta[c, jj]
                    Y[c, jj] = np.linalg.lstsq(H[c, jj], e1, rcond=None)[0]
            for j in range(m):
                X = X + col(Y[:, :, j]) * Z[j]
        print(json.dumps({"inner_iterations": k, "outer_m": m, "history": hist}), flush=True)


if __name__ == "__main__":
    main([tuple(int(v) for v in s.split("x")) for s in (sys.argv[1:] or ["50x4"])])
