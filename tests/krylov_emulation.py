"""Which Krylov method needs the fewest operator applications on the Green-function systems: a
CPU emulation with the reference's own FP64 action (oracle/_ref), every method right-
preconditioned with the separable cube-diagonal model the GPU solver uses, counting operator
applications until the max over columns of the relative residual is at most 1e-9.

  tfqmr     the reference's method (two applications per iteration), stopped by its QMR bound
            tau sqrt(m + 1) as the GPU solver is; the application count at which its true
            residual first reached the tolerance is printed beside it
  bicgstab  van der Vorst, SIAM J. Sci. Stat. Comput. 13 (1992) 631
  idrS      IDR(S) with biorthogonalization, van Gijzen and Sonneveld, ACM Trans. Math. Softw.
            38 (2011) 5 (Algorithm 913), shadow space of S random vectors orthonormalized per
            system, omega with the angle safeguard kappa = 0.7
  cocg      conjugate orthogonal CG, van der Vorst and Melissen, IEEE Trans. Magn. 26 (1990)
            706, for complex symmetric systems: only at the Gamma point, where the action is
            complex symmetric (u^T A v = v^T A u per column; the Bloch phases break it
            elsewhere), with the symmetric cube-diagonal preconditioner applied as in PCG

Every (source cube, column) pair is its own system with its own scalars, as in the GPU solver.
With --fp32 the vectors are complex64, the action the reference's FP32 one and the
preconditioner FP32 (inner products still accumulated in FP64), and the true FP64 residual of
the iterate is printed every 10 applications beside the method's own residual: where the two
part, the recurrence has lost accuracy (the floor a mixed-precision solver must work around).
No GPU; the CPU-runnable cell (periodic 4^3 cubes, one atom, one source cube) runs in a minute
per energy, the 8^3 cell with eight atoms in tens of minutes per method (some 0.6 s per action):

    python tests/krylov_emulation.py --energy=-0.3+0.05j --kpoint 0.1,0.2,0.3
    python tests/krylov_emulation.py --energy=-0.3+0.05j --kpoint 0,0,0 --methods tfqmr,cocg,idr4
    python tests/krylov_emulation.py --cell periodic8_8atoms_s1x1x1 --energy=-0.3+0.25j \\
        --kpoint 0.1,0,0.2 --methods idr4
    python tests/krylov_emulation.py --fp32 --kpoint 0,0,0 --methods cocg,idr4 --limit 300
    python tests/krylov_emulation.py --fp32 --replace 1e-2 --methods idr4,idr8 --limit 1500
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from fp32_floor_emulation import to_c, to_r  # noqa: E402
from precond_emulation import cell_setup  # noqa: E402


class System:
    """The reference's FP64 action on one cell, energy and k-point, the per-system inner
    products and the separable cube-diagonal preconditioner; counts operator applications."""

    def __init__(self, cell, E, k, fp32=False):
        self.w, self.ref, self.ci, self.ncols, self.B64 = cell_setup(cell, E, k)
        self.real = np.float32 if fp32 else np.float64
        self.cplx = np.complex64 if fp32 else np.complex128
        self.B = self.B64.astype(self.cplx)
        self.history = []                            # (applications, true, recursive) in FP32 runs
        self.replacements = []                       # (applications, true, recursive) at replacements
        self.fp32 = fp32
        ex = self.ref.export()
        veff = ex["veff_index"]
        self.applications = 0
        c8 = np.array([-14350, 8064, -1008, 128]) / 5040.
        D1 = [np.array([[pf * c8[abs(i - j)] for j in range(4)] for i in range(4)])
              for pf in ex["kinetic_prefactor"]]
        lam, Q = zip(*[np.linalg.eigh(d) for d in D1])
        Lsum = (lam[2][:, None, None] + lam[1][None, :, None] + lam[0][None, None, :]).reshape(64)
        self.Q = np.kron(np.kron(Q[2], Q[1]), Q[0]).astype(self.real)
        vbar = np.array([self.w.Vcell[int(c)].mean() if c >= 0 else 0.0 for c in veff])
        self.scale = (1.0 / (Lsum[None, :, None] + vbar[:, None, None] - E)).astype(self.cplx)

    def A(self, z):
        self.applications += 1
        return to_c(self.ref.action(to_r(z, self.real))).astype(self.cplx)

    def M(self, z):
        """M^-1 z: forward transform, scaling, back transform per block (M is complex symmetric)."""
        t = np.einsum("pq,bqc->bpc", self.Q.T, z) * self.scale
        return np.einsum("pq,bqc->bpc", self.Q, t).astype(self.cplx)

    def dot(self, a, b, conj=True):
        """per-system inner products [ncols][64], accumulated in FP64: sum over the system's
        blocks and points"""
        a = a.astype(np.complex128); b = b.astype(np.complex128)
        out = np.zeros((self.ncols, 64), complex)
        np.add.at(out, self.ci, ((np.conj(a) if conj else a) * b).sum(axis=1))
        return out

    def col(self, s):
        """per-system scalars broadcast over the blocks"""
        return s[self.ci][:, None, :].astype(self.cplx)

    def norm(self, R):
        return float(np.sqrt(self.dot(R, R).real).max())

    def true_residual(self, X):
        """max over the systems of |B - A X| with the FP64 action"""
        R = self.B64 - to_c(self.ref.action(to_r(X.astype(np.complex128), np.float64)))
        return self.norm(R)

    def converged(self, X, rnorm, tol):
        """the stopping test on the recursive residual (or estimate) rnorm; FP32 runs also record
        the true residual of X every 10 applications"""
        if self.fp32 and (not self.history or self.applications >= self.history[-1][0] + 10):
            self.history.append((self.applications, self.true_residual(X), rnorm))
        return rnorm <= tol


def tfqmr(S, tol, limit):
    B, dot, col = S.B, S.dot, S.col
    AM = lambda z: S.A(S.M(z))
    rng = np.random.default_rng(7)
    rt = (rng.uniform(-1, 1, B.shape) + 1j * rng.uniform(-1, 1, B.shape)).astype(S.cplx)
    X = np.zeros_like(B); w = B.copy(); y1 = B.copy(); v = AM(y1); Ay1 = v.copy(); d = np.zeros_like(B)
    tau = np.sqrt(dot(B, B).real); theta = np.zeros_like(tau); eta = np.zeros(tau.shape, complex)
    rho = dot(rt, w); m = 0; first = None
    while S.applications < limit:
        alpha = rho / dot(rt, v); y2 = y1 - col(alpha) * v; Ay2 = None
        for y, Ay in ((y1, Ay1), (y2, None)):
            if Ay is None:
                Ay = Ay2 = AM(y2)
            m += 1; w = w - col(alpha) * Ay
            th = np.sqrt(dot(w, w).real) / tau; c2 = 1 / (1 + th ** 2)
            d = y + col(theta ** 2 * eta / alpha) * d; eta = c2 * alpha; X = X + col(eta) * d
            tau = tau * th * np.sqrt(c2); theta = th
        if not S.fp32 and first is None and S.true_residual(S.M(X)) <= tol:
            first = S.applications
        if S.converged(S.M(X) if S.fp32 else X, float((tau * np.sqrt(m + 1)).max()), tol):
            break
        rho_new = dot(rt, w); beta = rho_new / rho; rho = rho_new
        y1 = w + col(beta) * y2; Ay1 = AM(y1); v = Ay1 + col(beta) * (Ay2 + col(beta) * v)
    return S.M(X), {"first_true_below_tol": first}


def bicgstab(S, tol, limit):
    B, dot, col = S.B, S.dot, S.col
    rng = np.random.default_rng(7)
    rt = (rng.uniform(-1, 1, B.shape) + 1j * rng.uniform(-1, 1, B.shape)).astype(S.cplx)
    X = np.zeros_like(B); R = B.copy(); P = R.copy(); rho = dot(rt, R)
    while S.applications < limit:
        Ph = S.M(P); V = S.A(Ph); alpha = rho / dot(rt, V)
        Sv = R - col(alpha) * V
        Sh = S.M(Sv); T = S.A(Sh)
        omega = dot(T, Sv) / dot(T, T).real
        X = X + col(alpha) * Ph + col(omega) * Sh
        R = Sv - col(omega) * T
        if S.converged(X, S.norm(R), tol):
            break
        rho_new = dot(rt, R); beta = (rho_new / rho) * (alpha / omega); rho = rho_new
        P = R + col(beta) * (P - col(omega) * V)
    return X, {}


def idr(S, tol, limit, s=4, kappa=0.7, replace=None):
    """IDR(s); with replace (FP32 runs): the solution is accumulated in FP64 and, at the start of
    a cycle once the recursive residual has fallen by the factor replace since the last
    replacement (or below the tolerance), replaced by the true residual of that solution computed
    with the FP64 action; the run ends when that true residual is below the tolerance.  G, U and
    P^H G are kept across a replacement."""
    B, dot, col = S.B, S.dot, S.col
    rng = np.random.default_rng(7)
    P = [rng.standard_normal(B.shape) + 1j * rng.standard_normal(B.shape) for _ in range(s)]
    for i in range(s):                               # orthonormal shadow space per system
        for j in range(i):
            P[i] = P[i] - dot(P[j], P[i])[S.ci][:, None, :] * P[j]
        P[i] = P[i] / np.sqrt(dot(P[i], P[i]).real)[S.ci][:, None, :]
    P = [p.astype(S.cplx) for p in P]
    shp = (S.ncols, 64)
    X = np.zeros_like(B); R = B.copy()
    G = [np.zeros_like(B) for _ in range(s)]; U = [np.zeros_like(B) for _ in range(s)]
    Mm = np.zeros(shp + (s, s), complex)             # M = P^H G, lower triangular
    for i in range(s):
        Mm[..., i, i] = 1.0
    om = np.ones(shp, complex)
    X64 = np.zeros(B.shape, np.complex128); ref = 1.0
    while S.applications < limit:
        if replace is not None:
            rn = S.norm(R)
            if rn <= replace * ref or rn <= tol:
                X64 = X64 + X.astype(np.complex128); X = np.zeros_like(B)
                Rt = S.B64 - to_c(S.ref.action(to_r(X64, np.float64)))
                S.replacements.append((S.applications, S.norm(Rt), rn))
                ref = S.replacements[-1][1]
                if ref <= tol:
                    break
                R = Rt.astype(S.cplx)
        f = np.stack([dot(P[i], R) for i in range(s)], axis=-1)
        for k in range(s):
            c = np.zeros(shp + (s - k,), complex)    # M[k:, k:] c = f[k:], forward substitution
            for i in range(k, s):
                acc = f[..., i].copy()
                for j in range(k, i):
                    acc -= Mm[..., i, j] * c[..., j - k]
                c[..., i - k] = acc / Mm[..., i, i]
            v = R.copy()
            for i in range(k, s):
                v = v - col(c[..., i - k]) * G[i]
            v = S.M(v)
            Uk = col(om) * v
            for i in range(k, s):
                Uk = Uk + col(c[..., i - k]) * U[i]
            Gk = S.A(Uk)
            for i in range(k):                       # make G_k orthogonal to P_0 .. P_(k-1)
                alpha = dot(P[i], Gk) / Mm[..., i, i]
                Gk = Gk - col(alpha) * G[i]; Uk = Uk - col(alpha) * U[i]
            G[k] = Gk; U[k] = Uk
            for i in range(k, s):
                Mm[..., i, k] = dot(P[i], Gk)
            beta = f[..., k] / Mm[..., k, k]
            R = R - col(beta) * Gk; X = X + col(beta) * Uk
            if replace is None and S.converged(X, S.norm(R), tol):
                return X, {}
            for i in range(k + 1, s):
                f[..., i] -= beta * Mm[..., i, k]
        v = S.M(R); t = S.A(v)                       # the dimension-reduction step
        tt = dot(t, t).real; tr = dot(t, R)
        o = tr / tt
        rho = np.abs(tr) / (np.sqrt(tt) * np.sqrt(dot(R, R).real))
        om = np.where(rho < kappa, o * kappa / np.maximum(rho, 1e-300), o)
        X = X + col(om) * v; R = R - col(om) * t
        if replace is None and S.converged(X, S.norm(R), tol):
            break
    if replace is not None:
        return X64 + X.astype(np.complex128), {"fp64_applications": len(S.replacements),
                                               "replacements": S.replacements}
    return X, {}


def cocg(S, tol, limit):
    B, dot, col = S.B, S.dot, S.col
    X = np.zeros_like(B); R = B.copy(); Z = S.M(R); P = Z.copy(); rho = dot(R, Z, False)
    while S.applications < limit:
        Q = S.A(P); alpha = rho / dot(P, Q, False)
        X = X + col(alpha) * P; R = R - col(alpha) * Q
        if S.converged(X, S.norm(R), tol):
            break
        Z = S.M(R); rho_new = dot(R, Z, False); beta = rho_new / rho; rho = rho_new
        P = Z + col(beta) * P
    return X, {}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cell", default="periodic4_1atom")
    ap.add_argument("--energy", type=complex, default=complex(-0.3, 0.05))
    ap.add_argument("--kpoint", default="0.1,0.2,0.3")
    ap.add_argument("--methods", default="tfqmr,bicgstab,idr4,idr8")
    ap.add_argument("--tolerance", type=float, default=1e-9)
    ap.add_argument("--limit", type=int, default=4000, help="operator applications at most")
    ap.add_argument("--fp32", action="store_true",
                    help="complex64 vectors, the reference's FP32 action and an FP32 preconditioner "
                         "(inner products in FP64); prints the true and recursive residuals every "
                         "10 applications and the lowest true residual (the floor)")
    ap.add_argument("--replace", type=float, default=None,
                    help="with --fp32, IDR(s) with residual replacement: the FP64 true residual "
                         "replaces the recursive one once that has fallen by this factor")
    a = ap.parse_args()
    k = [float(v) for v in a.kpoint.split(",")]
    out = {"cell": a.cell, "E": [a.energy.real, a.energy.imag], "k": k}
    for m in a.methods.split(","):
        S = System(a.cell, a.energy, k, fp32=a.fp32)
        if m == "cocg" and any(k):
            raise SystemExit("cocg needs the Gamma point (the action is complex symmetric only there)")
        if m.startswith("idr"):
            X, extra = idr(S, a.tolerance, a.limit, s=int(m[3:]), replace=a.replace if a.fp32 else None)
        else:
            X, extra = {"tfqmr": tfqmr, "bicgstab": bicgstab, "cocg": cocg}[m](S, a.tolerance, a.limit)
        out[m] = dict(applications=S.applications, true_residual=S.true_residual(X), **extra)
        if a.fp32 and S.history:
            out[m]["floor"] = min(t for _, t, _ in S.history)
            out[m]["history"] = [(n, float("%.3g" % t), float("%.3g" % r)) for n, t, r in S.history]
        print(json.dumps({m: out[m]}), flush=True)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
