"""TEST INFRASTRUCTURE ONLY -- tfQMR restated in numpy.

The reference's solver is the external header-only library tfQMRgpu (real-space/tfQMRgpu,
pinned at 572a4aa43fb80677ea9c7a2264d1206ff01df967 in external/CMakeLists.txt:30-39, absent
from the reference tree).  Its published algorithm is Freund's transpose-free QMR
(R. W. Freund, SIAM J. Sci. Comput. 14:470-482, 1993), applied to every column of the block
vector with its own scalars; the reference calls it as tfqmrgpu::solve(action, buffer, 1e-9,
maxiter, 0, true) (include/green_action.hxx:216) with B the unit blocks on the diagonal and
X starting from zero.  This restatement follows Freund's Algorithm 5.1 (Saad, Iterative
Methods for Sparse Linear Systems, Alg. 7.8) half step by half step, unfused.
"""
import numpy as np


def _to_c(x):
    return x[:, 0] + 1j * x[:, 1]


def _to_r(z):
    return np.ascontiguousarray(np.stack([z.real, z.imag], axis=1))


def solve_blocks(action, subset, colindx, nnzb, nCols, tol=1e-9, maxiter=500, seed=7):
    """Solve A X = B for B the unit diagonal blocks.  action(x) maps float64 [nnzb,2,64,64].
    Returns X (float64 blocks) and info {converged, iterations, estimate}."""
    ci = np.asarray(colindx, dtype=np.int64)

    def dot(a, b):                  # per column conj(a) . b  -> [nCols, 64]
        out = np.zeros((nCols, 64), complex)
        np.add.at(out, ci, (np.conj(a) * b).sum(axis=1))
        return out

    def col(s):                     # broadcast per-column scalars to blocks [nnzb, 1, 64]
        return s[ci][:, None, :]

    def A(z):
        return _to_c(action(_to_r(z)))

    B = np.zeros((nnzb, 64, 64), complex)
    for c, b in enumerate(subset):
        B[b][np.arange(64), np.arange(64)] = 1.0
    rng = np.random.default_rng(seed)
    rt = rng.uniform(-1, 1, B.shape) + 1j * rng.uniform(-1, 1, B.shape)
    X = np.zeros_like(B)
    w = B.copy(); y1 = B.copy()                       # w_1 = y_1 = r_0 = b (x_0 = 0)
    v = A(y1); Ay1 = v.copy()                         # v_0 = A y_1
    d = np.zeros_like(B)
    tau = np.sqrt(dot(B, B).real); bnorm = tau.copy()
    theta = np.zeros((nCols, 64)); eta = np.zeros((nCols, 64), complex)
    rho = dot(rt, w)
    active = bnorm > 0
    m = 0
    it = 0
    for it in range(1, maxiter + 1):
        sigma = dot(rt, v)                            # sigma_{n-1}, alpha_{n-1}
        alpha = np.where(active, rho / np.where(sigma == 0, 1, sigma), 0)
        y2 = y1 - col(alpha) * v                      # y_{2n}
        for y, Ay in ((y1, Ay1), (y2, None)):         # half steps m = 2n-1, 2n
            if Ay is None:
                Ay = Ay2 = A(y2)
            m += 1
            w = w - col(alpha) * Ay
            wn = np.sqrt(dot(w, w).real)
            th_new = wn / np.where(tau == 0, 1, tau)
            c2 = 1.0 / (1.0 + th_new ** 2)
            kd = np.where(active, theta ** 2 * eta / np.where(alpha == 0, 1, alpha), 0)
            d = y + col(kd) * d
            eta_new = c2 * alpha
            X = X + col(np.where(active, eta_new, 0)) * d
            tau = np.where(active, tau * th_new * np.sqrt(c2), tau)
            theta = np.where(active, th_new, theta); eta = np.where(active, eta_new, eta)
            active = active & ~(tau * np.sqrt(m + 1) <= tol * bnorm)
        if not active.any():
            break
        rho_new = dot(rt, w)                          # rho_n, beta_n
        beta = np.where(active, rho_new / np.where(rho == 0, 1, rho), 0)
        rho = rho_new
        y1 = w + col(beta) * y2                       # y_{2n+1}
        Ay1 = A(y1)
        v = Ay1 + col(beta) * (Ay2 + col(beta) * v)   # v_n
    est = float((tau * np.sqrt(m + 1) / np.where(bnorm == 0, 1, bnorm)).max())
    return _to_r(X), {"converged": not active.any(), "iterations": it, "estimate": est}


def solve_blocks_torch(action, subset, colindx, nnzb, nCols, tol=1e-9, maxiter=500, seed=7, history_every=0,
                       true_residual=None):
    """The same restatement on torch tensors (any device), for cells too large for numpy loops.
    action(x) maps float64 [nnzb,2,64,64] tensors.  history_every > 0 records, every that many
    iterations, true_residual(X) (a callable) next to the iteration number.  Returns X, info."""
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    ci = torch.as_tensor(np.asarray(colindx, dtype=np.int64), device=dev)

    def to_c(x):
        return torch.complex(x[:, 0], x[:, 1])

    def to_r(z):
        return torch.stack([z.real, z.imag], dim=1).contiguous()

    def dot(a, b):
        out = torch.zeros((nCols, 64), dtype=torch.complex128, device=dev)
        out.index_add_(0, ci, (torch.conj(a) * b).sum(dim=1))
        return out

    def col(s):
        return s[ci][:, None, :]

    def A(z):
        return to_c(action(to_r(z)))

    B = torch.zeros((nnzb, 64, 64), dtype=torch.complex128, device=dev)
    ar = torch.arange(64, device=dev)
    for c, b in enumerate(subset):
        B[int(b), ar, ar] = 1.0
    g = torch.Generator(device=dev).manual_seed(seed)
    rt = torch.complex(torch.rand(B.shape, generator=g, device=dev, dtype=torch.float64) * 2 - 1,
                       torch.rand(B.shape, generator=g, device=dev, dtype=torch.float64) * 2 - 1)
    X = torch.zeros_like(B)
    w = B.clone(); y1 = B.clone()
    v = A(y1); Ay1 = v.clone()
    d = torch.zeros_like(B)
    tau = dot(B, B).real.sqrt(); bnorm = tau.clone()
    theta = torch.zeros_like(tau); eta = torch.zeros_like(tau, dtype=torch.complex128)
    rho = dot(rt, w)
    active = bnorm > 0
    Z = torch.zeros_like(rho)
    one = torch.ones_like(rho)
    m = 0
    it = 0
    hist = []
    for it in range(1, maxiter + 1):
        sigma = dot(rt, v)
        alpha = torch.where(active, rho / torch.where(sigma == 0, one, sigma), Z)
        y2 = y1 - col(alpha) * v
        Ay2 = None
        for y, Ay in ((y1, Ay1), (y2, None)):
            if Ay is None:
                Ay = Ay2 = A(y2)
            m += 1
            w = w - col(alpha) * Ay
            wn = dot(w, w).real.sqrt()
            th_new = wn / torch.where(tau == 0, torch.ones_like(tau), tau)
            c2 = 1.0 / (1.0 + th_new ** 2)
            kd = torch.where(active, theta ** 2 * eta / torch.where(alpha == 0, one, alpha), Z)
            d = y + col(kd) * d
            eta_new = c2 * alpha
            X = X + col(torch.where(active, eta_new, Z)) * d
            tau = torch.where(active, tau * th_new * c2.sqrt(), tau)
            theta = torch.where(active, th_new, theta); eta = torch.where(active, eta_new, eta)
            active = active & ~(tau * np.sqrt(m + 1) <= tol * bnorm)
        if history_every and it % history_every == 0 and true_residual is not None:
            hist.append((it, float(true_residual(to_r(X)))))
        if not bool(active.any()):
            break
        rho_new = dot(rt, w)
        beta = torch.where(active, rho_new / torch.where(rho == 0, one, rho), Z)
        rho = rho_new
        y1 = w + col(beta) * y2
        Ay1 = A(y1)
        v = Ay1 + col(beta) * (Ay2 + col(beta) * v)
    est = float((tau * np.sqrt(m + 1) / torch.where(bnorm == 0, torch.ones_like(bnorm), bnorm)).max())
    return to_r(X), {"converged": not bool(active.any()), "iterations": it, "estimate": est, "history": hist}
