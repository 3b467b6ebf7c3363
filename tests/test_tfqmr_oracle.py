"""The numpy tfQMR restatement (oracle/tfqmr.py) against a dense direct solve on a small
block operator: the checker of the GPU solver is itself checked first."""
import numpy as np

from oracle import tfqmr


def test_tfqmr_matches_direct_solve():
    rng = np.random.default_rng(0)
    nnzb, nCols = 3, 2
    colindx = np.array([0, 1, 0])
    subset = np.array([0, 1])
    n = 64 * nnzb
    # a complex symmetric, shifted operator acting on the rows of each column
    M0 = rng.standard_normal((n, n)) * 0.05
    M = M0 + M0.T + np.diag(np.linspace(-1.0, 3.0, n)) - (0.2 + 0.3j) * np.eye(n)
    blocks_of = [np.where(colindx == c)[0] for c in range(nCols)]

    def action(x):
        z = x[:, 0] + 1j * x[:, 1]
        out = np.zeros_like(z)
        for c, bl in enumerate(blocks_of):
            v = z[bl].reshape(-1, 64)                  # rows of this column block
            m = len(bl) * 64
            out[bl] = (M[:m, :m] @ v).reshape(len(bl), 64, 64)
        return np.stack([out.real, out.imag], axis=1)

    X, info = tfqmr.solve_blocks(action, subset, colindx, nnzb, nCols, tol=1e-12, maxiter=400)
    assert info["converged"], info
    Z = X[:, 0] + 1j * X[:, 1]
    for c, bl in enumerate(blocks_of):
        m = len(bl) * 64
        B = np.zeros((m, 64), complex)
        pos = list(bl).index(subset[c])
        B[pos * 64 + np.arange(64), np.arange(64)] = 1
        ref = np.linalg.solve(M[:m, :m], B)
        assert np.abs(Z[bl].reshape(-1, 64) - ref).max() < 1e-9 * np.abs(ref).max()
