"""The CPU restatements of IDR(s) and COCG in tests/krylov_emulation.py (the algorithms a GPU
solver with fewer operator applications would be checked against) converge on the CPU-runnable
cell with the reference's FP64 action: true residual at most the tolerance, in fewer
applications than tfQMR needs there (196 at k = 0, 288 at k = (0.1, 0.2, 0.3))."""
import numpy as np
import pytest

import krylov_emulation as ke

pytestmark = pytest.mark.timeout(600)


def test_cocg_at_gamma():
    S = ke.System("periodic4_1atom", complex(-0.3, 0.05), [0.0, 0.0, 0.0])
    X, _ = ke.cocg(S, 1e-9, 400)
    assert S.true_residual(X) <= 1.5e-9
    assert S.applications <= 130


def test_idr4_off_gamma():
    S = ke.System("periodic4_1atom", complex(-0.3, 0.05), [0.1, 0.2, 0.3])
    X, _ = ke.idr(S, 1e-9, 400, s=4)
    assert S.true_residual(X) <= 1.5e-9
    assert S.applications <= 200


def test_action_symmetric_only_at_gamma():
    rng = np.random.default_rng(3)
    for k, symmetric in (([0.0, 0.0, 0.0], True), ([0.1, 0.2, 0.3], False)):
        S = ke.System("periodic4_1atom", complex(-0.3, 0.05), k)
        u = rng.standard_normal(S.B.shape) + 1j * rng.standard_normal(S.B.shape)
        v = rng.standard_normal(S.B.shape) + 1j * rng.standard_normal(S.B.shape)
        a, b = S.dot(u, S.A(v), False), S.dot(v, S.A(u), False)
        err = np.abs(a - b).max() / np.abs(a).max()
        assert (err < 1e-13) == symmetric, err
