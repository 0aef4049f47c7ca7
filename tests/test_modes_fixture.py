"""The 2-D port-mode fixture (``tests/golden/modes_wr90.npz``, written by
``tests/golden/make_golden.py`` from the reference's Numerical2DModeSolver):
its eigenpairs solve ``K v = lambda M v`` with ``v^T M v = 1`` and are the
lowest above the null-space threshold (checked against a dense float64
eigensolve here, on the CPU)."""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from conftest import GOLDEN


def test_mode_fixture_is_an_eigen_decomposition():
    d = np.load(GOLDEN / "modes_wr90.npz")
    n = d["m"].size
    K = sp.csr_matrix((d["data"], d["indices"], d["indptr"]), shape=(n, n))
    m = d["m"]
    lam, vec = d["eigvals"], d["eigvecs"]
    for q in range(lam.size):
        v = vec[:, q]
        r = K @ v - lam[q] * m * v
        assert np.max(np.abs(r)) <= 1e-9 * lam[q] * np.max(np.abs(m * v))
        assert abs(v @ (m * v) - 1.0) < 1e-12
    A = (K.toarray() / np.sqrt(m)[:, None]) / np.sqrt(m)[None, :]
    w = np.linalg.eigvalsh(A)
    w = w[w > float(d["threshold"])][: lam.size]
    assert np.allclose(w, lam, rtol=1e-10)
