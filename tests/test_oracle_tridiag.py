"""Cyclic tridiagonal solve (Thomas + Sherman-Morrison, poisson.F90 /
usteptime.F90) against a dense solve of the periodic system."""
import numpy as np
import pytest

import oracle_ctypes as oc


@pytest.mark.parametrize("n,w2", [(16, 0.3), (64, 2.0), (128, 1e-3)])
def test_cyclic_poisson_matches_dense(n, w2):
    dx2 = 0.05 ** 2
    a = np.full(n, 1 / dx2 - 0.25 * w2)
    b = np.full(n, -2 / dx2 - 0.5 * w2)
    c = a.copy()
    rng = np.random.default_rng(n)
    rr, ri = rng.standard_normal(n), rng.standard_normal(n)
    rc, xr, xi = oc.cyclic_solve(a, b, c, rr, ri)
    assert rc == 0
    A = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
    A[0, -1] = a[0]
    A[-1, 0] = c[-1]
    ref = np.linalg.solve(A, rr + 1j * ri)
    assert np.max(np.abs((xr + 1j * xi) - ref)) / np.max(np.abs(ref)) < 1e-11


def test_cyclic_viscous_matches_dense():
    n = 96
    d = 0.37
    a = np.full(n, -d); c = a.copy(); b = np.full(n, 1 + 2 * d + 0.1)
    rng = np.random.default_rng(1)
    rr, ri = rng.standard_normal(n), rng.standard_normal(n)
    rc, xr, xi = oc.cyclic_solve(a, b, c, rr, ri)
    A = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
    A[0, -1] = a[0]; A[-1, 0] = c[-1]
    ref = np.linalg.solve(A, rr + 1j * ri)
    assert rc == 0 and np.max(np.abs((xr + 1j * xi) - ref)) < 1e-13
