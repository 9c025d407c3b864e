"""GPU plane transforms (pibm_ff2rc / pibm_ff2cr) against the numpy golden
fixtures and the oracle.  Floating point: relative error <= 1e-13."""
import os

import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "fft_golden.npz"))
TOL = 1e-13


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [32, 64, 96, 128])
def test_ff2rc_matches_golden(n):
    got = pk.ff2rc(GOLD["r2c_in_%d" % n])
    assert rel(got, GOLD["r2c_out_%d" % n]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n", [32, 64, 96, 128])
def test_ff2cr_matches_golden(n):
    got = pk.ff2cr(GOLD["c2r_in_%d" % n], n)
    assert rel(got, GOLD["c2r_out_%d" % n]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 128])
def test_round_trip_many_planes(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((37, n, n))
    back = pk.ff2cr(pk.ff2rc(a), n)
    assert rel(back, a) < TOL
