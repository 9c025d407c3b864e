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


def _numpy_pair_256(rng):
    n = 256
    a = rng.standard_normal((3, n, n))
    ky = np.arange(n // 2 + 1)[None, None, :]
    kz = np.minimum(np.arange(n), n - np.arange(n))[None, :, None]
    amp = (1.0 + ky ** 2 + kz ** 2) ** (-5.0 / 6.0)
    b = (rng.standard_normal((3, n, n // 2 + 1)) + 1j * rng.standard_normal((3, n, n // 2 + 1))) * amp
    return a, b


@pytest.mark.gpu
def test_plane_transforms_256_against_numpy():
    """256^2 planes (8-CTA clusters): same conventions as the golden fixtures,
    with numpy computed here."""
    n = 256
    a, b = _numpy_pair_256(np.random.default_rng(256))
    got = pk.ff2rc(a)
    assert rel(got, np.fft.rfft2(a, axes=(1, 2)) / float(np.float32(n * n))) < TOL
    got = pk.ff2cr(b, n)
    assert rel(got, np.fft.irfft2(b, s=(n, n), axes=(1, 2)) * (n * n)) < TOL
    assert rel(pk.ff2cr(pk.ff2rc(a), n), a) < TOL
