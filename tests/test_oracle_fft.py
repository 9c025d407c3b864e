"""Pins the oracle's plane transforms (the restatement of ff2rc / ff2cr)
against numpy-generated golden vectors (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle_ctypes as oc

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "fft_golden.npz"))


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("n", [32, 64, 96, 128])
def test_oracle_r2c(n):
    assert rel(oc.ff2rc(GOLD["r2c_in_%d" % n]), GOLD["r2c_out_%d" % n]) < 1e-13


@pytest.mark.parametrize("n", [32, 64, 96, 128])
def test_oracle_c2r_non_hermitian_input(n):
    assert rel(oc.ff2cr(GOLD["c2r_in_%d" % n], n), GOLD["c2r_out_%d" % n]) < 1e-13


def test_single_mode_known_answer():
    n = 16
    y = np.arange(n)[None, :]
    z = np.arange(n)[:, None]
    a = np.cos(2 * np.pi * (3 * y + 5 * z) / n)[None]
    b = oc.ff2rc(a)[0]
    expect = np.zeros_like(b)
    expect[5, 3] = 0.5
    assert np.max(np.abs(b - expect)) < 1e-15
