"""The FP64 peak measurement (pibm_fp64_peak) that the bench reports the
step's flop fraction against: a positive rate below the chip's nominal FP64
vector peak plus headroom (B200: 37 TFLOP/s nominal)."""
import ctypes as C

import numpy as np
import pytest

import pureibm_ps2d_fd1d_b200 as pk

pytestmark = pytest.mark.gpu


def test_fp64_peak_is_measured():
    lib = pk.load_library()
    tf, ms = C.c_double(), C.c_double()
    assert lib.pibm_fp64_peak(C.byref(tf), C.byref(ms)) == 0
    assert ms.value > 0.0
    assert 1.0 < tf.value < 80.0


def test_reciprocal_division_equals_the_division():
    """The kernels divide by grid spacings, time-step coefficients and
    eigenvalues through qdiv (reciprocal, then one FMA correction); on the
    device it must give a / b bit for bit over operands spanning 2^-40..2^40,
    both signs and zero."""
    lib = pk.load_library()
    rng = np.random.default_rng(7)
    n = 1 << 21
    a = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-40, 40, n)) * rng.choice([-1.0, 1.0], n)
    a[:4] = [0.0, -0.0, 1.0, -1.0]
    b = np.concatenate([[0.05, 0.0025, 1.0 / 16, 1.5 / 64, 3.0, 1.0 / 3.0],
                        rng.uniform(1.0, 2.0, 58) * np.exp2(rng.integers(-20, 20, 58))])
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    bad = C.c_longlong(-1)
    dp = C.POINTER(C.c_double)
    assert lib.pibm_qdiv_check(a.ctypes.data_as(dp), n, b.ctypes.data_as(dp), len(b), C.byref(bad)) == 0
    assert bad.value == 0
