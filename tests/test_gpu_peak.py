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


def _hard_divisors():
    """Divisors whose mantissa is just below 2 (1/b just above a binade
    boundary, the hard case for the one-step correction), next to ordinary ones."""
    k = np.arange(1, 33, dtype=np.float64)
    hard = (2.0 - k * 2.0 ** -52) * np.exp2(np.arange(-16, 16))
    return np.ascontiguousarray(np.concatenate([hard, 1.0 + k * 2.0 ** -52, [3.0, 1.0 / 3.0, 0.05]]))


def _mismatches(a, b):
    lib = pk.load_library()
    bad = C.c_longlong(-1)
    dp = C.POINTER(C.c_double)
    a = np.ascontiguousarray(a)
    assert lib.pibm_qdiv_check(a.ctypes.data_as(dp), len(a), b.ctypes.data_as(dp), len(b), C.byref(bad)) == 0
    return bad.value


def test_reciprocal_division_hard_divisors_and_subnormal_numerators():
    """Normal numerators with normal quotients: bit for bit equal to a / b,
    also for divisors with mantissa 2 - k*2^-52.  Subnormal numerators (or
    quotients): the remainder a - q*b is no longer exact, and about 9% of
    these quotients differ from a / b, by one or two units in the last place
    (bounded on the CPU with the same arithmetic in test_qdiv_cpu.py).  A
    subnormal numerator in a kernel would change that result by those units
    only, far inside the 1e-10 parity bar."""
    rng = np.random.default_rng(11)
    b = _hard_divisors()
    n = 1 << 18
    # numerators 2^-1000..2^1000 over divisors 2^-16..2^16: every quotient normal
    normal = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-1000, 1000, n)) * rng.choice([-1.0, 1.0], n)
    assert _mismatches(normal, b) == 0
    sub = rng.uniform(0.0, 1.0, n) * 2.2250738585072014e-308 * rng.choice([-1.0, 1.0], n)
    bad = _mismatches(sub, b)
    # the same arithmetic on the CPU gives 1,609,582 of these 17,563,648 pairs
    assert bad <= 0.2 * n * len(b), bad

