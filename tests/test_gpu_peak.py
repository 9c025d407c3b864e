"""The FP64 peak measurement (pibm_fp64_peak) that the bench reports the
step's flop fraction against: a positive rate below the chip's nominal FP64
vector peak plus headroom (B200: 37 TFLOP/s nominal)."""
import ctypes as C

import pytest

import pureibm_ps2d_fd1d_b200 as pk

pytestmark = pytest.mark.gpu


def test_fp64_peak_is_measured():
    lib = pk.load_library()
    tf, ms = C.c_double(), C.c_double()
    assert lib.pibm_fp64_peak(C.byref(tf), C.byref(ms)) == 0
    assert ms.value > 0.0
    assert 1.0 < tf.value < 80.0
