"""Generate the FFT golden fixtures with numpy (independent FFT, same
conventions as the reference's FFTW calls in SRC/FLO/fftw_interface.F90):

  ff2rc(a) = rfft2 over axes (z, y) with y halved, divided by float(my*mz)
  ff2cr(b) = irfft2 over axes (z, y) times my*mz (FFTW c2r is unnormalised);
             numpy's irfft discards Im of the ky=0 and ky=Nyquist columns after
             the z transform, as FFTW's multi-dimensional c2r does.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    for n in (32, 64, 96, 128):
        a = rng.standard_normal((1, n, n))                     # (plane, z, y)
        out["r2c_in_%d" % n] = a
        out["r2c_out_%d" % n] = np.fft.rfft2(a, axes=(1, 2)) / float(np.float32(n * n))
        # arbitrary (non-Hermitian) half spectrum with k^-5/3-like decay
        ky = np.arange(n // 2 + 1)[None, None, :]
        kz = np.minimum(np.arange(n), n - np.arange(n))[None, :, None]
        amp = (1.0 + ky ** 2 + kz ** 2) ** (-5.0 / 6.0)
        b = (rng.standard_normal((1, n, n // 2 + 1)) + 1j * rng.standard_normal((1, n, n // 2 + 1))) * amp
        out["c2r_in_%d" % n] = b
        out["c2r_out_%d" % n] = np.fft.irfft2(b, s=(n, n), axes=(1, 2)) * (n * n)
    np.savez_compressed(os.path.join(HERE, "fft_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "fft_golden.npz"))


if __name__ == "__main__":
    main()
