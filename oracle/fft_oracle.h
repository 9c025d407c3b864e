// fft_oracle.h -- test infrastructure only (the CPU oracle's FFT).
//
// Restates the semantics of the reference's plane transforms ff2rc / ff2cr
// (SRC/FLO/fftw_interface.F90:48-133 for FFTW 2.1.x, :256-338 for FFTW 3):
//   ff2rc: real a(my,mz) -> complex b(my2,mz), y (first, contiguous) axis halved,
//          forward sign e^{-i}, then b = b / float(my*mz)          (:71-75)
//   ff2cr: complex a(my2,mz) -> real b(my,mz), sign e^{+i}, unnormalised.
// FFTW's multi-dimensional c2r first runs the complex transform along z and
// then a 1-D c2r along y, whose result depends only on the real parts of the
// ky=0 and ky=Nyquist elements; numpy.fft.irfft2 over axes (z, y) has the same
// semantics, which the golden fixtures in tests/golden pin.
// FFTW itself is third-party (prebuilt archives only in the reference tree);
// this is an independent mixed-radix (2,3,4) Stockham autosort FFT.
#pragma once
#include <complex>
#include <vector>
#include <cmath>
#include <cstring>

namespace orc {

typedef std::complex<double> cplx;

// Complex DFT of length n = 2^a 3^b with sign s (-1 forward, +1 inverse), unnormalised.
class CFFT {
public:
    int n = 0;
    double sign = -1;
    std::vector<cplx> w;        // w[k] = exp(sign*2*pi*i*k/n)
    std::vector<int> radices;
    void init(int n_, int sign_) {
        n = n_; sign = sign_;
        w.resize(n);
        for (int k = 0; k < n; ++k) {
            long double ang = (long double)sign_ * 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
            w[k] = cplx((double)cosl(ang), (double)sinl(ang));
        }
        radices.clear();
        int m = n;
        while (m % 4 == 0) { radices.push_back(4); m /= 4; }
        while (m % 2 == 0) { radices.push_back(2); m /= 2; }
        while (m % 3 == 0) { radices.push_back(3); m /= 3; }
        if (m != 1) radices.clear(), radices.push_back(-1);  // unsupported length
    }
    bool ok() const { return radices.empty() || radices[0] != -1; }
    // In-place on x using scratch y (both length n).
    void run(cplx *x, cplx *y) const {
        int len = n, s = 1;
        cplx *src = x, *dst = y;
        const double s3 = sign * 0.86602540378443864676372317075293618;  // sign*sqrt(3)/2
        for (size_t st = 0; st < radices.size(); ++st) {
            const int p = radices[st];
            const int m = len / p;
            const int tw = n / len;           // w_len^j = w[j*tw]
            for (int pi = 0; pi < m; ++pi) {
                for (int q = 0; q < s; ++q) {
                    if (p == 2) {
                        cplx a0 = src[q + s * (pi + 0 * m)];
                        cplx a1 = src[q + s * (pi + 1 * m)];
                        dst[q + s * (2 * pi + 0)] = a0 + a1;
                        dst[q + s * (2 * pi + 1)] = (a0 - a1) * w[(pi * tw) % n];
                    } else if (p == 4) {
                        cplx a0 = src[q + s * (pi + 0 * m)];
                        cplx a1 = src[q + s * (pi + 1 * m)];
                        cplx a2 = src[q + s * (pi + 2 * m)];
                        cplx a3 = src[q + s * (pi + 3 * m)];
                        cplx t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = a1 - a3;
                        // multiply t3 by (sign * i)
                        cplx jt3 = cplx(-sign * t3.imag(), sign * t3.real());
                        cplx b0 = t0 + t2, b1 = t1 + jt3, b2 = t0 - t2, b3 = t1 - jt3;
                        dst[q + s * (4 * pi + 0)] = b0;
                        dst[q + s * (4 * pi + 1)] = b1 * w[(1 * pi * tw) % n];
                        dst[q + s * (4 * pi + 2)] = b2 * w[(2 * pi * tw) % n];
                        dst[q + s * (4 * pi + 3)] = b3 * w[(3 * pi * tw) % n];
                    } else {  // p == 3
                        cplx a0 = src[q + s * (pi + 0 * m)];
                        cplx a1 = src[q + s * (pi + 1 * m)];
                        cplx a2 = src[q + s * (pi + 2 * m)];
                        cplx t1 = a1 + a2, t2 = a1 - a2;
                        cplx b0 = a0 + t1;
                        cplx c = a0 - 0.5 * t1;
                        cplx jt2 = cplx(-s3 * t2.imag(), s3 * t2.real());
                        cplx b1 = c + jt2, b2 = c - jt2;
                        dst[q + s * (3 * pi + 0)] = b0;
                        dst[q + s * (3 * pi + 1)] = b1 * w[(1 * pi * tw) % n];
                        dst[q + s * (3 * pi + 2)] = b2 * w[(2 * pi * tw) % n];
                    }
                }
            }
            len = m; s *= p;
            std::swap(src, dst);
        }
        if (src != x) std::memcpy(x, src, sizeof(cplx) * n);
    }
};

// 2-D plane transforms with the reference's conventions.
class PlaneFFT {
public:
    int my = 0, mz = 0, my2 = 0;
    CFFT fy, by, fz, bz;
    std::vector<cplx> row, rs, col, cs, work;
    void init(int my_, int mz_) {
        my = my_; mz = mz_; my2 = my / 2 + 1;
        fy.init(my, -1); by.init(my, +1); fz.init(mz, -1); bz.init(mz, +1);
        row.resize(my); rs.resize(my); col.resize(mz); cs.resize(mz);
        work.resize((size_t)my2 * mz);
    }
    // a: real (my, mz) y fastest; b: complex (my2, mz) y fastest.
    void r2c(const double *a, cplx *b) {
        for (int k = 0; k < mz; ++k) {
            for (int j = 0; j < my; ++j) row[j] = cplx(a[j + (size_t)my * k], 0.0);
            fy.run(row.data(), rs.data());
            for (int j = 0; j < my2; ++j) work[j + (size_t)my2 * k] = row[j];
        }
        const double nrm = (double)(float)(my * mz);
        for (int j = 0; j < my2; ++j) {
            for (int k = 0; k < mz; ++k) col[k] = work[j + (size_t)my2 * k];
            fz.run(col.data(), cs.data());
            for (int k = 0; k < mz; ++k) b[j + (size_t)my2 * k] = col[k] / nrm;
        }
    }
    // a: complex (my2, mz); b: real (my, mz).
    void c2r(const cplx *a, double *b) {
        for (int j = 0; j < my2; ++j) {
            for (int k = 0; k < mz; ++k) col[k] = a[j + (size_t)my2 * k];
            bz.run(col.data(), cs.data());
            for (int k = 0; k < mz; ++k) work[j + (size_t)my2 * k] = col[k];
        }
        for (int k = 0; k < mz; ++k) {
            const cplx *g = &work[(size_t)my2 * k];
            row[0] = cplx(g[0].real(), 0.0);
            for (int j = 1; j < my2 - 1; ++j) { row[j] = g[j]; row[my - j] = std::conj(g[j]); }
            row[my / 2] = cplx(g[my / 2].real(), 0.0);
            by.run(row.data(), rs.data());
            for (int j = 0; j < my; ++j) b[j + (size_t)my * k] = row[j].real();
        }
    }
};

}  // namespace orc
